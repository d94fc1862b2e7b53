// pair_pass.cu -- single-system kernel of the warp-synchronous row passes
// (the walk itself is in pair_pass.cuh).
#include "pair_pass.cuh"

namespace ljc {

namespace {
constexpr int kPassThreads = 128;
}  // namespace

// One thread per target of [kb, ke) (pass_target).
__global__ void __launch_bounds__(kPassThreads) k_pair_pass(GridDev g, PairParams pp, const float4* __restrict__ p,
                                                            const int* __restrict__ cs, const int* __restrict__ off,
                                                            int n, int kb, int ke, float* __restrict__ energy,
                                                            float* __restrict__ force, Partial* part,
                                                            unsigned* counter, lj_totals* totals, unsigned* status) {
    const int k = kb + blockIdx.x * kPassThreads + threadIdx.x;
    const bool active = k < ke;
    int c = 0;
    if (active) {
        c = __ldg(&cs[k]);
        if (c < 0 || c >= g.gx * g.gy * g.gz) {
            atomicOr(status, kFlagRange);
            c = 0;
        }
    }
    PassAcc a;
    pass_target(g, pp, p, off, 0, n, k, c, active, a);
    const float ea = a.e.x + a.e.y, wa = a.w.x + a.w.y;
    const int o = active ? out_slot(pp, p, k, n, status) : -1;
    if (o >= 0) {
        if (energy) energy[o] = pp.e4 * ea;
        if (force) {
            const float nf = -pp.fscale;
            force[3 * (size_t)o + 0] = nf * (a.fx.x + a.fx.y);
            force[3 * (size_t)o + 1] = nf * (a.fy.x + a.fy.y);
            force[3 * (size_t)o + 2] = nf * (a.fz.x + a.fz.y);
        }
    }
    reduce_totals<kPassThreads>(0.5 * (double)pp.e4 * (double)ea, 0.5 * (double)pp.e24 * (double)wa,
                                (unsigned long long)a.np, part, counter, totals);
}

// Two targets per thread (pass_target2): thread t of the launch takes targets kb + 2t and kb + 2t + 1;
// registers capped for 8 blocks per SM, the windows parked in shared memory during the walk.
template <int BLOCK = kPassThreads>
__global__ void __launch_bounds__(BLOCK, 8) k_pair_pass2(GridDev g, PairParams pp, const float4* __restrict__ p,
                                                             const int* __restrict__ cs, const int* __restrict__ off,
                                                             int n, int kb, int ke, float* __restrict__ energy,
                                                             float* __restrict__ force, Partial* part,
                                                             unsigned* counter, lj_totals* totals, unsigned* status) {
    const int ka = kb + 2 * (blockIdx.x * BLOCK + threadIdx.x);
    const bool activeA = ka < ke, activeB = ka + 1 < ke;
    const int ncell = g.gx * g.gy * g.gz;
    int ca = 0, cb = 0;
    if (activeA) {
        ca = __ldg(&cs[ka]);
        if (ca < 0 || ca >= ncell) {
            atomicOr(status, kFlagRange);
            ca = 0;
        }
    }
    if (activeB) {
        cb = __ldg(&cs[ka + 1]);
        if (cb < 0 || cb >= ncell) {
            atomicOr(status, kFlagRange);
            cb = 0;
        }
    }
    Pass2Acc a;
    __shared__ int2 s_win[9][BLOCK];
    pass_target2<BLOCK>(g, pp, p, off, 0, n, ka, ca, cb, activeA, activeB, a, s_win);
    const float nf = -pp.fscale;
    const int oa = activeA ? out_slot(pp, p, ka, n, status) : -1;
    const int ob = activeB ? out_slot(pp, p, ka + 1, n, status) : -1;
    if (oa >= 0) {
        if (energy) energy[oa] = pp.e4 * a.e.x;
        if (force) {
            force[3 * (size_t)oa + 0] = nf * a.fx.x;
            force[3 * (size_t)oa + 1] = nf * a.fy.x;
            force[3 * (size_t)oa + 2] = nf * a.fz.x;
        }
    }
    if (ob >= 0) {
        if (energy) energy[ob] = pp.e4 * a.e.y;
        if (force) {
            force[3 * (size_t)ob + 0] = nf * a.fx.y;
            force[3 * (size_t)ob + 1] = nf * a.fy.y;
            force[3 * (size_t)ob + 2] = nf * a.fz.y;
        }
    }
    reduce_totals<BLOCK>(0.5 * (double)pp.e4 * ((double)a.e.x + (double)a.e.y),
                         0.5 * (double)pp.e24 * ((double)a.w.x + (double)a.w.y), (unsigned long long)a.np, part,
                         counter, totals);
}

lj_status launch_pair_pass(lj_ctx* ctx, const lj_grid* g, const PairParams& pp, int n, const float* xyzi,
                           const int* cs, const int* off, bool two, float* energy, float* force, lj_totals* totals,
                           int kb, int ke) {
    const int per_block = two ? 2 * kPassThreads : kPassThreads;
    const int blocks = (ke - kb + per_block - 1) / per_block;
    const size_t need = 256 + (size_t)blocks * sizeof(Partial);
    if (need > ctx->red_bytes) {
        lj_status s = grow(&ctx->red, &ctx->red_bytes, need);
        if (s != LJ_OK) return s;
        if (cudaMemsetAsync(ctx->red, 0, 256, ctx->stream) != cudaSuccess) return LJ_ECUDA;
    }
    unsigned* counter = static_cast<unsigned*>(ctx->red);
    Partial* part = reinterpret_cast<Partial*>(static_cast<char*>(ctx->red) + 256);
    const float4* p4 = reinterpret_cast<const float4*>(xyzi);
    const GridDev gd = to_dev(*g);
    if (two)
        k_pair_pass2<><<<blocks, kPassThreads, 0, ctx->stream>>>(gd, pp, p4, cs, off, n, kb, ke, energy, force, part,
                                                                counter, totals, ctx->d_status);
    else
        k_pair_pass<<<blocks, kPassThreads, 0, ctx->stream>>>(gd, pp, p4, cs, off, n, kb, ke, energy, force, part,
                                                              counter, totals, ctx->d_status);
    return last_launch_status();
}

}  // namespace ljc
