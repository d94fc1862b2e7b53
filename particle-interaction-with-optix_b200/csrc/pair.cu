// pair.cu -- the interaction stage on the device.
//
// k_pair_compat replaces ComputeParticleInterationsParPartNoLoop
// (cudaLJ.cu:299-341) with the reference's law and stencil: every particle of
// the clamped 27-cell block except itself, r = sqrt(d.d + 1e-5), IEEE sqrt and
// division, 4 eps ((1/r)^12 - (1/r)^6) with eps = sigma = 1, no cutoff.  The 27
// cells are read as 9 rows of 3 consecutive cells, contiguous in cell order,
// and positions come as one float4 load instead of three scalar loads.
//
// k_pair_config evaluates the truncated law with forces.  One thread per
// sorted target particle.  For each of the 9 stencil rows it bounds the
// squared distance from the target to the row in (y, z); rows that cannot
// hold a partner are skipped, and, when particles are x-sorted within cells
// (LJ_ORDER_X, so every row of 3 cells is x-sorted), binary search narrows
// the row to the x-window [x - h, x + h], h = sqrt(rc^2 - dyz^2) plus a
// rounding slack.  The windows are a superset of the interacting partners,
// so the shared float distance test alone decides, and the pair count is
// exact.  Pair math is FP32 from r^-2 (one approximate reciprocal), sums are
// accumulated in registers, and the totals (energy, virial, pair count) are
// reduced in FP64 / u64 per block and then by the last block in a fixed
// order, so they are deterministic.
#include <cfloat>

#include "pair_common.cuh"

namespace ljc {

constexpr double kPairCell = 2.0;    // particles per cell from which the default takes two targets per lane

// Default pair kernel for LJ_ORDER_X (measured on B200, 10M particles): the packed row passes with two
// targets per lane (kernel 10) from 2 particles per cell up (10 per cell: 2.38 ms against 2.88 ms for
// one target per lane; 80 per cell: 11.9 ms against 12.6 ms for the SoA walk); below, one target per
// lane (0.5 per cell: 0.45 ms against 0.48 ms), where the merged windows of two targets add more
// candidates than the shared loads save.
int default_pair_kernel(int n, const lj_grid& g) {
    return (double)n / ((double)g.dim[0] * g.dim[1] * g.dim[2]) >= kPairCell ? 10 : 6;
}

template <bool XWIN>
__global__ void __launch_bounds__(kPairThreads) k_pair_config(GridDev g, PairParams pp, const float4* __restrict__ p,
                                                              const int* __restrict__ cs,
                                                              const int* __restrict__ off, int n, int kb, int ke,
                                                              float* __restrict__ energy, float* __restrict__ force,
                                                              Partial* part, unsigned* counter, lj_totals* totals,
                                                              unsigned* status) {
    __shared__ int2 s_win[kMaxWin][kPairThreads];
    const int k = kb + blockIdx.x * kPairThreads + threadIdx.x;   // targets [kb, ke) of the n sorted particles
    float ea = 0.f, fx = 0.f, fy = 0.f, fz = 0.f, wa = 0.f;
    unsigned np = 0;
    if (k < ke) {
        int c = cs[k];
        if (c < 0 || c >= g.gx * g.gy * g.gz) {
            atomicOr(status, kFlagRange);
            c = 0;
        }
        pair_target<XWIN, kPairThreads>(g, pp, p, off, n, k, c, s_win, ea, fx, fy, fz, wa, np);
        if (energy) energy[k] = pp.e4 * ea;
        if (force) {
            force[3 * (size_t)k + 0] = pp.fscale * fx;
            force[3 * (size_t)k + 1] = pp.fscale * fy;
            force[3 * (size_t)k + 2] = pp.fscale * fz;
        }
    }
    reduce_totals<kPairThreads>(0.5 * (double)pp.e4 * (double)ea, 0.5 * (double)pp.e24 * (double)wa,
                                (unsigned long long)np, part, counter, totals);
}

__global__ void __launch_bounds__(kPairThreads) k_pair_compat(GridDev g, const float4* __restrict__ p,
                                                              const int* __restrict__ cs,
                                                              const int* __restrict__ off, int n,
                                                              float* __restrict__ v, unsigned* status) {
    const int k = blockIdx.x * kPairThreads + threadIdx.x;
    if (k >= n) return;
    const float4 pi = p[k];
    int c = cs[k];
    if (c < 0 || c >= g.gx * g.gy * g.gz) {
        atomicOr(status, kFlagRange);
        c = 0;
    }
    int cx, cy, cz;
    decode_cell(g, c, cx, cy, cz);
    const int xl = max(cx - 1, 0), xh = min(cx + 1, g.gx - 1);
    float pot = 0.f;
    for (int z = max(cz - 1, 0); z <= min(cz + 1, g.gz - 1); ++z)
        for (int y = max(cy - 1, 0); y <= min(cy + 1, g.gy - 1); ++y) {
            const int rb = (z * g.gy + y) * g.gx;
            const int s = min(max(__ldg(&off[rb + xl]), 0), n);
            const int e = min(max(__ldg(&off[rb + xh + 1]), s), n);
            for (int j = s; j < e; ++j) {
                if (j == k) continue;
                const float4 q = __ldg(&p[j]);
                const float dx = q.x - pi.x, dy = q.y - pi.y, dz = q.z - pi.z;
                const float r = sqrtf(dx * dx + dy * dy + dz * dz + 1e-5f);
                const float sdr = 1.0f / r;
                const float r6 = (sdr * sdr) * (sdr * sdr) * (sdr * sdr);
                const float r12 = r6 * r6;
                pot += 4.0f * (r12 - r6);
            }
        }
    v[k] = pot;
}

float grid_slack(const lj_grid& g) {
    float m = 0.f;
    for (int d = 0; d < 3; ++d) {
        const float a = fabsf(g.origin[d]) + (float)g.dim[d] * g.width;
        m = a > m ? a : m;
    }
    return 8.0f * FLT_EPSILON * (m + g.width) + 1e-30f;
}

lj_status launch_pair_config(lj_ctx* ctx, const lj_grid* g, const lj_params* prm, int n, const float* xyzi,
                             const int* cs, const int* off, lj_order order, float* energy, float* force,
                             lj_totals* totals, int kb, int ke) {
    if (ke < 0) ke = n;
    if (kb < 0 || kb > ke || ke > n) return LJ_EINVAL;
    if (kb == ke) {
        if (totals && cudaMemsetAsync(totals, 0, sizeof(lj_totals), ctx->stream) != cudaSuccess) return LJ_ECUDA;
        return LJ_OK;
    }
    PairParams pp;
    pp.rc2 = prm->cutoff * prm->cutoff;
    pp.rc2w = pp.rc2 * (1.0f + 1e-5f);
    pp.sig2 = prm->sigma * prm->sigma;
    pp.e4 = 4.0f * prm->epsilon;
    pp.e24 = 24.0f * prm->epsilon;
    pp.fscale = -pp.e24 / pp.sig2;
    pp.slack = grid_slack(*g);
    if (order == LJ_ORDER_X) {
        int kernel = ctx->tuning.pair_kernel;
        if (kernel == 0) kernel = default_pair_kernel(n, *g);
        switch (kernel) {
            case 4:  // cell-block tiles cover whole target ranges only; a sub-range runs kernel 1
                if (kb == 0 && ke == n) return launch_pair_tiled(ctx, g, pp, n, xyzi, off, energy, force, totals);
                break;
            case 7: return launch_pair_pass(ctx, g, pp, n, xyzi, cs, off, 2, energy, force, totals, kb, ke);
            case 8: return launch_pair_pass(ctx, g, pp, n, xyzi, cs, off, 3, energy, force, totals, kb, ke);
            case 9: return launch_pair_pass(ctx, g, pp, n, xyzi, cs, off, 4, energy, force, totals, kb, ke);
            case 10: return launch_pair_pass(ctx, g, pp, n, xyzi, cs, off, 5, energy, force, totals, kb, ke);
            case 6: return launch_pair_pass(ctx, g, pp, n, xyzi, cs, off, 1, energy, force, totals, kb, ke);
            case 5: return launch_pair_pass(ctx, g, pp, n, xyzi, cs, off, 0, energy, force, totals, kb, ke);
            case 3: return launch_pair_direct(ctx, g, pp, n, xyzi, cs, off, true, energy, force, totals, kb, ke);
            case 2: return launch_pair_direct(ctx, g, pp, n, xyzi, cs, off, false, energy, force, totals, kb, ke);
            default: break;  // 1: windows in shared memory (below)
        }
    }
    const int blocks = (ke - kb + kPairThreads - 1) / kPairThreads;
    const size_t need = 256 + (size_t)blocks * sizeof(Partial);
    if (need > ctx->red_bytes) {
        lj_status s = grow(&ctx->red, &ctx->red_bytes, need);
        if (s != LJ_OK) return s;
        if (cudaMemsetAsync(ctx->red, 0, 256, ctx->stream) != cudaSuccess) return LJ_ECUDA;
    }
    unsigned* counter = static_cast<unsigned*>(ctx->red);
    Partial* part = reinterpret_cast<Partial*>(static_cast<char*>(ctx->red) + 256);
    const float4* p4 = reinterpret_cast<const float4*>(xyzi);
    if (order == LJ_ORDER_X)
        k_pair_config<true><<<blocks, kPairThreads, 0, ctx->stream>>>(to_dev(*g), pp, p4, cs, off, n, kb, ke, energy,
                                                                      force, part, counter, totals, ctx->d_status);
    else
        k_pair_config<false><<<blocks, kPairThreads, 0, ctx->stream>>>(to_dev(*g), pp, p4, cs, off, n, kb, ke,
                                                                       energy, force, part, counter, totals,
                                                                       ctx->d_status);
    return last_launch_status();
}

}  // namespace ljc

using namespace ljc;

extern "C" lj_status lj_compute_compat(lj_ctx* ctx, const lj_grid* g, int n, const float* sorted_xyzi,
                                       const int* sorted_cell, const int* offsets, float* v) {
    if (!ctx || !g || n < 0 || (n > 0 && (!sorted_xyzi || !sorted_cell || !offsets || !v))) return LJ_EINVAL;
    if (!(g->width > 0.0f) || g->dim[0] < 1 || g->dim[1] < 1 || g->dim[2] < 1) return LJ_EINVAL;
    if (reinterpret_cast<uintptr_t>(sorted_xyzi) & 15) return LJ_EINVAL;
    if (n == 0) return LJ_OK;
    k_pair_compat<<<(n + kPairThreads - 1) / kPairThreads, kPairThreads, 0, ctx->stream>>>(
        to_dev(*g), reinterpret_cast<const float4*>(sorted_xyzi), sorted_cell, offsets, n, v, ctx->d_status);
    return last_launch_status();
}

extern "C" lj_status lj_compute(lj_ctx* ctx, const lj_grid* g, const lj_params* p, int n, const float* sorted_xyzi,
                                const int* sorted_cell, const int* offsets, lj_order order, float* energy,
                                float* force, lj_totals* totals) {
    if (!ctx || !g || !p || n < 0) return LJ_EINVAL;
    if (n > 0 && (!sorted_xyzi || !sorted_cell || !offsets)) return LJ_EINVAL;
    if (!(g->width > 0.0f) || g->dim[0] < 1 || g->dim[1] < 1 || g->dim[2] < 1) return LJ_EINVAL;
    if (!(p->cutoff > 0.0f) || !(p->cutoff <= g->width) || !(p->sigma > 0.0f)) return LJ_EINVAL;
    if (order != LJ_ORDER_INDEX && order != LJ_ORDER_X) return LJ_EINVAL;
    if (reinterpret_cast<uintptr_t>(sorted_xyzi) & 15) return LJ_EINVAL;
    return launch_pair_config(ctx, g, p, n, sorted_xyzi, sorted_cell, offsets, order, energy, force, totals, 0, n);
}

extern "C" lj_status lj_autotune_compute(lj_ctx* ctx, const lj_grid* g, const lj_params* p, int n,
                                         const float* sorted_xyzi, const int* sorted_cell, const int* offsets,
                                         int* best_kernel, float* best_ms) {
    if (!ctx || !g || !p || n < 1 || !sorted_xyzi || !sorted_cell || !offsets) return LJ_EINVAL;
    const lj_tuning saved = ctx->tuning;
    cudaEvent_t e0, e1;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) return LJ_ECUDA;
    int best = 1;
    float bt = 3.4e38f;
    lj_status st = LJ_OK;
    static const int kCandidates[] = {1, 2, 3, 5, 6, 7, 8, 9, 10};
    for (int ki = 0; ki < 9 && st == LJ_OK; ++ki) {
        const int k = kCandidates[ki];
        ctx->tuning.pair_kernel = k;
        float ms = 3.4e38f;
        for (int r = 0; r < 3 && st == LJ_OK; ++r) {  // the first run warms up
            float one = 0.f;
            if (cudaEventRecord(e0, ctx->stream) != cudaSuccess) st = LJ_ECUDA;
            if (st == LJ_OK)
                st = lj_compute(ctx, g, p, n, sorted_xyzi, sorted_cell, offsets, LJ_ORDER_X, nullptr, nullptr,
                                nullptr);
            if (st == LJ_OK && (cudaEventRecord(e1, ctx->stream) != cudaSuccess ||
                                cudaEventSynchronize(e1) != cudaSuccess ||
                                cudaEventElapsedTime(&one, e0, e1) != cudaSuccess))
                st = LJ_ECUDA;
            if (r > 0 && one < ms) ms = one;
        }
        if (st == LJ_OK && ms < bt) {
            bt = ms;
            best = k;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    ctx->tuning = saved;
    if (st != LJ_OK) return st;
    ctx->tuning.pair_kernel = best;
    if (best_kernel) *best_kernel = best;
    if (best_ms) *best_ms = bt;
    return lj_sync(ctx);
}
