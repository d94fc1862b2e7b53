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

// ---------------------------------------------------------------- kernel 12: cell pairs, whole rows
// On sparse grids (a sphere shell: 1% of the cells occupied, about 6 particles each) consecutive
// targets 2m, 2m + 1 often lie in different cells, so kernel 10's merged windows mix two stencils and
// a lane whose targets lie in different rows takes a second sweep; and the x-window searches cost
// more than the few candidates of a sparse row they remove.  Here the targets are paired inside
// their cell instead: target k of [kb, ke) opens a pair when its rank among the range's targets of
// its cell is even, and takes k + 1 as its partner when k + 1 is in the same cell.  Both targets then
// have the same 27-cell stencil, so its non-empty rows are walked whole, end to end, each candidate
// loaded once and evaluated against both targets in paired FP32 (eval2), with no window search and
// no second sweep.  The lanes take the pairs from a list built on the device: flags, their exclusive
// scan (k_scan), and the list; so a lane's targets are consecutive in sorted order and the warp's 32
// pairs cover a few neighbouring cells.  The distance test and the pair count are those of every other
// kernel; per-target sums run in a different order (FP32 tolerance).  A target's sums do not depend on
// its partner (each half of a paired operation rounds as the scalar one), so a range of targets gives
// the bits of the whole launch.  Measured on B200 (4M sphere shell, 64M cells, rc = 0.005): 0.517 ms
// with the list against 0.597 ms for kernel 11; the 5 lockstep passes of kernel 10 over the same whole
// rows took 0.593 ms (each pass waits for its own longest lane: 70% of the lanes' steps are useful
// against 88% for one pass).

// Flag of target k: 1 when it opens a pair (even rank among the range's targets of its cell).
__global__ void __launch_bounds__(256) k_cellpair_flags(const int* __restrict__ cs, const int* __restrict__ off,
                                                        int ncell, int kb, int ke, int* __restrict__ flag,
                                                        unsigned* status) {
    for (int k = kb + blockIdx.x * blockDim.x + threadIdx.x; k < ke; k += gridDim.x * blockDim.x) {
        const int c = __ldg(&cs[k]);
        int f = 1;  // a target whose cell id is out of range stays alone (and is reported)
        if (c < 0 || c >= ncell) {
            atomicOr(status, kFlagRange);
        } else {
            const int s = min(max(__ldg(&off[c]), kb), k);
            f = ((k - s) & 1) == 0 ? 1 : 0;
        }
        flag[k - kb] = f;
    }
}

// list[pos[i]] = kb + i for every flagged i: the pairs' first targets in sorted order.
__global__ void __launch_bounds__(256) k_cellpair_list(const int* __restrict__ flag, const int* __restrict__ pos,
                                                       int nk, int kb, int* __restrict__ list) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nk; i += gridDim.x * blockDim.x) {
        const int q = pos[i];
        if (flag[i] && q >= 0 && q < nk) list[q] = kb + i;
    }
}

// One lane per pair: list[t] = a, b = a + 1 when in a's cell.  npairs is read on the device (pos[nk],
// at most nk); the grid covers nk lanes, the most pairs there can be.
template <int BLOCK = kPassThreads>
__global__ void __launch_bounds__(BLOCK, 8) k_pair_cellpair(GridDev g, PairParams pp, const float4* __restrict__ p,
                                                            const int* __restrict__ cs, const int* __restrict__ off,
                                                            int n, int nk, int ke, const int* __restrict__ list,
                                                            const int* __restrict__ npairs_p,
                                                            float* __restrict__ energy, float* __restrict__ force,
                                                            Partial* part, unsigned* counter, lj_totals* totals,
                                                            unsigned* status) {
    __shared__ int2 s_win[9][BLOCK];
    const int t = blockIdx.x * BLOCK + threadIdx.x;
    const int ncell = g.gx * g.gy * g.gz;
    const bool activeA = t < min(__ldg(npairs_p), nk);
    bool activeB = false;
    int ka = 0;
    float4 pa = make_float4(0.f, 0.f, 0.f, 0.f), pb = pa;
    int ws[9], wl[9];
#pragma unroll
    for (int r = 0; r < 9; ++r) ws[r] = wl[r] = 0;
    if (activeA) {
        ka = min(max(__ldg(&list[t]), 0), n - 1);
        int c = __ldg(&cs[ka]);
        if (c < 0 || c >= ncell) {
            atomicOr(status, kFlagRange);
            c = 0;
        }
        activeB = ka + 1 < ke && __ldg(&cs[ka + 1]) == c;
        pa = __ldg(&p[ka]);
        if (activeB) pb = __ldg(&p[ka + 1]);
        int cx, cy, cz;
        decode_cell(g, c, cx, cy, cz);
        const int xl = max(cx - 1, 0), xh = min(cx + 1, g.gx - 1);
#pragma unroll
        for (int r = 0; r < 9; ++r) {
            const int z = cz + r / 3 - 1, y = cy + r % 3 - 1;
            if (z < 0 || z >= g.gz || y < 0 || y >= g.gy) continue;
            const int rb = (z * g.gy + y) * g.gx;
            const int s = min(max(__ldg(&off[rb + xl]), 0), n);
            const int e = min(max(__ldg(&off[rb + xh + 1]), s), n);
            ws[r] = s;
            wl[r] = e - s;
        }
    }
    Pass2Acc a;
    a.e = a.w = a.fx = a.fy = a.fz = make_float2(0.f, 0.f);
    a.np = 0;
    const int kb2 = ka + 1;
    const float2 nx = make_float2(-pa.x, -pb.x), ny = make_float2(-pa.y, -pb.y), nz = make_float2(-pa.z, -pb.z);
    int nw = 0, L = 0;
#pragma unroll
    for (int r = 0; r < 9; ++r)
        if (wl[r] > 0) {
            s_win[nw++][threadIdx.x] = make_int2(ws[r], ws[r] + wl[r]);
            L += wl[r];
        }
    walk_flat2<BLOCK>(p, ka, kb2, ka, activeA, activeB, nx, ny, nz, s_win, nw, L, pp.rc2, pp.sig2, a);
    const float2 s12 = a.e, ns6 = a.w;
    a.e = __fadd2_rn(s12, ns6);
    a.w = __ffma2_rn(make_float2(2.0f, 2.0f), s12, ns6);
    const float nf = -pp.fscale;
    const int oa = activeA ? out_slot(pp, p, ka, n, status) : -1;
    const int ob = activeB ? out_slot(pp, p, kb2, n, status) : -1;
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

lj_status launch_pair_cellpair(lj_ctx* ctx, const lj_grid* g, const PairParams& pp, int n, const float* xyzi,
                               const int* cs, const int* off, float* energy, float* force, lj_totals* totals,
                               int kb, int ke) {
    const long long nk = ke - kb;
    const int blocks = (int)((nk + kPassThreads - 1) / kPassThreads);
    const size_t need_red = 256 + (size_t)blocks * sizeof(Partial);
    lj_status s;
    if (need_red > ctx->red_bytes) {
        if ((s = grow(&ctx->red, &ctx->red_bytes, need_red)) != LJ_OK) return s;
        if (cudaMemsetAsync(ctx->red, 0, 256, ctx->stream) != cudaSuccess) return LJ_ECUDA;
    }
    // flag[nk] | pos[nk + 1] | list[nk], each array starting on a 16-byte boundary (the scan's vector path)
    const size_t words = ((size_t)nk + 4) & ~(size_t)3;
    if ((s = grow(&ctx->cellpair, &ctx->cellpair_bytes, 3 * words * sizeof(int) + 64)) != LJ_OK) return s;
    int* flag = static_cast<int*>(ctx->cellpair);
    int* pos = flag + words;
    int* list = pos + words;
    cudaStream_t st = ctx->stream;
    const int ncell = g->dim[0] * g->dim[1] * g->dim[2];
    k_cellpair_flags<<<grid_for(ctx, nk, 256), 256, 0, st>>>(cs, off, ncell, kb, ke, flag, ctx->d_status);
    if ((s = last_launch_status()) != LJ_OK) return s;
    if ((s = launch_scan(ctx, flag, nk, pos)) != LJ_OK) return s;
    k_cellpair_list<<<grid_for(ctx, nk, 256), 256, 0, st>>>(flag, pos, (int)nk, kb, list);
    if ((s = last_launch_status()) != LJ_OK) return s;
    unsigned* counter = static_cast<unsigned*>(ctx->red);
    Partial* part = reinterpret_cast<Partial*>(static_cast<char*>(ctx->red) + 256);
    k_pair_cellpair<><<<blocks, kPassThreads, 0, st>>>(to_dev(*g), pp, reinterpret_cast<const float4*>(xyzi), cs, off,
                                                       n, (int)nk, ke, list, pos + nk, energy, force, part, counter,
                                                       totals, ctx->d_status);
    return last_launch_status();
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
