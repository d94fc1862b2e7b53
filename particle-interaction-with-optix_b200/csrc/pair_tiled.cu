// pair_tiled.cu -- the truncated-LJ pair kernel on cell-block tiles staged in
// shared memory by TMA bulk copies.
//
// Tiles.  k_build_tiles cuts every row of cells (fixed y, z) into runs of
// consecutive cells holding about T targets: tile m of a row starts at the
// first cell start at or after particle index row_start + m T.  A tile is
// (targets [k0, k1), first cell, last cell), all in one row.
//
// Staging.  The neighbours of a tile are the 9 rows (y +- 1, z +- 1) over the
// cells [first - 1, last + 1]: 9 contiguous ranges of the cell-ordered float4
// array.  One thread issues one cp.async.bulk per range into shared memory,
// completing on an mbarrier (plain copies, no multicast).  A tile whose
// neighbourhood exceeds the staging capacity reads global memory instead.
//
// Per target (one thread each): rows that cannot hold a partner are skipped
// and the others are cut to the x-window [x - h, x + h] by binary search in
// the staged, x-sorted row (particles binned with LJ_ORDER_X), exactly as in
// pair.cu; the windows are walked as one flat list so a lane stays busy until
// its own list ends.  The CTA is persistent and takes tiles from a counter.
// Replaces ComputeParticleInterationsParPartNoLoop (cudaLJ.cu:299-341) for
// the truncated law; the loads that the reference makes per candidate from
// global memory come from shared memory here.
#include "pair_common.cuh"

namespace ljc {

constexpr int kTileThreads = 256;
constexpr unsigned kMbarSpinLimit = 1u << 20;  // try_wait polls: about a second at most

extern __shared__ float4 s_stage[];

// ---------------------------------------------------------------- PTX helpers (mbarrier + bulk copy)
__device__ __forceinline__ unsigned smem_addr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait for the barrier phase; false if the limit ran out.
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long* bar, unsigned parity) {
    for (unsigned i = 0; i < kMbarSpinLimit; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Global -> shared bulk copy (16-byte aligned addresses, size a multiple of 16).
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

// ---------------------------------------------------------------- tiles
// last c in [0, m] with o[c] <= v  (o non-decreasing, o[0] <= v)
__device__ __forceinline__ int last_le(const int* __restrict__ o, int m, int v) {
    int lo = 0, hi = m;  // invariant: o[lo] <= v
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(&o[mid]) <= v)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}
// first c in [0, m] with o[c] >= v, or m + 1 if none
__device__ __forceinline__ int first_ge(const int* __restrict__ o, int m, int v) {
    int lo = 0, hi = m + 1;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (__ldg(&o[mid]) < v)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

// One warp per row of cells.  The row's offsets o[0..gx] (o[gx] = row end)
// list the starts of its non-empty cells (an empty cell repeats the next start).
__global__ void __launch_bounds__(256) k_build_tiles(GridDev g, const int* __restrict__ off, int T,
                                                     int4* __restrict__ tiles, int cap, unsigned* ntiles,
                                                     unsigned* status) {
    const int lane = threadIdx.x & 31;
    const long long gwarp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    const long long nrows = (long long)g.gy * g.gz;
    for (long long r = gwarp; r < nrows; r += nwarps) {
        const int* o = off + r * g.gx;
        const int rs = __ldg(&o[0]), re = __ldg(&o[g.gx]);
        const int cnt = re - rs;
        if (cnt <= 0) continue;
        const int nt = (cnt + T - 1) / T;
        for (int m = lane; m < nt; m += 32) {
            const int ia = first_ge(o, g.gx, rs + m * T);
            const int k0 = ia <= g.gx ? __ldg(&o[ia]) : re;
            int k1 = re;
            if (m + 1 < nt) {
                const int ib = first_ge(o, g.gx, rs + (m + 1) * T);
                k1 = ib <= g.gx ? __ldg(&o[ib]) : re;
            }
            if (k0 >= k1) continue;  // a large cell absorbed this slice
            const int ca = last_le(o, g.gx, k0);
            const int cb = last_le(o, g.gx, k1 - 1);
            const unsigned slot = atomicAdd(ntiles, 1u);
            if ((int)slot < cap)
                tiles[slot] = make_int4(k0, k1, (int)(r * g.gx + ca), (int)(r * g.gx + cb));
            else
                atomicOr(status, kFlagRange);
        }
    }
}

// ---------------------------------------------------------------- per-target work
struct TileRows {
    int beg[9];  // row start in the index space of the source (shared or global)
    int len[9];
    int gbeg[9];  // row start in the global index space
};

struct Acc {
    float e, fx, fy, fz, w;
    unsigned np;
};

__device__ __forceinline__ void pair_body(const float4& pi, const float4& q, float rc2, float sig2, Acc& a) {
    const float dx = q.x - pi.x, dy = q.y - pi.y, dz = q.z - pi.z;
    const float r2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
    if (r2 < rc2) {
        const float ir2 = rcp_approx(r2);
        const float s2 = sig2 * ir2;
        const float s6 = s2 * s2 * s2;
        const float s12 = s6 * s6;
        a.e += s12 - s6;
        const float t = fmaf(2.0f, s12, -s6);
        a.w += t;
        const float fs = t * s2;
        a.fx = fmaf(fs, dx, a.fx);
        a.fy = fmaf(fs, dy, a.fy);
        a.fz = fmaf(fs, dz, a.fz);
        ++a.np;
    }
}

template <bool STAGED>
__device__ __forceinline__ float4 ld4(const float4* __restrict__ p, int i) {
    if constexpr (STAGED)
        return s_stage[i];
    else
        return __ldg(&p[i]);
}
template <bool STAGED>
__device__ __forceinline__ float ldx(const float4* __restrict__ p, int i) {
    if constexpr (STAGED)
        return s_stage[i].x;
    else
        return __ldg(&p[i].x);
}
template <bool STAGED>
__device__ __forceinline__ int lower_bound_x(const float4* __restrict__ p, int lo, int hi, float v) {
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (ldx<STAGED>(p, mid) < v)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}
template <bool STAGED>
__device__ __forceinline__ int upper_bound_x(const float4* __restrict__ p, int lo, int hi, float v) {
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (ldx<STAGED>(p, mid) <= v)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

// Windows of target `ks` (source index) in the 9 rows.  Calls f(lo, hi) per window.
template <bool STAGED, class F>
__device__ __forceinline__ void for_windows(const GridDev& g, const PairParams& pp, const float4* __restrict__ p,
                                            const TileRows& rows, int cy, int cz, const float4& pi, int ks,
                                            float slack, F&& f) {
#pragma unroll
    for (int r = 0; r < 9; ++r) {
        const int len = rows.len[r];
        if (len == 0) continue;
        const int dz = r / 3 - 1, dy = r % 3 - 1;
        float dzm = 0.f, dym = 0.f;
        if (dz < 0) dzm = pi.z - fmaf((float)cz, g.w, g.oz);
        if (dz > 0) dzm = fmaf((float)(cz + 1), g.w, g.oz) - pi.z;
        if (dy < 0) dym = pi.y - fmaf((float)cy, g.w, g.oy);
        if (dy > 0) dym = fmaf((float)(cy + 1), g.w, g.oy) - pi.y;
        dzm = fmaxf(dzm - slack, 0.f);
        dym = fmaxf(dym - slack, 0.f);
        const float d2 = fmaf(dym, dym, dzm * dzm);
        if (d2 >= pp.rc2w) continue;
        const float h = sqrtf(pp.rc2w - d2) + slack;
        const int b = rows.beg[r];
        const int lo = lower_bound_x<STAGED>(p, b, b + len, pi.x - h);
        const int hi = upper_bound_x<STAGED>(p, lo, b + len, pi.x + h);
        if (r == 4) {
            f(lo, ks);
            f(ks + 1, hi);
        } else {
            f(lo, hi);
        }
    }
}

// Staged path: windows packed as lo | hi << 16 in shared memory, walked flat.
__device__ __forceinline__ void target_staged(const GridDev& g, const PairParams& pp, const TileRows& rows, int cy,
                                              int cz, int ks, unsigned (*s_win)[kTileThreads], Acc& a) {
    const int tid = threadIdx.x;
    const float4 pi = s_stage[ks];
    const float slack = pp.slack + 8.0f * FLT_EPSILON * fmaxf(fabsf(pi.x), fmaxf(fabsf(pi.y), fabsf(pi.z)));
    int nw = 0;
    for_windows<true>(g, pp, nullptr, rows, cy, cz, pi, ks, slack, [&](int lo, int hi) {
        if (lo < hi) s_win[nw++][tid] = (unsigned)lo | ((unsigned)hi << 16);
    });
    if (nw == 0) return;
    const float rc2 = pp.rc2, sig2 = pp.sig2;
    int w = 0;
    unsigned wv = s_win[0][tid];
    int j = (int)(wv & 0xffffu), je = (int)(wv >> 16);
    while (true) {
        if (j >= je) {
            if (++w >= nw) break;
            wv = s_win[w][tid];
            j = (int)(wv & 0xffffu);
            je = (int)(wv >> 16);
        }
        pair_body(pi, s_stage[j], rc2, sig2, a);
        ++j;
    }
}

// Global path (a tile whose neighbourhood does not fit the stage): row by row.
__device__ __forceinline__ void target_global(const GridDev& g, const PairParams& pp, const float4* __restrict__ p,
                                              const TileRows& rows, int cy, int cz, int k, Acc& a) {
    const float4 pi = __ldg(&p[k]);
    const float slack = pp.slack + 8.0f * FLT_EPSILON * fmaxf(fabsf(pi.x), fmaxf(fabsf(pi.y), fabsf(pi.z)));
    const float rc2 = pp.rc2, sig2 = pp.sig2;
    for_windows<false>(g, pp, p, rows, cy, cz, pi, k, slack, [&](int lo, int hi) {
        for (int j = lo; j < hi; ++j) pair_body(pi, __ldg(&p[j]), rc2, sig2, a);
    });
}

__global__ void __launch_bounds__(kTileThreads) k_pair_tiled(GridDev g, PairParams pp, const float4* __restrict__ p,
                                                             const int* __restrict__ off, int n,
                                                             const int4* __restrict__ tiles,
                                                             const unsigned* __restrict__ ntiles_p, int tile_cap,
                                                             unsigned* tile_counter, int stage_cap,
                                                             float* __restrict__ energy, float* __restrict__ force,
                                                             Partial* part, unsigned* counter, lj_totals* totals,
                                                             unsigned* status) {
    __shared__ unsigned s_win[kMaxWin][kTileThreads];
    __shared__ __align__(8) unsigned long long s_bar;
    __shared__ TileRows s_rows;
    __shared__ int4 s_desc;
    __shared__ int s_tile, s_staged, s_fail;
    const int tid = threadIdx.x;
    if (tid == 0) {
        mbar_init(&s_bar, 1);
        s_fail = 0;
    }
    __syncthreads();
    unsigned phase = 0;
    const int ntiles = min((int)*ntiles_p, tile_cap);
    double te = 0.0, tw = 0.0;
    unsigned long long tnp = 0;
    const int gxy = g.gx * g.gy;
    while (true) {
        if (tid == 0) s_tile = (int)atomicAdd(tile_counter, 1u);
        __syncthreads();
        const int t = s_tile;
        if (t >= ntiles || s_fail) break;
        if (tid < 9) {
            const int4 d = tiles[t];
            const int cz = d.z / gxy, cy = (d.z - cz * gxy) / g.gx;
            const int xa = d.z - cz * gxy - cy * g.gx, xb = d.w - cz * gxy - cy * g.gx;
            const int z = cz + tid / 3 - 1, y = cy + tid % 3 - 1;
            int gb = 0, gl = 0;
            if (z >= 0 && z < g.gz && y >= 0 && y < g.gy) {
                const int rb = (z * g.gy + y) * g.gx;
                gb = min(max(__ldg(&off[rb + max(xa - 1, 0)]), 0), n);
                const int ge = min(max(__ldg(&off[rb + min(xb + 1, g.gx - 1) + 1]), gb), n);
                gl = ge - gb;
            }
            s_rows.gbeg[tid] = gb;
            s_rows.len[tid] = gl;
            if (tid == 0) s_desc = d;
        }
        __syncthreads();
        if (tid == 0) {
            int tot = 0;
            for (int r = 0; r < 9; ++r) {
                s_rows.beg[r] = tot;
                tot += s_rows.len[r];
            }
            const bool st = tot > 0 && tot <= stage_cap;
            s_staged = st;
            if (st) {
                fence_proxy_async_smem();
                mbar_arrive_expect_tx(&s_bar, (unsigned)tot * 16u);
                for (int r = 0; r < 9; ++r)
                    if (s_rows.len[r] > 0)
                        bulk_g2s(&s_stage[s_rows.beg[r]], p + s_rows.gbeg[r], (unsigned)s_rows.len[r] * 16u, &s_bar);
            } else {
                for (int r = 0; r < 9; ++r) s_rows.beg[r] = s_rows.gbeg[r];
            }
        }
        __syncthreads();
        const bool staged = s_staged;
        if (staged) {
            if (!mbar_wait_bounded(&s_bar, phase)) atomicExch(&s_fail, 1);
            phase ^= 1u;
        }
        __syncthreads();
        if (s_fail) {
            // the copies did not complete in time: record it, wait (bounded) for them, stop taking tiles
            if (tid == 0) atomicOr(status, kFlagTimeout);
            mbar_wait_bounded(&s_bar, phase ^ 1u);
            break;
        }
        const int4 d = s_desc;
        const int cz = d.z / gxy, cy = (d.z - cz * gxy) / g.gx;
        const TileRows& rows = s_rows;
        for (int k = d.x + tid; k < d.y; k += kTileThreads) {
            Acc a{0.f, 0.f, 0.f, 0.f, 0.f, 0u};
            if (staged)
                target_staged(g, pp, rows, cy, cz, rows.beg[4] + (k - rows.gbeg[4]), s_win, a);
            else
                target_global(g, pp, p, rows, cy, cz, k, a);
            if (energy) energy[k] = pp.e4 * a.e;
            if (force) {
                force[3 * (size_t)k + 0] = pp.fscale * a.fx;
                force[3 * (size_t)k + 1] = pp.fscale * a.fy;
                force[3 * (size_t)k + 2] = pp.fscale * a.fz;
            }
            te += 0.5 * (double)pp.e4 * (double)a.e;
            tw += 0.5 * (double)pp.e24 * (double)a.w;
            tnp += a.np;
        }
        __syncthreads();
    }
    reduce_totals<kTileThreads>(te, tw, tnp, part, counter, totals);
}

// ---------------------------------------------------------------- host side
lj_status launch_pair_tiled(lj_ctx* ctx, const lj_grid* g, const PairParams& pp, int n, const float* xyzi,
                            const int* off, float* energy, float* force, lj_totals* totals) {
    const GridDev gd = to_dev(*g);
    const long long nrows = (long long)g->dim[1] * g->dim[2];
    const double rho = (double)n / ((double)g->dim[0] * g->dim[1] * g->dim[2]);  // particles per cell
    const int T = kTileThreads;
    const long long tile_cap = (long long)n / T + nrows + 1;
    // scratch: [0] tile counter, [1] ntiles, then the tiles
    const size_t need = 256 + (size_t)tile_cap * sizeof(int4);
    lj_status s = grow(&ctx->tiles, &ctx->tiles_bytes, need);
    if (s != LJ_OK) return s;
    unsigned* hdr = static_cast<unsigned*>(ctx->tiles);
    int4* tiles = reinterpret_cast<int4*>(static_cast<char*>(ctx->tiles) + 256);
    if (cudaMemsetAsync(hdr, 0, 256, ctx->stream) != cudaSuccess) return LJ_ECUDA;
    long long bwarps = (nrows + 7) / 8;
    int bblocks = (int)(bwarps < (long long)ctx->sm_count * 16 ? (bwarps > 0 ? bwarps : 1) : ctx->sm_count * 16);
    k_build_tiles<<<bblocks, 256, 0, ctx->stream>>>(gd, off, T, tiles, (int)tile_cap, hdr + 1, ctx->d_status);
    if ((s = last_launch_status()) != LJ_OK) return s;
    // stage capacity: the expected neighbourhood of a T-target tile with margin, 2048..6144 particles
    int cap = (int)(9.0 * ((double)T / (rho > 1e-9 ? rho : 1e-9) + 2.5) * rho * 1.4);
    cap = cap < 2048 ? 2048 : (cap > 6144 ? 6144 : cap);
    cap = (cap + 255) & ~255;
    const size_t dyn = (size_t)cap * sizeof(float4);
    static size_t attr_set = 0;
    if (dyn > attr_set) {
        if (cudaFuncSetAttribute(k_pair_tiled, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn) !=
            cudaSuccess)
            return LJ_ECUDA;
        attr_set = dyn;
    }
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pair_tiled, kTileThreads, dyn) != cudaSuccess ||
        per_sm < 1)
        per_sm = 1;
    const int blocks = ctx->sm_count * per_sm;
    const size_t rneed = 256 + (size_t)blocks * sizeof(Partial);
    if (rneed > ctx->red_bytes) {
        if ((s = grow(&ctx->red, &ctx->red_bytes, rneed)) != LJ_OK) return s;
        if (cudaMemsetAsync(ctx->red, 0, 256, ctx->stream) != cudaSuccess) return LJ_ECUDA;
    }
    unsigned* counter = static_cast<unsigned*>(ctx->red);
    Partial* part = reinterpret_cast<Partial*>(static_cast<char*>(ctx->red) + 256);
    k_pair_tiled<<<blocks, kTileThreads, dyn, ctx->stream>>>(gd, pp, reinterpret_cast<const float4*>(xyzi), off, n,
                                                             tiles, hdr + 1, (int)tile_cap, hdr, cap, energy, force,
                                                             part, counter, totals, ctx->d_status);
    return last_launch_status();
}

}  // namespace ljc
