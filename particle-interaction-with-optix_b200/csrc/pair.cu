// pair.cu -- the interaction stage on the device.
//
// k_pair_compat replaces ComputeParticleInterationsParPartNoLoop
// (cudaLJ.cu:299-341) with the reference's law and stencil: every particle of
// the clamped 27-cell block except itself, r = sqrt(d.d + 1e-5),
// 4 eps ((1/r)^12 - (1/r)^6) with eps = sigma = 1, no cutoff; 1/r from the
// approximate reciprocal square root, within the reference's own tolerance
// (see the kernel).  Two targets per lane, the 27 cells read as 9 rows of 3
// consecutive cells (contiguous in cell order) in lockstep passes, one float4
// load per candidate shared by both targets.
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
#include <climits>

#include "pair_common.cuh"

namespace ljc {

constexpr double kPairCell = 2.0;    // particles per cell from which the default takes two targets per lane

// Default pair kernel for LJ_ORDER_X (measured on B200): the packed row passes with two targets per
// lane (kernel 10) from 2 particles per cell up (10M at 10 per cell: 2.33 ms against 2.88 ms for one
// target per lane; 80 per cell: 11.4 ms against 12.6 ms for the SoA walk); below, the targets paired
// inside their cell over whole rows (kernel 12: a 4M sphere shell on 64M cells 0.517 ms against 0.597
// for kernel 11 and 0.75 for kernel 6; 0.5M uniform on 100^3 cells 0.055 ms against 0.060 for
// kernel 6), where windows merged across cells add more candidates than the shared loads save.
int default_pair_kernel(int n, const lj_grid& g) {
    return (double)n / ((double)g.dim[0] * g.dim[1] * g.dim[2]) >= kPairCell ? 10 : 12;
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
        const int o = out_slot(pp, p, k, n, status);
        if (o >= 0 && energy) energy[o] = pp.e4 * ea;
        if (o >= 0 && force) {
            force[3 * (size_t)o + 0] = pp.fscale * fx;
            force[3 * (size_t)o + 1] = pp.fscale * fy;
            force[3 * (size_t)o + 2] = pp.fscale * fz;
        }
    }
    reduce_totals<kPairThreads>(0.5 * (double)pp.e4 * (double)ea, 0.5 * (double)pp.e24 * (double)wa,
                                (unsigned long long)np, part, counter, totals);
}

// ---------------------------------------------------------------- reference law (compat)
// Lane m of a warp takes the consecutive sorted targets a = 2m and b = 2m + 1.  Every particle of a
// target's clamped 27-cell stencil except itself is a partner (no cutoff), so its 9 rows of 3 cells
// are walked whole.  When a and b sit in the same (y, z) row of cells (cxb >= cxa) their rows are the
// same rows of cells shifted by cxb - cxa: each row is walked once over the union of the two ranges
// and each candidate loaded once is evaluated for both targets in paired FP32, each target masked to
// its own 3 cells and to j != itself.  The rows are taken in 5 passes, all lanes of a warp in
// lockstep (the own row, then opposite rows paired), so the warp's loads fall on a few neighbouring
// lines.  A lane whose targets lie in different rows walks a's rows, then, in a second sweep that only
// warps holding such a lane take, b's.
//
// The law is the reference's, 4 eps ((s/r)^12 - (s/r)^6) with eps = s = 1 and
// r = sqrt(d.d + 1e-5), with s/r taken from the approximate reciprocal square root (rsqrt.approx.ftz,
// at most 2 ulp) where the reference divides 1 by an IEEE square root: (s/r)^12 then carries at most
// about 12 * 2^-22 relative error, and every term is positive whenever r < 1 (always within a stencil
// of cells narrower than 1/sqrt(3)), so a particle's energy stays within about 3e-6 of the
// reference's law (the reference's own check allows 1e-5, cudaLJ.cu:246-250).  A masked candidate
// gets r^2 = +inf, whose reciprocal square root is an exact 0: no branch.
__device__ __forceinline__ float rsqrt_approx(float x) {
    float r;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// Candidate q against targets (a, b) (minus their coordinates in nx, ny, nz); masks ma, mb.
__device__ __forceinline__ void compat2(const float4& q, bool ma, bool mb, float2 nx, float2 ny, float2 nz,
                                        float2& pot) {
    const float inf = __int_as_float(0x7f800000);
    const float2 dx = __fadd2_rn(make_float2(q.x, q.x), nx);
    const float2 dy = __fadd2_rn(make_float2(q.y, q.y), ny);
    const float2 dz = __fadd2_rn(make_float2(q.z, q.z), nz);
    const float2 d2 = __ffma2_rn(dz, dz, __ffma2_rn(dy, dy, __fmul2_rn(dx, dx)));
    const float2 r2 = __fadd2_rn(d2, make_float2(1e-5f, 1e-5f));
    const float2 sdr = make_float2(rsqrt_approx(ma ? r2.x : inf), rsqrt_approx(mb ? r2.y : inf));
    const float2 s2 = __fmul2_rn(sdr, sdr);
    const float2 s4 = __fmul2_rn(s2, s2);
    const float2 r6 = __fmul2_rn(s4, s2);
    const float2 r12 = __fmul2_rn(r6, r6);
    pot = __fadd2_rn(pot, __ffma2_rn(r6, make_float2(-1.0f, -1.0f), r12));  // r12 - r6, one rounding
}

// One window of a row for both targets: candidates [s, e); target a takes those below ea, target b
// those from sb on (a's 3 cells start the union, b's end it).
struct CompatRow {
    int s, e, ea, sb;
};

// Row (dy, dz) of cell (cx, cy, cz) clamped to the grid: [s, e), the particles of cells cx-1..cx+1;
// (0, 0) off the grid.
__device__ __forceinline__ int2 compat_range(const GridDev& g, const int* __restrict__ off, int n, int cx, int cy,
                                             int cz, int dy, int dz) {
    const int z = cz + dz, y = cy + dy;
    if (z < 0 || z >= g.gz || y < 0 || y >= g.gy) return make_int2(0, 0);
    const int rb = (z * g.gy + y) * g.gx;
    const int s = min(max(__ldg(&off[rb + max(cx - 1, 0)]), 0), n);
    const int e = min(max(__ldg(&off[rb + min(cx + 1, g.gx - 1) + 1]), s), n);
    return make_int2(s, e);
}

// Row (dy, dz) for this round: useA / useB select the targets, same: b shares a's rows.
__device__ __forceinline__ CompatRow compat_row(const GridDev& g, const int* __restrict__ off, int n, bool useA,
                                                bool useB, bool same, int cxa, int cya, int cza, int cxb, int cyb,
                                                int czb, int dy, int dz) {
    CompatRow r{0, 0, 0, INT_MAX};
    if (useA) {
        const int2 a = compat_range(g, off, n, cxa, cya, cza, dy, dz);
        r.s = a.x;
        r.e = a.y;
        r.ea = a.y;
        if (same) {
            const int2 b = compat_range(g, off, n, cxb, cyb, czb, dy, dz);
            r.e = max(a.y, b.y);
            r.sb = b.x;
        }
    } else if (useB) {
        const int2 b = compat_range(g, off, n, cxb, cyb, czb, dy, dz);
        r.s = b.x;
        r.e = b.y;
        r.ea = INT_MIN;
        r.sb = b.x;
    }
    return r;
}

// One window, all lanes of the warp in lockstep, two candidates per step.
__device__ __forceinline__ void compat_walk(const float4* __restrict__ p, int kl, const CompatRow& R, float2 nx,
                                            float2 ny, float2 nz, float2& pot) {
    const int L = R.e - R.s;
    const int maxL = (int)__reduce_max_sync(0xffffffffu, (unsigned)L);
    for (int v = 0; v < maxL; v += 2) {
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            const int w = v + u;
            const bool ok = w < L;
            const int j = R.s + w;
            const float4 q = __ldg(&p[ok ? j : kl]);
            compat2(q, ok && j < R.ea, ok && j >= R.sb, nx, ny, nz, pot);
        }
    }
}

// The 9 rows of this round: the own row in two windows around the targets ([s, lo_self) and
// [hi_self, e)), then opposite rows (-y, +y), (-z, +z), (-y-z, +y+z), (+y-z, -y+z).
__device__ __forceinline__ void compat_rows(const GridDev& g, const float4* __restrict__ p,
                                            const int* __restrict__ off, int n, int kl, int lo_self, int hi_self,
                                            bool useA, bool useB, bool same, int cxa, int cya, int cza, int cxb,
                                            int cyb, int czb, float2 nx, float2 ny, float2 nz, float2& pot) {
    {
        const CompatRow own = compat_row(g, off, n, useA, useB, same, cxa, cya, cza, cxb, cyb, czb, 0, 0);
        CompatRow lo = own, hi = own;
        lo.e = max(min(own.e, lo_self), own.s);
        hi.s = min(max(own.s, hi_self), own.e);
        compat_walk(p, kl, lo, nx, ny, nz, pot);
        compat_walk(p, kl, hi, nx, ny, nz, pot);
    }
#pragma unroll 1
    for (int q = 0; q < 8; ++q) {
        // (-y, +y), (-z, +z), (-y-z, +y+z), (+y-z, -y+z): each row followed by its opposite
        const int h = q >> 1, sg = (q & 1) ? -1 : 1;
        const int dy = sg * (h == 0 ? -1 : (h == 1 ? 0 : (h == 2 ? -1 : 1)));
        const int dz = sg * (h == 0 ? 0 : -1);
        compat_walk(p, kl, compat_row(g, off, n, useA, useB, same, cxa, cya, cza, cxb, cyb, czb, dy, dz), nx, ny, nz,
                    pot);
    }
}

__global__ void __launch_bounds__(kPairThreads) k_pair_compat(GridDev g, const float4* __restrict__ p,
                                                              const int* __restrict__ cs,
                                                              const int* __restrict__ off, int n,
                                                              float* __restrict__ v, unsigned* status) {
    const int ka = 2 * (blockIdx.x * kPairThreads + (int)threadIdx.x), kb = ka + 1;
    const bool activeA = ka < n, activeB = kb < n;
    const int ncell = g.gx * g.gy * g.gz;
    const float far = 1e30f;  // a parked target: every squared distance overflows to +inf
    float4 pa = make_float4(far, far, far, 0.f), pb = pa;
    int cxa = 0, cya = 0, cza = 0, cxb = 0, cyb = 0, czb = 0;
    if (activeA) {
        int c = __ldg(&cs[ka]);
        if (c < 0 || c >= ncell) {
            atomicOr(status, kFlagRange);
            c = 0;
        }
        decode_cell(g, c, cxa, cya, cza);
        pa = __ldg(&p[ka]);
    }
    if (activeB) {
        int c = __ldg(&cs[kb]);
        if (c < 0 || c >= ncell) {
            atomicOr(status, kFlagRange);
            c = 0;
        }
        decode_cell(g, c, cxb, cyb, czb);
        pb = __ldg(&p[kb]);
    }
    const bool same = activeA && activeB && cya == cyb && cza == czb && cxb >= cxa;
    const bool apart = activeB && !same;
    const int kl = min(ka, n - 1);
    const float2 nx = make_float2(-pa.x, -pb.x), ny = make_float2(-pa.y, -pb.y), nz = make_float2(-pa.z, -pb.z);
    float2 pot = make_float2(0.f, 0.f);
    // first sweep: a, and b when it shares a's rows (the own row walked around both)
    compat_rows(g, p, off, n, kl, ka, same ? kb + 1 : ka + 1, activeA, false, same, cxa, cya, cza, cxb, cyb, czb, nx,
                ny, nz, pot);
    // second sweep: b alone, only in warps holding a lane whose targets lie in different rows
    if (__any_sync(0xffffffffu, apart))
        compat_rows(g, p, off, n, kl, kb, kb + 1, false, apart, false, cxa, cya, cza, cxb, cyb, czb, nx, ny, nz, pot);
    if (same) {  // the pair (a, b), left out of the own row: each counts when in the other's 3 cells
        const bool ba = cxb <= cxa + 1;  // symmetric: cxb >= cxa in one row
        const float4 qb = pb;
        const float4 qa = pa;
        float2 t = make_float2(0.f, 0.f);
        // a's partner b in half x (the y half masked), then b's partner a in half y
        compat2(qb, ba, false, nx, ny, nz, t);
        compat2(qa, false, ba, nx, ny, nz, t);
        pot = __fadd2_rn(pot, t);
    }
    if (activeA) v[ka] = 4.0f * pot.x;
    if (activeB) v[kb] = 4.0f * pot.y;
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
                             lj_totals* totals, int kb, int ke, bool by_index) {
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
    pp.by_index = by_index ? 1 : 0;
    if (order == LJ_ORDER_X) {
        int kernel = ctx->tuning.pair_kernel;
        if (kernel == 0) kernel = default_pair_kernel(n, *g);
        switch (kernel) {
            // retired variants run the surviving kernel of their family: 2, 3, 4 -> 1; 5, 7 -> 6; 8, 9 -> 10
            case 5:
            case 6:
            case 7: return launch_pair_pass(ctx, g, pp, n, xyzi, cs, off, false, energy, force, totals, kb, ke);
            case 8:
            case 9:
            case 10: return launch_pair_pass(ctx, g, pp, n, xyzi, cs, off, true, energy, force, totals, kb, ke);
            case 12: return launch_pair_cellpair(ctx, g, pp, n, xyzi, cs, off, energy, force, totals, kb, ke);
            default: break;  // 1 (and 2, 3, 4): windows in shared memory; 11: whole rows (below)
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
    // kernel 11 walks the 9 rows whole, without the culling and x-window searches: on sparse grids
    // (few particles per row) the searches cost more than the candidates they remove
    const bool xwin = order == LJ_ORDER_X && ctx->tuning.pair_kernel != 11;
    if (xwin)
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
    const NvtxRange nvtx_range("lj_compute_compat");
    if (!ctx || !g || n < 0 || (n > 0 && (!sorted_xyzi || !sorted_cell || !offsets || !v))) return LJ_EINVAL;
    if (!(g->width > 0.0f) || g->dim[0] < 1 || g->dim[1] < 1 || g->dim[2] < 1) return LJ_EINVAL;
    if (reinterpret_cast<uintptr_t>(sorted_xyzi) & 15) return LJ_EINVAL;
    if (n == 0) return LJ_OK;
    k_pair_compat<<<(n + 2 * kPairThreads - 1) / (2 * kPairThreads), kPairThreads, 0, ctx->stream>>>(
        to_dev(*g), reinterpret_cast<const float4*>(sorted_xyzi), sorted_cell, offsets, n, v, ctx->d_status);
    return last_launch_status();
}

extern "C" lj_status lj_compute(lj_ctx* ctx, const lj_grid* g, const lj_params* p, int n, const float* sorted_xyzi,
                                const int* sorted_cell, const int* offsets, lj_order order, float* energy,
                                float* force, lj_totals* totals) {
    const NvtxRange nvtx_range("lj_compute");
    if (!ctx || !g || !p || n < 0) return LJ_EINVAL;
    if (n > 0 && (!sorted_xyzi || !sorted_cell || !offsets)) return LJ_EINVAL;
    if (!(g->width > 0.0f) || g->dim[0] < 1 || g->dim[1] < 1 || g->dim[2] < 1) return LJ_EINVAL;
    if (!(p->cutoff > 0.0f) || !(p->cutoff <= g->width) || !(p->sigma > 0.0f)) return LJ_EINVAL;
    if (order != LJ_ORDER_INDEX && order != LJ_ORDER_X) return LJ_EINVAL;
    if (reinterpret_cast<uintptr_t>(sorted_xyzi) & 15) return LJ_EINVAL;
    return launch_pair_config(ctx, g, p, n, sorted_xyzi, sorted_cell, offsets, order, energy, force, totals, 0, n);
}

extern "C" lj_status lj_compute_range(lj_ctx* ctx, const lj_grid* g, const lj_params* p, int n,
                                      const float* sorted_xyzi, const int* sorted_cell, const int* offsets,
                                      lj_order order, int kb, int ke, float* energy, float* force,
                                      lj_totals* totals) {
    const NvtxRange nvtx_range("lj_compute_range");
    if (!ctx || !g || !p || n < 0 || kb < 0 || kb > ke || ke > n) return LJ_EINVAL;
    if (n > 0 && (!sorted_xyzi || !sorted_cell || !offsets)) return LJ_EINVAL;
    if (!(g->width > 0.0f) || g->dim[0] < 1 || g->dim[1] < 1 || g->dim[2] < 1) return LJ_EINVAL;
    if (!(p->cutoff > 0.0f) || !(p->cutoff <= g->width) || !(p->sigma > 0.0f)) return LJ_EINVAL;
    if (order != LJ_ORDER_INDEX && order != LJ_ORDER_X) return LJ_EINVAL;
    if (reinterpret_cast<uintptr_t>(sorted_xyzi) & 15) return LJ_EINVAL;
    return launch_pair_config(ctx, g, p, n, sorted_xyzi, sorted_cell, offsets, order, energy, force, totals, kb, ke);
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
    static const int kCandidates[] = {1, 6, 10, 11, 12};
    for (int ki = 0; ki < 5 && st == LJ_OK; ++ki) {
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
