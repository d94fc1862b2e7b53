// pair_pass.cuh -- warp-synchronous row passes for the truncated-LJ pair stage
// (per-target routine shared by k_pair_pass in pair_pass.cu and the batched
// kernel in batch.cu).
//
// Same windows, float test and law as k_pair_config (pair.cu); what changes is
// the order in which a warp walks them.  The 9 stencil rows are taken in 5
// passes, each pass walked by the whole warp in lockstep for as many steps as
// its longest lane needs:
//
//     pass 0: own row (dy, dz) = (0, 0)
//     pass 1: (-1, 0) then (+1, 0)      pass 2: (0, -1) then (0, +1)
//     pass 3: (-1, -1) then (+1, +1)    pass 4: (+1, -1) then (-1, +1)
//
// Rows on opposite sides of the target are paired because their window
// lengths are anti-correlated (a target close to one face has a long window on
// that side and a short or empty one on the other), so a lane's pass length
// varies little across the warp.  The 32 targets of a warp are consecutive in
// the sorted order (a few neighbouring cells of one row) and their windows in
// a row start at nearby indices, so at each step the warp's loads fall on a
// handful of cache lines instead of one line per lane, and no lane ever
// branches away from the others: the loop bound is the warp's maximum.
//
// PACKED: two candidates per step evaluated with the sm_100 paired FP32
// instructions (__fadd2_rn / __fmul2_rn / __ffma2_rn), each lane of the pair
// rounding exactly as the scalar operation.  The distance test is therefore
// bit-identical to the scalar kernels (pair counts equal); per-target sums are
// kept as two partial sums (even and odd steps) added at the end.
#pragma once

#include <cfloat>

#include "pair_common.cuh"

namespace ljc {

struct PassAcc {
    float2 e, w, fx, fy, fz;  // partial sums (two for the packed form; .y unused in the scalar one)
    unsigned np;
};

// Non-blocking hint that brings the 128-byte line holding *ptr into L1 (no register is written, so the
// warp does not wait for it).
__device__ __forceinline__ void prefetch_l1(const void* ptr) {
    asm volatile("prefetch.global.L1 [%0];" ::"l"(ptr));
}

// Hints for the first lines of window [s, s + L) of float4 records (8 records per line).
__device__ __forceinline__ void prefetch_window(const float4* __restrict__ p, int s, int L) {
    if (L > 0) prefetch_l1(p + s);
    if (L > 8) prefetch_l1(p + s + 8);
    if (L > 16) prefetch_l1(p + s + 16);
}

// One pass: window A = [sA, sA + LA), then window B = [offB + LA, offB + L).  OWN: skip j == k.
// CLAMP: a lane past the end of its windows loads its own record (index k) instead of skipping the
// load, so no default value has to be kept in registers; the masks discard it either way.
template <bool PACKED, bool OWN, bool CLAMP = false>
__device__ __forceinline__ void walk_pass(const float4* __restrict__ p, int k, const float4& pi, int sA, int LA,
                                          int offB, int L, float rc2, float sig2, PassAcc& a) {
    const int maxL = (int)__reduce_max_sync(0xffffffffu, (unsigned)L);
    if (PACKED) {
        const float2 npx = make_float2(-pi.x, -pi.x), npy = make_float2(-pi.y, -pi.y),
                     npz = make_float2(-pi.z, -pi.z);
        const float2 nsig2 = make_float2(-sig2, -sig2), two = make_float2(2.0f, 2.0f);
        for (int v = 0; v < maxL; v += 2) {
            const int v1 = v + 1;
            const bool ok0 = v < L, ok1 = v1 < L;
            const int j0 = v + (v < LA ? sA : offB);
            const int j1 = v1 + (v1 < LA ? sA : offB);
            float4 q0, q1;
            if (CLAMP) {
                q0 = __ldg(&p[ok0 ? j0 : k]);
                q1 = __ldg(&p[ok1 ? j1 : k]);
            } else {
                q0 = pi;
                q1 = pi;
                if (ok0) q0 = __ldg(&p[j0]);
                if (ok1) q1 = __ldg(&p[j1]);
            }
            bool m0 = ok0, m1 = ok1;
            if (OWN) {
                m0 = m0 && j0 != k;
                m1 = m1 && j1 != k;
            }
            const float2 dx = __fadd2_rn(make_float2(q0.x, q1.x), npx);
            const float2 dy = __fadd2_rn(make_float2(q0.y, q1.y), npy);
            const float2 dz = __fadd2_rn(make_float2(q0.z, q1.z), npz);
            const float2 r2 = __ffma2_rn(dz, dz, __ffma2_rn(dy, dy, __fmul2_rn(dx, dx)));
            const bool in0 = m0 && r2.x < rc2, in1 = m1 && r2.y < rc2;
            const float2 ir2 = make_float2(in0 ? rcp_approx(r2.x) : 0.f, in1 ? rcp_approx(r2.y) : 0.f);
            const float2 s2n = __fmul2_rn(nsig2, ir2);  // -s2
            const float2 s4 = __fmul2_rn(s2n, s2n);     // s2 * s2
            const float2 ns6 = __fmul2_rn(s4, s2n);     // -s6
            const float2 s12 = __fmul2_rn(ns6, ns6);    // s6 * s6
            a.e = __fadd2_rn(a.e, __fadd2_rn(s12, ns6));
            const float2 t = __ffma2_rn(two, s12, ns6);  // 2 s12 - s6
            a.w = __fadd2_rn(a.w, t);
            const float2 fsn = __fmul2_rn(t, s2n);  // -(t s2): the sums below hold minus the force sums
            a.fx = __ffma2_rn(fsn, dx, a.fx);
            a.fy = __ffma2_rn(fsn, dy, a.fy);
            a.fz = __ffma2_rn(fsn, dz, a.fz);
            a.np += (unsigned)in0 + (unsigned)in1;
        }
    } else {
        for (int v = 0; v < maxL; ++v) {
            const bool ok = v < L;
            const int j = v + (v < LA ? sA : offB);
            float4 q = pi;
            if (ok) q = __ldg(&p[j]);
            const bool m = OWN ? (ok && j != k) : ok;
            const float dx = q.x - pi.x, dy = q.y - pi.y, dz = q.z - pi.z;
            const float r2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
            if (m && r2 < rc2) {
                const float ir2 = rcp_approx(r2);
                const float s2 = sig2 * ir2;
                const float s6 = s2 * s2 * s2;
                const float s12 = s6 * s6;
                a.e.x += s12 - s6;
                const float t = fmaf(2.0f, s12, -s6);
                a.w.x += t;
                const float fs = t * s2;
                a.fx.x = fmaf(-fs, dx, a.fx.x);
                a.fy.x = fmaf(-fs, dy, a.fy.x);
                a.fz.x = fmaf(-fs, dz, a.fz.x);
                ++a.np;
            }
        }
    }
}

// Packed walk over SoA positions in aligned pairs: step t covers (j, j + 1) with j even, loaded as one
// 8-byte load per coordinate, so each coordinate pair arrives in one register pair.  The pass's
// windows A = [sA, eA) and B = [sB, eB) are rounded out to even starts; elements outside the window
// (and the target itself when OWN) are masked.  x2 / y2 / z2 hold n + 1 readable elements.
template <bool OWN>
__device__ __forceinline__ void walk_pass_soa(const float2* __restrict__ x2, const float2* __restrict__ y2,
                                              const float2* __restrict__ z2, int k, const float4& pi, int sA,
                                              int eA, int sB, int eB, float rc2, float sig2, PassAcc& a) {
    const int aA = sA & ~1, aB = sB & ~1;
    const int PA = eA > sA ? (eA - aA + 1) >> 1 : 0;
    const int PB = eB > sB ? (eB - aB + 1) >> 1 : 0;
    const int P = PA + PB;
    const int hB = (aB >> 1) - PA;  // pair index of step t in window B: hB + t
    const int hA = aA >> 1;
    const int maxP = (int)__reduce_max_sync(0xffffffffu, (unsigned)P);
    const float2 npx = make_float2(-pi.x, -pi.x), npy = make_float2(-pi.y, -pi.y), npz = make_float2(-pi.z, -pi.z);
    const float2 nsig2 = make_float2(-sig2, -sig2), two = make_float2(2.0f, 2.0f);
    float2 qx = make_float2(pi.x, pi.x), qy = make_float2(pi.y, pi.y), qz = make_float2(pi.z, pi.z);
    for (int t = 0; t < maxP; ++t) {
        const bool inA = t < PA;
        const int h = (inA ? hA : hB) + t;
        const int j = 2 * h;
        const int sc = inA ? sA : sB, ec = inA ? eA : eB;
        const bool okp = t < P;
        if (okp) {
            qx = __ldg(&x2[h]);
            qy = __ldg(&y2[h]);
            qz = __ldg(&z2[h]);
        }
        bool m0 = okp && j >= sc, m1 = okp && j + 1 < ec;
        if (OWN) {
            m0 = m0 && j != k;
            m1 = m1 && j + 1 != k;
        }
        const float2 dx = __fadd2_rn(qx, npx);
        const float2 dy = __fadd2_rn(qy, npy);
        const float2 dz = __fadd2_rn(qz, npz);
        const float2 r2 = __ffma2_rn(dz, dz, __ffma2_rn(dy, dy, __fmul2_rn(dx, dx)));
        const bool in0 = m0 && r2.x < rc2, in1 = m1 && r2.y < rc2;
        const float2 ir2 = make_float2(in0 ? rcp_approx(r2.x) : 0.f, in1 ? rcp_approx(r2.y) : 0.f);
        const float2 s2n = __fmul2_rn(nsig2, ir2);
        const float2 s4 = __fmul2_rn(s2n, s2n);
        const float2 ns6 = __fmul2_rn(s4, s2n);
        const float2 s12 = __fmul2_rn(ns6, ns6);
        a.e = __fadd2_rn(a.e, __fadd2_rn(s12, ns6));
        const float2 tt = __ffma2_rn(two, s12, ns6);
        a.w = __fadd2_rn(a.w, tt);
        const float2 fsn = __fmul2_rn(tt, s2n);
        a.fx = __ffma2_rn(fsn, dx, a.fx);
        a.fy = __ffma2_rn(fsn, dy, a.fy);
        a.fz = __ffma2_rn(fsn, dz, a.fz);
        a.np += (unsigned)in0 + (unsigned)in1;
    }
}

// The 9 row windows of target k (local indices in [0, n)): for row r = (dz + 1) * 3 + (dy + 1),
// [ws[r], ws[r] + wl[r]), empty when the row is off the grid or its (y, z) distance bound exceeds the
// cutoff.  `off` holds the offsets of the target's grid; obase is subtracted from them (the index of
// the system's first particle when the offsets count from a larger array).  Same culling, slack and
// searches as pair_target (pair_common.cuh), so the windows are identical.
__device__ __forceinline__ void pass_windows(const GridDev& g, const PairParams& pp, const float4* __restrict__ p,
                                             const int* __restrict__ off, int obase, int n, const float4& pi, int c,
                                             int (&ws)[9], int (&wl)[9]) {
    int cx, cy, cz;
    decode_cell(g, c, cx, cy, cz);
    const int xl = max(cx - 1, 0), xh = min(cx + 1, g.gx - 1);
    const float slack = pp.slack + 8.0f * FLT_EPSILON * fmaxf(fabsf(pi.x), fmaxf(fabsf(pi.y), fabsf(pi.z)));
#pragma unroll
    for (int r = 0; r < 9; ++r) {
        const int dz = r / 3 - 1, dy = r % 3 - 1;
        const int z = cz + dz, y = cy + dy;
        if (z < 0 || z >= g.gz || y < 0 || y >= g.gy) continue;
        float dzm = 0.f, dym = 0.f;
        if (dz < 0) dzm = pi.z - fmaf((float)cz, g.w, g.oz);
        if (dz > 0) dzm = fmaf((float)(cz + 1), g.w, g.oz) - pi.z;
        if (dy < 0) dym = pi.y - fmaf((float)cy, g.w, g.oy);
        if (dy > 0) dym = fmaf((float)(cy + 1), g.w, g.oy) - pi.y;
        dzm = fmaxf(dzm - slack, 0.f);
        dym = fmaxf(dym - slack, 0.f);
        const float d2 = fmaf(dym, dym, dzm * dzm);
        if (d2 >= pp.rc2w) continue;
        const int rb = (z * g.gy + y) * g.gx;
        int s = min(max(__ldg(&off[rb + xl]) - obase, 0), n);
        int e = min(max(__ldg(&off[rb + xh + 1]) - obase, s), n);
        const float h = sqrtf(pp.rc2w - d2) + slack;
        s = lower_x(p, s, e, pi.x - h);
        e = upper_x(p, s, e, pi.x + h);
        ws[r] = s;
        wl[r] = e - s;
    }
}

// As pass_windows, in two phases: first every row's cell range [s, e) is read and L1 hints are issued
// for all of its lines (the ranges of the 32 targets of a warp overlap, so the hints of a warp cover a
// few dozen distinct lines), then the binary searches run.  The searches and the walk then find the
// rows in L1 instead of waiting for each first touch in turn.
__device__ __forceinline__ void pass_windows_pf(const GridDev& g, const PairParams& pp, const float4* __restrict__ p,
                                                const int* __restrict__ off, int obase, int n, const float4& pi, int c,
                                                int (&ws)[9], int (&wl)[9]) {
    int cx, cy, cz;
    decode_cell(g, c, cx, cy, cz);
    const int xl = max(cx - 1, 0), xh = min(cx + 1, g.gx - 1);
    const float slack = pp.slack + 8.0f * FLT_EPSILON * fmaxf(fabsf(pi.x), fmaxf(fabsf(pi.y), fabsf(pi.z)));
    float hs[9];
#pragma unroll
    for (int r = 0; r < 9; ++r) {
        const int dz = r / 3 - 1, dy = r % 3 - 1;
        const int z = cz + dz, y = cy + dy;
        hs[r] = -1.f;
        if (z < 0 || z >= g.gz || y < 0 || y >= g.gy) continue;
        float dzm = 0.f, dym = 0.f;
        if (dz < 0) dzm = pi.z - fmaf((float)cz, g.w, g.oz);
        if (dz > 0) dzm = fmaf((float)(cz + 1), g.w, g.oz) - pi.z;
        if (dy < 0) dym = pi.y - fmaf((float)cy, g.w, g.oy);
        if (dy > 0) dym = fmaf((float)(cy + 1), g.w, g.oy) - pi.y;
        dzm = fmaxf(dzm - slack, 0.f);
        dym = fmaxf(dym - slack, 0.f);
        const float d2 = fmaf(dym, dym, dzm * dzm);
        if (d2 >= pp.rc2w) continue;
        const int rb = (z * g.gy + y) * g.gx;
        const int s = min(max(__ldg(&off[rb + xl]) - obase, 0), n);
        const int e = min(max(__ldg(&off[rb + xh + 1]) - obase, s), n);
        ws[r] = s;
        wl[r] = e;
        hs[r] = sqrtf(pp.rc2w - d2) + slack;
    }
#pragma unroll
    for (int r = 0; r < 9; ++r)
        if (hs[r] >= 0.f)
            for (int q = ws[r] & ~7; q < wl[r]; q += 8) prefetch_l1(p + q);
#pragma unroll
    for (int r = 0; r < 9; ++r) {
        if (hs[r] < 0.f) {
            ws[r] = wl[r] = 0;
            continue;
        }
        const int s = lower_x(p, ws[r], wl[r], pi.x - hs[r]);
        const int e = upper_x(p, s, wl[r], pi.x + hs[r]);
        ws[r] = s;
        wl[r] = e - s;
    }
}

// Per-target pass walk.  Every lane of the warp must call it (inactive lanes with active = false):
// the passes' loop bounds are warp maxima.  MODE 0: scalar, float4 neighbours; 1: packed, float4
// neighbours; 2: packed, SoA neighbours x2 / y2 / z2 (pairs of the local arrays, even-aligned);
// 3: as 1 with clamped loads and L1 hints for the next pass's windows issued before each pass;
// 4: as 1 with the hints only; 5: as 1 with clamped loads only; 6: as 5, with every stencil row's
// lines hinted into L1 before the window searches (pass_windows_pf).
// Indices k, and those of p / x2 / y2 / z2, are local: [0, n).
template <int MODE>
__device__ __forceinline__ void pass_target(const GridDev& g, const PairParams& pp, const float4* __restrict__ p,
                                            const float2* __restrict__ x2, const float2* __restrict__ y2,
                                            const float2* __restrict__ z2, const int* __restrict__ off, int obase,
                                            int n, int k, int c, bool active, PassAcc& a) {
    int ws[9], wl[9];
#pragma unroll
    for (int r = 0; r < 9; ++r) ws[r] = wl[r] = 0;
    float4 pi = make_float4(0.f, 0.f, 0.f, 0.f);
    if (active) {
        pi = __ldg(&p[k]);
        if (MODE == 6)
            pass_windows_pf(g, pp, p, off, obase, n, pi, c, ws, wl);
        else
            pass_windows(g, pp, p, off, obase, n, pi, c, ws, wl);
    }
    a.e = a.w = a.fx = a.fy = a.fz = make_float2(0.f, 0.f);
    a.np = 0;
    const float rc2 = pp.rc2, sig2 = pp.sig2;
    if (MODE == 2) {
        walk_pass_soa<true>(x2, y2, z2, k, pi, ws[4], ws[4] + wl[4], 0, 0, rc2, sig2, a);
        walk_pass_soa<false>(x2, y2, z2, k, pi, ws[3], ws[3] + wl[3], ws[5], ws[5] + wl[5], rc2, sig2, a);
        walk_pass_soa<false>(x2, y2, z2, k, pi, ws[1], ws[1] + wl[1], ws[7], ws[7] + wl[7], rc2, sig2, a);
        walk_pass_soa<false>(x2, y2, z2, k, pi, ws[0], ws[0] + wl[0], ws[8], ws[8] + wl[8], rc2, sig2, a);
        walk_pass_soa<false>(x2, y2, z2, k, pi, ws[2], ws[2] + wl[2], ws[6], ws[6] + wl[6], rc2, sig2, a);
    } else {
        constexpr bool PACKED = MODE != 0;
        constexpr bool CL = MODE == 3 || MODE == 5 || MODE == 6;
        constexpr bool PF = MODE == 3 || MODE == 4;
        if (PF) {
            prefetch_window(p, ws[3], wl[3]);
            prefetch_window(p, ws[5], wl[5]);
        }
        walk_pass<PACKED, true, CL>(p, k, pi, ws[4], wl[4], 0, wl[4], rc2, sig2, a);
        if (PF) {
            prefetch_window(p, ws[1], wl[1]);
            prefetch_window(p, ws[7], wl[7]);
        }
        walk_pass<PACKED, false, CL>(p, k, pi, ws[3], wl[3], ws[5] - wl[3], wl[3] + wl[5], rc2, sig2, a);
        if (PF) {
            prefetch_window(p, ws[0], wl[0]);
            prefetch_window(p, ws[8], wl[8]);
        }
        walk_pass<PACKED, false, CL>(p, k, pi, ws[1], wl[1], ws[7] - wl[1], wl[1] + wl[7], rc2, sig2, a);
        if (PF) {
            prefetch_window(p, ws[2], wl[2]);
            prefetch_window(p, ws[6], wl[6]);
        }
        walk_pass<PACKED, false, CL>(p, k, pi, ws[0], wl[0], ws[8] - wl[0], wl[0] + wl[8], rc2, sig2, a);
        walk_pass<PACKED, false, CL>(p, k, pi, ws[2], wl[2], ws[6] - wl[2], wl[2] + wl[6], rc2, sig2, a);
    }
}

// Copies x, y, z of n sorted float4 records into three arrays (leading dimension ld >= n + 2, two
// zero pads after the last record so the last even-aligned pair is readable).
__global__ void k_split_soa(const float4* __restrict__ p, int n, int ld, float* __restrict__ s);

}  // namespace ljc
