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
// Two candidates per step are evaluated with the sm_100 paired FP32
// instructions (__fadd2_rn / __fmul2_rn / __ffma2_rn), each lane of the pair
// rounding exactly as the scalar operation.  The distance test is therefore
// bit-identical to the scalar kernels (pair counts equal); per-target sums are
// kept as two partial sums (even and odd steps) added at the end.
#pragma once

#include <cfloat>

#include "pair_common.cuh"

namespace ljc {

struct PassAcc {
    float2 e, w, fx, fy, fz;  // two partial sums each (even and odd steps); e, w as in Pass2Acc
    unsigned np;
};

// One pass: window A = [sA, sA + LA), then window B = [offB + LA, offB + L).  OWN: skip j == k.
// A lane past the end of its windows loads record kl (a valid index: the target itself,
// or the last record for a lane without a target) instead of skipping the load, so no default value
// has to be kept in registers; the masks discard it.
template <bool OWN>
__device__ __forceinline__ void walk_pass(const float4* __restrict__ p, int k, int kl, const float4& pi, int sA,
                                          int LA, int offB, int L, float rc2, float sig2, PassAcc& a) {
    const int maxL = (int)__reduce_max_sync(0xffffffffu, (unsigned)L);
    const float2 npx = make_float2(-pi.x, -pi.x), npy = make_float2(-pi.y, -pi.y),
                 npz = make_float2(-pi.z, -pi.z);
    const float2 nsig2 = make_float2(-sig2, -sig2), two = make_float2(2.0f, 2.0f);
    for (int v = 0; v < maxL; v += 2) {
        const int v1 = v + 1;
        const bool ok0 = v < L, ok1 = v1 < L;
        const int j0 = v + (v < LA ? sA : offB);
        const int j1 = v1 + (v1 < LA ? sA : offB);
        const float4 q0 = __ldg(&p[ok0 ? j0 : kl]);
        const float4 q1 = __ldg(&p[ok1 ? j1 : kl]);
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
        const float2 ir2 = make_float2(rcp_hit(in0, r2.x), rcp_hit(in1, r2.y));
        const float2 s2n = __fmul2_rn(nsig2, ir2);  // -s2
        const float2 s4 = __fmul2_rn(s2n, s2n);     // s2 * s2
        const float2 ns6 = __fmul2_rn(s4, s2n);     // -s6
        const float2 s12 = __fmul2_rn(ns6, ns6);    // s6 * s6
        a.e = __fadd2_rn(a.e, s12);                  // sum s12 (converted in pass_target)
        a.w = __fadd2_rn(a.w, ns6);                  // sum -s6
        const float2 t = __ffma2_rn(two, s12, ns6);  // 2 s12 - s6
        const float2 fsn = __fmul2_rn(t, s2n);  // -(t s2): the sums below hold minus the force sums
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

// Per-target pass walk, two candidates per step in paired FP32.  Every lane of the warp must call it
// (inactive lanes with active = false): the passes' loop bounds are warp maxima.  Indices k, and
// those of p, are local: [0, n).
__device__ __forceinline__ void pass_target(const GridDev& g, const PairParams& pp, const float4* __restrict__ p,
                                            const int* __restrict__ off, int obase, int n, int k, int c, bool active,
                                            PassAcc& a) {
    int ws[9], wl[9];
#pragma unroll
    for (int r = 0; r < 9; ++r) ws[r] = wl[r] = 0;
    float4 pi = make_float4(0.f, 0.f, 0.f, 0.f);
    if (active) {
        pi = __ldg(&p[k]);
        pass_windows(g, pp, p, off, obase, n, pi, c, ws, wl);
    }
    a.e = a.w = a.fx = a.fy = a.fz = make_float2(0.f, 0.f);
    a.np = 0;
    const float rc2 = pp.rc2, sig2 = pp.sig2;
    const int kl = min(k, n - 1);
    walk_pass<true>(p, k, kl, pi, ws[4], wl[4], 0, wl[4], rc2, sig2, a);
    walk_pass<false>(p, k, kl, pi, ws[3], wl[3], ws[5] - wl[3], wl[3] + wl[5], rc2, sig2, a);
    walk_pass<false>(p, k, kl, pi, ws[1], wl[1], ws[7] - wl[1], wl[1] + wl[7], rc2, sig2, a);
    walk_pass<false>(p, k, kl, pi, ws[0], wl[0], ws[8] - wl[0], wl[0] + wl[8], rc2, sig2, a);
    walk_pass<false>(p, k, kl, pi, ws[2], wl[2], ws[6] - wl[2], wl[2] + wl[6], rc2, sig2, a);
    const float2 s12 = a.e, ns6 = a.w;
    a.e = __fadd2_rn(s12, ns6);
    a.w = __ffma2_rn(make_float2(2.0f, 2.0f), s12, ns6);
}

}  // namespace ljc

namespace ljc {

// ---------------------------------------------------------------- two targets per lane
// Lane l of a warp takes the consecutive sorted targets a = 2m and b = 2m + 1.  When both lie in the
// same (y, z) row of cells their 9 row windows are merged (per row: one search for the lowest start,
// one for the highest end, over the row's cells from a's cx - 1 to b's cx + 1), and every candidate
// loaded once is tested against both targets in one paired FP32 evaluation: the x, y and z
// differences of (j, a) and (j, b) form the two halves of each packed operand.  Each half rounds as
// the scalar kernels do, so the distance test and the pair count are those of the single-target
// walks.  A lane whose targets lie in different rows walks a's windows with b masked; b's own windows
// are walked afterwards in a second sweep of passes that only warps holding such a lane take.

// During the walk e holds the sum of s^12 and w the sum of -s^6; pass_target2 turns them into the
// energy sum s^12 - s^6 and the virial sum 2 s^12 - s^6 at the end, which saves one paired add per
// candidate over summing the two combinations themselves (measured: 2.33 against 2.37 ms at 10M,
// rc = 0.01).
struct Pass2Acc {
    float2 e, w, fx, fy, fz;  // .x target a, .y target b
    unsigned np;
};

// One packed evaluation of candidate q (index j) against targets (a, b), minus coordinates in nx/ny/nz.
template <bool OWN>
__device__ __forceinline__ void eval2(const float4& q, int j, bool ok, bool useA, bool useB, int ka, int kb,
                                      float2 nx, float2 ny, float2 nz, float rc2, float2 nsig2, Pass2Acc& a) {
    bool ma = ok && useA, mb = ok && useB;
    if (OWN) {
        ma = ma && j != ka;
        mb = mb && j != kb;
    }
    const float2 dx = __fadd2_rn(make_float2(q.x, q.x), nx);
    const float2 dy = __fadd2_rn(make_float2(q.y, q.y), ny);
    const float2 dz = __fadd2_rn(make_float2(q.z, q.z), nz);
    const float2 r2 = __ffma2_rn(dz, dz, __ffma2_rn(dy, dy, __fmul2_rn(dx, dx)));
    const bool ia = ma && r2.x < rc2, ib = mb && r2.y < rc2;
    const float2 ir2 = make_float2(rcp_hit(ia, r2.x), rcp_hit(ib, r2.y));
    const float2 s2n = __fmul2_rn(nsig2, ir2);
    const float2 s4 = __fmul2_rn(s2n, s2n);
    const float2 ns6 = __fmul2_rn(s4, s2n);
    const float2 s12 = __fmul2_rn(ns6, ns6);
    a.e = __fadd2_rn(a.e, s12);
    a.w = __fadd2_rn(a.w, ns6);
    const float2 t = __ffma2_rn(make_float2(2.0f, 2.0f), s12, ns6);
    const float2 fsn = __fmul2_rn(t, s2n);
    a.fx = __ffma2_rn(fsn, dx, a.fx);
    a.fy = __ffma2_rn(fsn, dy, a.fy);
    a.fz = __ffma2_rn(fsn, dz, a.fz);
    a.np += (unsigned)ia + (unsigned)ib;
}

// One pass of two windows (A = [sA, sA + LA), then B = [offB + LA, offB + L)), two candidates per step.
// kl: index loaded by a lane past the end of its windows (valid, masked).
template <bool OWN>
__device__ __forceinline__ void walk_pass2(const float4* __restrict__ p, int ka, int kb, int kl, bool useA, bool useB,
                                           float2 nx, float2 ny, float2 nz, int sA, int LA, int offB, int L,
                                           float rc2, float sig2, Pass2Acc& a) {
    const int maxL = (int)__reduce_max_sync(0xffffffffu, (unsigned)L);
    const float2 nsig2 = make_float2(-sig2, -sig2);
    for (int v = 0; v < maxL; v += 2) {
        const int v1 = v + 1;
        const bool ok0 = v < L, ok1 = v1 < L;
        const int j0 = v + (v < LA ? sA : offB);
        const int j1 = v1 + (v1 < LA ? sA : offB);
        const float4 q0 = __ldg(&p[ok0 ? j0 : kl]);
        const float4 q1 = __ldg(&p[ok1 ? j1 : kl]);
        eval2<OWN>(q0, j0, ok0, useA, useB, ka, kb, nx, ny, nz, rc2, nsig2, a);
        eval2<OWN>(q1, j1, ok1, useA, useB, ka, kb, nx, ny, nz, rc2, nsig2, a);
    }
}

// The lane's non-empty rows (sw[0..nw), start and end) walked end to end as one sequence of L
// candidates, all lanes of the warp in lockstep for the warp's longest sequence, two candidates per
// step.  One pass instead of five: on a sparse grid the rows are short and their lengths vary from
// lane to lane, so five lockstep passes would each wait for their own longest lane.  Every candidate
// is masked against both targets' own indices (the own row is one of the windows).
template <int BLOCK>
__device__ __forceinline__ void walk_flat2(const float4* __restrict__ p, int ka, int kb, int kl, bool useA, bool useB,
                                           float2 nx, float2 ny, float2 nz, const int2 (*sw)[BLOCK], int nw, int L,
                                           float rc2, float sig2, Pass2Acc& a) {
    const int maxL = (int)__reduce_max_sync(0xffffffffu, (unsigned)L);
    const float2 nsig2 = make_float2(-sig2, -sig2);
    const int t = threadIdx.x;
    int w = 0;
    int2 cur = nw > 0 ? sw[0][t] : make_int2(0, 0);  // (next candidate, end of its row)
    for (int v = 0; v < maxL; v += 2) {
        const bool ok0 = v < L, ok1 = v + 1 < L;
        const int j0 = cur.x++;
        if (cur.x == cur.y && w + 1 < nw) cur = sw[++w][t];
        const int j1 = cur.x++;
        if (cur.x == cur.y && w + 1 < nw) cur = sw[++w][t];
        const float4 q0 = __ldg(&p[ok0 ? j0 : kl]);
        const float4 q1 = __ldg(&p[ok1 ? j1 : kl]);
        eval2<true>(q0, j0, ok0, useA, useB, ka, kb, nx, ny, nz, rc2, nsig2, a);
        eval2<true>(q1, j1, ok1, useA, useB, ka, kb, nx, ny, nz, rc2, nsig2, a);
    }
}

// Lower bound of the (y, z) distance from position q to stencil row (dy, dz) of cell (cy, cz), minus
// the slack; d2 >= rc2w culls the row (as pass_windows).
__device__ __forceinline__ float row_d2(const GridDev& g, int cy, int cz, int dy, int dz, float qy, float qz,
                                        float slack) {
    float dzm = 0.f, dym = 0.f;
    if (dz < 0) dzm = qz - fmaf((float)cz, g.w, g.oz);
    if (dz > 0) dzm = fmaf((float)(cz + 1), g.w, g.oz) - qz;
    if (dy < 0) dym = qy - fmaf((float)cy, g.w, g.oy);
    if (dy > 0) dym = fmaf((float)(cy + 1), g.w, g.oy) - qy;
    dzm = fmaxf(dzm - slack, 0.f);
    dym = fmaxf(dym - slack, 0.f);
    return fmaf(dym, dym, dzm * dzm);
}

// Merged windows of targets a (cell (cxa, cy, cz)) and, when useB, b (cell (cxb, cy, cz), cxb >= cxa):
// per row the candidates of both targets' windows (a superset of each), empty when the row is culled
// for both.  Without useB, a's own windows.
__device__ __forceinline__ void pass_windows2(const GridDev& g, const PairParams& pp, const float4* __restrict__ p,
                                              const int* __restrict__ off, int obase, int n, const float4& pa,
                                              const float4& pb, bool useB, int cxa, int cxb, int cy, int cz,
                                              int (&ws)[9], int (&wl)[9]) {
    const int xl = max(cxa - 1, 0), xh = min((useB ? cxb : cxa) + 1, g.gx - 1);
    float m = fmaxf(fabsf(pa.x), fmaxf(fabsf(pa.y), fabsf(pa.z)));
    if (useB) m = fmaxf(m, fmaxf(fabsf(pb.x), fmaxf(fabsf(pb.y), fabsf(pb.z))));
    const float slack = pp.slack + 8.0f * FLT_EPSILON * m;
#pragma unroll
    for (int r = 0; r < 9; ++r) {
        const int dz = r / 3 - 1, dy = r % 3 - 1;
        const int z = cz + dz, y = cy + dy;
        ws[r] = wl[r] = 0;
        if (z < 0 || z >= g.gz || y < 0 || y >= g.gy) continue;
        const float d2a = row_d2(g, cy, cz, dy, dz, pa.y, pa.z, slack);
        const float d2b = useB ? row_d2(g, cy, cz, dy, dz, pb.y, pb.z, slack) : pp.rc2w;
        const bool la = d2a < pp.rc2w, lb = d2b < pp.rc2w;
        if (!la && !lb) continue;
        float lo = 3.4e38f, hi = -3.4e38f;
        if (la) {
            const float h = sqrtf(pp.rc2w - d2a) + slack;
            lo = pa.x - h;
            hi = pa.x + h;
        }
        if (lb) {
            const float h = sqrtf(pp.rc2w - d2b) + slack;
            lo = fminf(lo, pb.x - h);
            hi = fmaxf(hi, pb.x + h);
        }
        const int rb = (z * g.gy + y) * g.gx;
        int s = min(max(__ldg(&off[rb + xl]) - obase, 0), n);
        int e = min(max(__ldg(&off[rb + xh + 1]) - obase, s), n);
        s = lower_x(p, s, e, lo);
        e = upper_x(p, s, e, hi);
        ws[r] = s;
        wl[r] = e - s;
    }
}

// The 5 passes of both targets, the windows read from shared memory (sw[r][threadIdx.x] = (start,
// length) of row r) at the start of each pass, so they hold no registers during the walk.
template <int BLOCK>
__device__ __forceinline__ void passes2_smem(const float4* __restrict__ p, int ka, int kb, int kl, bool useA,
                                             bool useB, float2 nx, float2 ny, float2 nz, const int2 (*sw)[BLOCK],
                                             float rc2, float sig2, Pass2Acc& a) {
    const int t = threadIdx.x;
    {
        const int2 w = sw[4][t];
        walk_pass2<true>(p, ka, kb, kl, useA, useB, nx, ny, nz, w.x, w.y, 0, w.y, rc2, sig2, a);
    }
#pragma unroll 1
    for (int q = 0; q < 4; ++q) {
        // passes (3, 5), (1, 7), (0, 8), (2, 6)
        const int ra = q == 0 ? 3 : (q == 1 ? 1 : (q == 2 ? 0 : 2));
        const int2 A = sw[ra][t], B = sw[8 - ra][t];
        walk_pass2<false>(p, ka, kb, kl, useA, useB, nx, ny, nz, A.x, A.y, B.x - A.y, A.y + B.y, rc2, sig2, a);
    }
}

// Both targets of a lane (a = ka, b = ka + 1; activeA / activeB: inside the target range).  Every
// lane of the warp must call it.  Cells ca, cb are the targets' cells (as read from the sorted cell
// ids).  Results: a.x for target a, a.y for target b.
// sw: shared memory, BLOCK entries per row, where the windows are parked during the walk.
template <int BLOCK = 128>
__device__ __forceinline__ void pass_target2(const GridDev& g, const PairParams& pp, const float4* __restrict__ p,
                                             const int* __restrict__ off, int obase, int n, int ka, int ca, int cb,
                                             bool activeA, bool activeB, Pass2Acc& a, int2 (*sw)[BLOCK]) {
    const int kb = ka + 1;
    float4 pa = make_float4(0.f, 0.f, 0.f, 0.f), pb = pa;
    int ws[9], wl[9];
    int cxa = 0, cya = 0, cza = 0, cxb = 0, cyb = 0, czb = 0;
    if (activeA) {
        pa = __ldg(&p[ka]);
        decode_cell(g, ca, cxa, cya, cza);
    }
    if (activeB) {
        pb = __ldg(&p[kb]);
        decode_cell(g, cb, cxb, cyb, czb);
    }
    const bool same = activeA && activeB && cya == cyb && cza == czb && cxb >= cxa;
    const bool straddle = activeB && !same;  // b walked in the second sweep
    if (activeA) {
        pass_windows2(g, pp, p, off, obase, n, pa, pb, same, cxa, cxb, cya, cza, ws, wl);
    } else {
#pragma unroll
        for (int r = 0; r < 9; ++r) ws[r] = wl[r] = 0;
    }
    a.e = a.w = a.fx = a.fy = a.fz = make_float2(0.f, 0.f);
    a.np = 0;
    const float rc2 = pp.rc2, sig2 = pp.sig2;
    {
        const float2 nx = make_float2(-pa.x, -pb.x), ny = make_float2(-pa.y, -pb.y), nz = make_float2(-pa.z, -pb.z);
#pragma unroll
        for (int r = 0; r < 9; ++r) sw[r][threadIdx.x] = make_int2(ws[r], wl[r]);
        passes2_smem<BLOCK>(p, ka, kb, min(ka, n - 1), activeA, same, nx, ny, nz, sw, rc2, sig2, a);
    }
    if (__any_sync(0xffffffffu, straddle)) {
        if (straddle) {
            pass_windows2(g, pp, p, off, obase, n, pb, pb, false, cxb, cxb, cyb, czb, ws, wl);
        } else {
#pragma unroll
            for (int r = 0; r < 9; ++r) ws[r] = wl[r] = 0;
        }
        const float2 nx = make_float2(-pb.x, -pb.x), ny = make_float2(-pb.y, -pb.y), nz = make_float2(-pb.z, -pb.z);
#pragma unroll
        for (int r = 0; r < 9; ++r) sw[r][threadIdx.x] = make_int2(ws[r], wl[r]);
        passes2_smem<BLOCK>(p, kb, kb, min(kb, n - 1), false, straddle, nx, ny, nz, sw, rc2, sig2, a);
    }
    const float2 s12 = a.e, ns6 = a.w;
    a.e = __fadd2_rn(s12, ns6);
    a.w = __ffma2_rn(make_float2(2.0f, 2.0f), s12, ns6);
}

}  // namespace ljc
