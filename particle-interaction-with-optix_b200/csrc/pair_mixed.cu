// pair_mixed.cu -- the mixed-precision form of the truncated-LJ pair kernel.
//
// Storage.  One 8-byte record per sorted particle: x in FP32, and y, z as
// FP16 offsets from the particle's cell origin in units of the cell width
// (u = (y - (oy + cy w)) / w, rounded to binary16).  Stored positions are
// therefore (x, oy + (cy + uy) w, oz + (cz + uz) w): FP32 cell origin + FP16
// cell-relative offset in y and z, x exact because every stencil row is
// x-sorted and the window search runs on it.  A candidate load moves 8 bytes
// instead of 16.
//
// Arithmetic.  FP32, in cell units: for the stencil row at cell offset
// (dy, dz) the target's frame Ty = uy_i - dy, Tz = uz_i - dz is set once per
// window, so a candidate costs dy = uy_j - Ty, dz = uz_j - Tz and
// dx = (x_j - x_i) / w.  Test r2 < (rc / w)^2 (exactly restated by the oracle).
//
// Accumulation.  Per window a plain FP32 partial; at each window switch the
// partial is added to the running (sum, compensation) pair with TwoSum
// (Knuth), so each particle's energy and force are compensated sums of
// window partials.  Totals (energy, virial, pairs) reduce in FP64 as in
// pair.cu.
#include <cuda_fp16.h>

#include "pair_common.cuh"

namespace ljc {

struct MixParams {
    float invw;    // 1 / cell width
    float w;       // cell width
    float rc2u;    // (cutoff / w)^2 as rc2 * invw * invw: the distance test
    float rc2uw;   // rc2u * (1 + 1e-5): row-skip and window bound
    float sig2u;   // (sigma / w)^2
    float e4;      // 4 eps
    float e24;     // 24 eps
    float fscale;  // -24 eps w / sigma^2: force from the sum of t s2 d (cell units)
    float slack;   // absolute slack of the x window (as pair.cu)
};

// Knuth TwoSum: s + c absorbs the rounding error of adding v.
__device__ __forceinline__ void two_sum_add(float& s, float& c, float v) {
    const float t = s + v;
    const float bp = t - s;
    const float err = (s - (t - bp)) + (v - bp);
    s = t;
    c += err;
}

__global__ void __launch_bounds__(256) k_pack_mixed(GridDev g, const float4* __restrict__ p,
                                                    const int* __restrict__ cs, int n, float2* __restrict__ rec) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const float4 q = p[k];
        int cx, cy, cz;
        int c = cs[k];
        const int nc = g.gx * g.gy * g.gz;
        c = c < 0 ? 0 : (c >= nc ? nc - 1 : c);
        decode_cell(g, c, cx, cy, cz);
        const float uy = __fdiv_rn(__fsub_rn(q.y, fmaf((float)cy, g.w, g.oy)), g.w);
        const float uz = __fdiv_rn(__fsub_rn(q.z, fmaf((float)cz, g.w, g.oz)), g.w);
        const __half2 h = __floats2half2_rn(uy, uz);
        rec[k] = make_float2(q.x, __uint_as_float(*reinterpret_cast<const unsigned*>(&h)));
    }
}

__device__ __forceinline__ float2 unpack_yz(float bits) {
    const unsigned u = __float_as_uint(bits);
    return __half22float2(*reinterpret_cast<const __half2*>(&u));
}

// first j in [lo, hi) with rec[j].x >= v / > v (x-sorted rows)
__device__ __forceinline__ int lower_rx(const float2* __restrict__ r, int lo, int hi, float v) {
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (__ldg(&r[mid].x) < v)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}
__device__ __forceinline__ int upper_rx(const float2* __restrict__ r, int lo, int hi, float v) {
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (__ldg(&r[mid].x) <= v)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

constexpr int kMixThreads = 128;

__global__ void __launch_bounds__(kMixThreads) k_pair_mixed(GridDev g, MixParams mp, const float2* __restrict__ rec,
                                                            const int* __restrict__ cs, const int* __restrict__ off,
                                                            int n, float* __restrict__ energy,
                                                            float* __restrict__ force, Partial* part,
                                                            unsigned* counter, lj_totals* totals, unsigned* status) {
    __shared__ int2 s_win[kMaxWin][kMixThreads];
    __shared__ unsigned char s_row[kMaxWin][kMixThreads];
    const int tid = threadIdx.x;
    const int k = blockIdx.x * kMixThreads + tid;
    float se = 0.f, ce = 0.f, sx = 0.f, cx_ = 0.f, sy = 0.f, cy_ = 0.f, sz = 0.f, cz_ = 0.f, wa = 0.f;
    unsigned np = 0;
    if (k < n) {
        const float2 ri = __ldg(&rec[k]);
        const float xi = ri.x;
        const float2 ui = unpack_yz(ri.y);
        int c = __ldg(&cs[k]);
        if (c < 0 || c >= g.gx * g.gy * g.gz) {
            atomicOr(status, kFlagRange);
            c = 0;
        }
        int cx, cy, cz;
        decode_cell(g, c, cx, cy, cz);
        const int xl = max(cx - 1, 0), xh = min(cx + 1, g.gx - 1);
        const float slack = mp.slack + 8.0f * FLT_EPSILON * fabsf(xi);
        const float slack_u = 1e-5f;
        int nw = 0;
#pragma unroll
        for (int r = 0; r < 9; ++r) {
            const int dz = r / 3 - 1, dy = r % 3 - 1;
            const int z = cz + dz, y = cy + dy;
            if (z < 0 || z >= g.gz || y < 0 || y >= g.gy) continue;
            // lower bound of the (y, z) distance to the row, cell units: rows below/above start at the cell faces
            float dzm = dz < 0 ? ui.y : (dz > 0 ? 1.0f - ui.y : 0.f);
            float dym = dy < 0 ? ui.x : (dy > 0 ? 1.0f - ui.x : 0.f);
            dzm = fmaxf(dzm - slack_u, 0.f);
            dym = fmaxf(dym - slack_u, 0.f);
            const float d2 = fmaf(dym, dym, dzm * dzm);
            if (d2 >= mp.rc2uw) continue;
            const int rb = (z * g.gy + y) * g.gx;
            int s = min(max(__ldg(&off[rb + xl]), 0), n);
            int e = min(max(__ldg(&off[rb + xh + 1]), s), n);
            const float h = sqrtf(mp.rc2uw - d2) * mp.w + slack;
            s = lower_rx(rec, s, e, xi - h);
            e = upper_rx(rec, s, e, xi + h);
            if (r == 4) {
                s_win[nw][tid] = make_int2(s, k);
                s_row[nw++][tid] = (unsigned char)r;
                s_win[nw][tid] = make_int2(k + 1, e);
                s_row[nw++][tid] = (unsigned char)r;
            } else {
                s_win[nw][tid] = make_int2(s, e);
                s_row[nw++][tid] = (unsigned char)r;
            }
        }
        const float rc2u = mp.rc2u, sig2u = mp.sig2u, invw = mp.invw;
        // flat walk over the windows (the own row always gives two, so nw >= 2)
        int w = 0;
        int2 cur = s_win[0][tid];
        int r = s_row[0][tid];
        float ty = ui.x - (float)(r % 3 - 1), tz = ui.y - (float)(r / 3 - 1);
        float pe = 0.f, px = 0.f, py = 0.f, pz = 0.f;
        while (true) {
            if (cur.x >= cur.y) {
                // window done: add its partial sums with compensation
                two_sum_add(se, ce, pe);
                two_sum_add(sx, cx_, px);
                two_sum_add(sy, cy_, py);
                two_sum_add(sz, cz_, pz);
                pe = px = py = pz = 0.f;
                do {
                    if (++w >= nw) goto walked;
                    cur = s_win[w][tid];
                } while (cur.x >= cur.y);
                r = s_row[w][tid];
                ty = ui.x - (float)(r % 3 - 1);
                tz = ui.y - (float)(r / 3 - 1);
            }
            {
                const float2 q = __ldg(&rec[cur.x]);
                ++cur.x;
                const float2 uj = unpack_yz(q.y);
                const float dx = __fmul_rn(__fsub_rn(q.x, xi), invw);
                const float dy = __fsub_rn(uj.x, ty);
                const float dz = __fsub_rn(uj.y, tz);
                const float r2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
                if (r2 < rc2u) {
                    const float ir2 = rcp_approx(r2);
                    const float s2 = sig2u * ir2;
                    const float s6 = s2 * s2 * s2;
                    const float s12 = s6 * s6;
                    pe += s12 - s6;
                    const float t = fmaf(2.0f, s12, -s6);
                    wa += t;
                    const float fs = t * s2;
                    px = fmaf(fs, dx, px);
                    py = fmaf(fs, dy, py);
                    pz = fmaf(fs, dz, pz);
                    ++np;
                }
            }
        }
    walked:
        if (energy) energy[k] = mp.e4 * (se + ce);
        if (force) {
            force[3 * (size_t)k + 0] = mp.fscale * (sx + cx_);
            force[3 * (size_t)k + 1] = mp.fscale * (sy + cy_);
            force[3 * (size_t)k + 2] = mp.fscale * (sz + cz_);
        }
    }
    reduce_totals<kMixThreads>(0.5 * (double)mp.e4 * ((double)se + (double)ce), 0.5 * (double)mp.e24 * (double)wa,
                               (unsigned long long)np, part, counter, totals);
}

// The same with the windows in registers (slot r = stencil row r, slot 9 =
// the own row after the target), walked by shifting: no shared memory, so the
// whole L1 caches neighbour records.  Faster on dense grids, as for the plain
// form (pair_direct.cu).
__global__ void __launch_bounds__(kMixThreads) k_pair_mixed_reg(GridDev g, MixParams mp,
                                                                const float2* __restrict__ rec,
                                                                const int* __restrict__ cs,
                                                                const int* __restrict__ off, int n,
                                                                float* __restrict__ energy, float* __restrict__ force,
                                                                Partial* part, unsigned* counter, lj_totals* totals,
                                                                unsigned* status) {
    const int k = blockIdx.x * kMixThreads + threadIdx.x;
    float se = 0.f, ce = 0.f, sx = 0.f, cx_ = 0.f, sy = 0.f, cy_ = 0.f, sz = 0.f, cz_ = 0.f, wa = 0.f;
    unsigned np = 0;
    if (k < n) {
        const float2 ri = __ldg(&rec[k]);
        const float xi = ri.x;
        const float2 ui = unpack_yz(ri.y);
        int c = __ldg(&cs[k]);
        if (c < 0 || c >= g.gx * g.gy * g.gz) {
            atomicOr(status, kFlagRange);
            c = 0;
        }
        int cx, cy, cz;
        decode_cell(g, c, cx, cy, cz);
        const int xl = max(cx - 1, 0), xh = min(cx + 1, g.gx - 1);
        const float slack = mp.slack + 8.0f * FLT_EPSILON * fabsf(xi);
        int2 slot[10];
#pragma unroll
        for (int i = 0; i < 10; ++i) slot[i] = make_int2(0, 0);
#pragma unroll
        for (int r = 0; r < 9; ++r) {
            const int dz = r / 3 - 1, dy = r % 3 - 1;
            const int z = cz + dz, y = cy + dy;
            if (z < 0 || z >= g.gz || y < 0 || y >= g.gy) continue;
            float dzm = dz < 0 ? ui.y : (dz > 0 ? 1.0f - ui.y : 0.f);
            float dym = dy < 0 ? ui.x : (dy > 0 ? 1.0f - ui.x : 0.f);
            dzm = fmaxf(dzm - 1e-5f, 0.f);
            dym = fmaxf(dym - 1e-5f, 0.f);
            const float d2 = fmaf(dym, dym, dzm * dzm);
            if (d2 >= mp.rc2uw) continue;
            const int rb = (z * g.gy + y) * g.gx;
            const int s = min(max(__ldg(&off[rb + xl]), 0), n);
            const int e = min(max(__ldg(&off[rb + xh + 1]), s), n);
            const float h = sqrtf(mp.rc2uw - d2) * mp.w + slack;
            const int lo = lower_rx(rec, s, e, xi - h);
            const int hi = upper_rx(rec, lo, e, xi + h);
            if (r == 4) {
                slot[4] = make_int2(lo, k);
                slot[9] = make_int2(k + 1, hi);
            } else {
                slot[r] = make_int2(lo, hi);
            }
        }
        const float rc2u = mp.rc2u, sig2u = mp.sig2u, invw = mp.invw;
        int idx = 0;  // slot being walked; its row is idx (idx < 9) or 4 (idx = 9)
        int2 cur = slot[0];
        float ty = ui.x + 1.0f, tz = ui.y + 1.0f;  // row 0: dy = dz = -1
        float pe = 0.f, px = 0.f, py = 0.f, pz = 0.f;
        while (true) {
            if (cur.x >= cur.y) {
                two_sum_add(se, ce, pe);
                two_sum_add(sx, cx_, px);
                two_sum_add(sy, cy_, py);
                two_sum_add(sz, cz_, pz);
                pe = px = py = pz = 0.f;
                do {
                    if (++idx == 10) goto walked;
                    cur = slot[1];
#pragma unroll
                    for (int i = 1; i < 9; ++i) slot[i] = slot[i + 1];
                    slot[9] = make_int2(0, 0);
                } while (cur.x >= cur.y);
                const int row = idx < 9 ? idx : 4;
                ty = ui.x - (float)(row % 3 - 1);
                tz = ui.y - (float)(row / 3 - 1);
            }
            {
                const float2 q = __ldg(&rec[cur.x]);
                ++cur.x;
                const float2 uj = unpack_yz(q.y);
                const float dx = __fmul_rn(__fsub_rn(q.x, xi), invw);
                const float dy = __fsub_rn(uj.x, ty);
                const float dz = __fsub_rn(uj.y, tz);
                const float r2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
                if (r2 < rc2u) {
                    const float ir2 = rcp_approx(r2);
                    const float s2 = sig2u * ir2;
                    const float s6 = s2 * s2 * s2;
                    const float s12 = s6 * s6;
                    pe += s12 - s6;
                    const float t = fmaf(2.0f, s12, -s6);
                    wa += t;
                    const float fs = t * s2;
                    px = fmaf(fs, dx, px);
                    py = fmaf(fs, dy, py);
                    pz = fmaf(fs, dz, pz);
                    ++np;
                }
            }
        }
    walked:
        if (energy) energy[k] = mp.e4 * (se + ce);
        if (force) {
            force[3 * (size_t)k + 0] = mp.fscale * (sx + cx_);
            force[3 * (size_t)k + 1] = mp.fscale * (sy + cy_);
            force[3 * (size_t)k + 2] = mp.fscale * (sz + cz_);
        }
    }
    reduce_totals<kMixThreads>(0.5 * (double)mp.e4 * ((double)se + (double)ce), 0.5 * (double)mp.e24 * (double)wa,
                               (unsigned long long)np, part, counter, totals);
}

// ---------------------------------------------------------------- row passes
// The mixed records walked as the plain default walks its float4 records (pair_pass.cuh): the 9 rows
// in 5 warp-synchronous passes (own row; then opposite rows paired), two candidates per step in the
// paired FP32 instructions, each half rounding as the scalar kernels above, so the distance test and
// the pair count are those of k_pair_mixed.  Each candidate takes the target frame of its row.  Sums:
// per pass two FP32 partials (even and odd steps), added to the running (sum, compensation) pairs with
// TwoSum when the pass ends.

struct MixPassAcc {
    float se, ce, sx, cx, sy, cy, sz, cz;  // compensated sums
    float2 w;                              // virial partials (the totals reduce in FP64)
    unsigned np;
};

__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }

// One pass: window A = [sA, sA + LA) of row ra, then window B = [offB + LA, offB + L) of row rb.
// kl: index loaded by a lane past the end of its windows (valid; the masks discard it).
template <bool OWN>
__device__ __forceinline__ void mix_walk_pass(const float2* __restrict__ rec, int k, int kl, float xi, float2 ui, int ra,
                                              int sA, int LA, int rb, int offB, int L, const MixParams& mp,
                                              MixPassAcc& a) {
    const int maxL = (int)__reduce_max_sync(0xffffffffu, (unsigned)L);
    const float ntyA = (float)(ra % 3 - 1) - ui.x, ntzA = (float)(ra / 3 - 1) - ui.y;
    const float ntyB = (float)(rb % 3 - 1) - ui.x, ntzB = (float)(rb / 3 - 1) - ui.y;
    const float2 nxi = f2(-xi, -xi), invw = f2(mp.invw, mp.invw), nsig2 = f2(-mp.sig2u, -mp.sig2u),
                 two = f2(2.0f, 2.0f);
    const float rc2 = mp.rc2u;
    float2 pe = f2(0.f, 0.f), px = pe, py = pe, pz = pe;
    for (int v = 0; v < maxL; v += 2) {
        const int v1 = v + 1;
        const bool ok0 = v < L, ok1 = v1 < L;
        const bool a0 = v < LA, a1 = v1 < LA;
        const int j0 = v + (a0 ? sA : offB);
        const int j1 = v1 + (a1 ? sA : offB);
        const float2 q0 = __ldg(&rec[ok0 ? j0 : kl]);
        const float2 q1 = __ldg(&rec[ok1 ? j1 : kl]);
        bool m0 = ok0, m1 = ok1;
        if (OWN) {
            m0 = m0 && j0 != k;
            m1 = m1 && j1 != k;
        }
        const float2 u0 = unpack_yz(q0.y), u1 = unpack_yz(q1.y);
        const float2 dx = __fmul2_rn(__fadd2_rn(f2(q0.x, q1.x), nxi), invw);
        const float2 dy = __fadd2_rn(f2(u0.x, u1.x), f2(a0 ? ntyA : ntyB, a1 ? ntyA : ntyB));
        const float2 dz = __fadd2_rn(f2(u0.y, u1.y), f2(a0 ? ntzA : ntzB, a1 ? ntzA : ntzB));
        const float2 r2 = __ffma2_rn(dz, dz, __ffma2_rn(dy, dy, __fmul2_rn(dx, dx)));
        const bool in0 = m0 && r2.x < rc2, in1 = m1 && r2.y < rc2;
        const float2 ir2 = f2(rcp_hit(in0, r2.x), rcp_hit(in1, r2.y));
        const float2 s2n = __fmul2_rn(nsig2, ir2);
        const float2 s4 = __fmul2_rn(s2n, s2n);
        const float2 ns6 = __fmul2_rn(s4, s2n);
        const float2 s12 = __fmul2_rn(ns6, ns6);
        pe = __fadd2_rn(pe, __fadd2_rn(s12, ns6));
        const float2 t = __ffma2_rn(two, s12, ns6);
        a.w = __fadd2_rn(a.w, t);
        const float2 fsn = __fmul2_rn(t, s2n);  // minus the force sums, as in pair_pass.cuh
        px = __ffma2_rn(fsn, dx, px);
        py = __ffma2_rn(fsn, dy, py);
        pz = __ffma2_rn(fsn, dz, pz);
        a.np += (unsigned)in0 + (unsigned)in1;
    }
    two_sum_add(a.se, a.ce, pe.x);
    two_sum_add(a.se, a.ce, pe.y);
    two_sum_add(a.sx, a.cx, -px.x);
    two_sum_add(a.sx, a.cx, -px.y);
    two_sum_add(a.sy, a.cy, -py.x);
    two_sum_add(a.sy, a.cy, -py.y);
    two_sum_add(a.sz, a.cz, -pz.x);
    two_sum_add(a.sz, a.cz, -pz.y);
}

__global__ void __launch_bounds__(kMixThreads) k_pair_mixed_pass(GridDev g, MixParams mp,
                                                                 const float2* __restrict__ rec,
                                                                 const int* __restrict__ cs,
                                                                 const int* __restrict__ off, int n,
                                                                 float* __restrict__ energy, float* __restrict__ force,
                                                                 Partial* part, unsigned* counter, lj_totals* totals,
                                                                 unsigned* status) {
    const int k = blockIdx.x * kMixThreads + threadIdx.x;
    const bool active = k < n;
    int ws[9], wl[9];
#pragma unroll
    for (int r = 0; r < 9; ++r) ws[r] = wl[r] = 0;
    float xi = 0.f;
    float2 ui = f2(0.f, 0.f);
    if (active) {
        const float2 ri = __ldg(&rec[k]);
        xi = ri.x;
        ui = unpack_yz(ri.y);
        int c = __ldg(&cs[k]);
        if (c < 0 || c >= g.gx * g.gy * g.gz) {
            atomicOr(status, kFlagRange);
            c = 0;
        }
        int cx, cy, cz;
        decode_cell(g, c, cx, cy, cz);
        const int xl = max(cx - 1, 0), xh = min(cx + 1, g.gx - 1);
        const float slack = mp.slack + 8.0f * FLT_EPSILON * fabsf(xi);
        // the windows of k_pair_mixed_reg
#pragma unroll
        for (int r = 0; r < 9; ++r) {
            const int dz = r / 3 - 1, dy = r % 3 - 1;
            const int z = cz + dz, y = cy + dy;
            if (z < 0 || z >= g.gz || y < 0 || y >= g.gy) continue;
            float dzm = dz < 0 ? ui.y : (dz > 0 ? 1.0f - ui.y : 0.f);
            float dym = dy < 0 ? ui.x : (dy > 0 ? 1.0f - ui.x : 0.f);
            dzm = fmaxf(dzm - 1e-5f, 0.f);
            dym = fmaxf(dym - 1e-5f, 0.f);
            const float d2 = fmaf(dym, dym, dzm * dzm);
            if (d2 >= mp.rc2uw) continue;
            const int rb = (z * g.gy + y) * g.gx;
            const int s = min(max(__ldg(&off[rb + xl]), 0), n);
            const int e = min(max(__ldg(&off[rb + xh + 1]), s), n);
            const float h = sqrtf(mp.rc2uw - d2) * mp.w + slack;
            const int lo = lower_rx(rec, s, e, xi - h);
            const int hi = upper_rx(rec, lo, e, xi + h);
            ws[r] = lo;
            wl[r] = hi - lo;
        }
    }
    const int kl = min(k, n - 1);
    MixPassAcc a;
    a.se = a.ce = a.sx = a.cx = a.sy = a.cy = a.sz = a.cz = 0.f;
    a.w = f2(0.f, 0.f);
    a.np = 0;
    mix_walk_pass<true>(rec, k, kl, xi, ui, 4, ws[4], wl[4], 4, 0, wl[4], mp, a);
    mix_walk_pass<false>(rec, k, kl, xi, ui, 3, ws[3], wl[3], 5, ws[5] - wl[3], wl[3] + wl[5], mp, a);
    mix_walk_pass<false>(rec, k, kl, xi, ui, 1, ws[1], wl[1], 7, ws[7] - wl[1], wl[1] + wl[7], mp, a);
    mix_walk_pass<false>(rec, k, kl, xi, ui, 0, ws[0], wl[0], 8, ws[8] - wl[0], wl[0] + wl[8], mp, a);
    mix_walk_pass<false>(rec, k, kl, xi, ui, 2, ws[2], wl[2], 6, ws[6] - wl[2], wl[2] + wl[6], mp, a);
    if (active) {
        if (energy) energy[k] = mp.e4 * (a.se + a.ce);
        if (force) {
            force[3 * (size_t)k + 0] = mp.fscale * (a.sx + a.cx);
            force[3 * (size_t)k + 1] = mp.fscale * (a.sy + a.cy);
            force[3 * (size_t)k + 2] = mp.fscale * (a.sz + a.cz);
        }
    }
    reduce_totals<kMixThreads>(0.5 * (double)mp.e4 * ((double)a.se + (double)a.ce),
                               0.5 * (double)mp.e24 * ((double)a.w.x + (double)a.w.y), (unsigned long long)a.np,
                               part, counter, totals);
}

// ---------------------------------------------------------------- two targets per lane
// The mixed records on the two-target walk of pair_pass.cuh (pass_target2): lane m takes the
// consecutive sorted targets a = 2m and b = 2m + 1; when they share a (y, z) row of cells their
// windows are merged and each record is loaded once and evaluated against both, the two halves of
// every packed operand holding (j - a) and (j - b) in cell units.  A lane whose targets lie in
// different rows walks b in a second sweep.  Each half rounds as k_pair_mixed, so the distance test
// and the pair count are unchanged; per-target sums are compensated per pass (TwoSum), as above.

struct MixAcc2 {
    float2 se, ce, sx, cx, sy, cy, sz, cz;  // compensated sums, .x target a, .y target b
    float2 w;
    unsigned np;
};

__device__ __forceinline__ void two_sum_add2(float2& s, float2& c, float2 v) {
    two_sum_add(s.x, c.x, v.x);
    two_sum_add(s.y, c.y, v.y);
}

template <bool OWN>
__device__ __forceinline__ void mix_walk_pass2(const float2* __restrict__ rec, int ka, int kb, int kl, bool useA,
                                               bool useB, float2 nx, float2 ntyA, float2 ntzA, float2 ntyB,
                                               float2 ntzB, int sA, int LA, int offB, int L, const MixParams& mp,
                                               MixAcc2& a) {
    const int maxL = (int)__reduce_max_sync(0xffffffffu, (unsigned)L);
    const float2 invw = f2(mp.invw, mp.invw), nsig2 = f2(-mp.sig2u, -mp.sig2u), two = f2(2.0f, 2.0f);
    const float rc2 = mp.rc2u;
    float2 pe = f2(0.f, 0.f), px = pe, py = pe, pz = pe;
    auto eval = [&](const float2& q, int j, bool ok, bool inA) {
        bool ma = ok && useA, mb = ok && useB;
        if (OWN) {
            ma = ma && j != ka;
            mb = mb && j != kb;
        }
        const float2 u = unpack_yz(q.y);
        const float2 dx = __fmul2_rn(__fadd2_rn(f2(q.x, q.x), nx), invw);
        const float2 dy = __fadd2_rn(f2(u.x, u.x), inA ? ntyA : ntyB);
        const float2 dz = __fadd2_rn(f2(u.y, u.y), inA ? ntzA : ntzB);
        const float2 r2 = __ffma2_rn(dz, dz, __ffma2_rn(dy, dy, __fmul2_rn(dx, dx)));
        const bool ia = ma && r2.x < rc2, ib = mb && r2.y < rc2;
        const float2 ir2 = f2(rcp_hit(ia, r2.x), rcp_hit(ib, r2.y));
        const float2 s2n = __fmul2_rn(nsig2, ir2);
        const float2 s4 = __fmul2_rn(s2n, s2n);
        const float2 ns6 = __fmul2_rn(s4, s2n);
        const float2 s12 = __fmul2_rn(ns6, ns6);
        pe = __fadd2_rn(pe, __fadd2_rn(s12, ns6));
        const float2 t = __ffma2_rn(two, s12, ns6);
        a.w = __fadd2_rn(a.w, t);
        const float2 fsn = __fmul2_rn(t, s2n);
        px = __ffma2_rn(fsn, dx, px);
        py = __ffma2_rn(fsn, dy, py);
        pz = __ffma2_rn(fsn, dz, pz);
        a.np += (unsigned)ia + (unsigned)ib;
    };
    // two candidates per step: both records are loaded before either is evaluated
    for (int v = 0; v < maxL; v += 2) {
        const int v1 = v + 1;
        const bool ok0 = v < L, ok1 = v1 < L;
        const bool inA0 = v < LA, inA1 = v1 < LA;
        const int j0 = v + (inA0 ? sA : offB), j1 = v1 + (inA1 ? sA : offB);
        const float2 q0 = __ldg(&rec[ok0 ? j0 : kl]);
        const float2 q1 = __ldg(&rec[ok1 ? j1 : kl]);
        eval(q0, j0, ok0, inA0);
        eval(q1, j1, ok1, inA1);
    }
    two_sum_add2(a.se, a.ce, pe);
    two_sum_add2(a.sx, a.cx, f2(-px.x, -px.y));
    two_sum_add2(a.sy, a.cy, f2(-py.x, -py.y));
    two_sum_add2(a.sz, a.cz, f2(-pz.x, -pz.y));
}

// Merged mixed windows of a (and b when useB): per row the union of both targets' x windows over the
// row's cells from a's cx - 1 to b's cx + 1, culled for a target by its cell-unit (y, z) bound.
__device__ __forceinline__ void mix_windows2(const GridDev& g, const MixParams& mp, const float2* __restrict__ rec,
                                             const int* __restrict__ off, int n, float xa, float2 ua, float xb,
                                             float2 ub, bool useB, int cxa, int cxb, int cy, int cz, int (&ws)[9],
                                             int (&wl)[9]) {
    const int xl = max(cxa - 1, 0), xh = min((useB ? cxb : cxa) + 1, g.gx - 1);
    const float slack = mp.slack + 8.0f * FLT_EPSILON * fmaxf(fabsf(xa), useB ? fabsf(xb) : 0.f);
#pragma unroll
    for (int r = 0; r < 9; ++r) {
        const int dz = r / 3 - 1, dy = r % 3 - 1;
        const int z = cz + dz, y = cy + dy;
        ws[r] = wl[r] = 0;
        if (z < 0 || z >= g.gz || y < 0 || y >= g.gy) continue;
        auto d2_of = [&](float2 u) {
            float dzm = dz < 0 ? u.y : (dz > 0 ? 1.0f - u.y : 0.f);
            float dym = dy < 0 ? u.x : (dy > 0 ? 1.0f - u.x : 0.f);
            dzm = fmaxf(dzm - 1e-5f, 0.f);
            dym = fmaxf(dym - 1e-5f, 0.f);
            return fmaf(dym, dym, dzm * dzm);
        };
        const float d2a = d2_of(ua);
        const float d2b = useB ? d2_of(ub) : mp.rc2uw;
        const bool la = d2a < mp.rc2uw, lb = d2b < mp.rc2uw;
        if (!la && !lb) continue;
        float lo = 3.4e38f, hi = -3.4e38f;
        if (la) {
            const float h = sqrtf(mp.rc2uw - d2a) * mp.w + slack;
            lo = xa - h;
            hi = xa + h;
        }
        if (lb) {
            const float h = sqrtf(mp.rc2uw - d2b) * mp.w + slack;
            lo = fminf(lo, xb - h);
            hi = fmaxf(hi, xb + h);
        }
        const int rb = (z * g.gy + y) * g.gx;
        const int s0 = min(max(__ldg(&off[rb + xl]), 0), n);
        const int e0 = min(max(__ldg(&off[rb + xh + 1]), s0), n);
        const int lo_i = lower_rx(rec, s0, e0, lo);
        const int hi_i = upper_rx(rec, lo_i, e0, hi);
        ws[r] = lo_i;
        wl[r] = hi_i - lo_i;
    }
}

template <int BLOCK>
__device__ __forceinline__ void mix_passes2(const float2* __restrict__ rec, int ka, int kb, int kl, bool useA,
                                            bool useB, float2 nx, float2 uy, float2 uz, const int2 (*sw)[BLOCK],
                                            const MixParams& mp, MixAcc2& a) {
    const int t = threadIdx.x;
    // frame of row r for both halves: minus (u - row offset)
    auto nty = [&](int r) { return f2((float)(r % 3 - 1) - uy.x, (float)(r % 3 - 1) - uy.y); };
    auto ntz = [&](int r) { return f2((float)(r / 3 - 1) - uz.x, (float)(r / 3 - 1) - uz.y); };
    {
        const int2 w = sw[4][t];
        mix_walk_pass2<true>(rec, ka, kb, kl, useA, useB, nx, nty(4), ntz(4), nty(4), ntz(4), w.x, w.y, 0, w.y, mp, a);
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int ra = q == 0 ? 3 : (q == 1 ? 1 : (q == 2 ? 0 : 2));
        const int rb = 8 - ra;
        const int2 A = sw[ra][t], B = sw[rb][t];
        mix_walk_pass2<false>(rec, ka, kb, kl, useA, useB, nx, nty(ra), ntz(ra), nty(rb), ntz(rb), A.x, A.y,
                              B.x - A.y, A.y + B.y, mp, a);
    }
}

__global__ void __launch_bounds__(kMixThreads, 6) k_pair_mixed_pass2(GridDev g, MixParams mp,
                                                                     const float2* __restrict__ rec,
                                                                     const int* __restrict__ cs,
                                                                     const int* __restrict__ off, int n,
                                                                     float* __restrict__ energy,
                                                                     float* __restrict__ force, Partial* part,
                                                                     unsigned* counter, lj_totals* totals,
                                                                     unsigned* status) {
    __shared__ int2 s_win[9][kMixThreads];
    const int ka = 2 * (blockIdx.x * kMixThreads + threadIdx.x);
    const int kb = ka + 1;
    const bool activeA = ka < n, activeB = kb < n;
    const int ncell = g.gx * g.gy * g.gz;
    float xa = 0.f, xb = 0.f;
    float2 ua = f2(0.f, 0.f), ub = ua;
    int cxa = 0, cya = 0, cza = 0, cxb = 0, cyb = 0, czb = 0;
    if (activeA) {
        const float2 r = __ldg(&rec[ka]);
        xa = r.x;
        ua = unpack_yz(r.y);
        int c = __ldg(&cs[ka]);
        if (c < 0 || c >= ncell) {
            atomicOr(status, kFlagRange);
            c = 0;
        }
        decode_cell(g, c, cxa, cya, cza);
    }
    if (activeB) {
        const float2 r = __ldg(&rec[kb]);
        xb = r.x;
        ub = unpack_yz(r.y);
        int c = __ldg(&cs[kb]);
        if (c < 0 || c >= ncell) {
            atomicOr(status, kFlagRange);
            c = 0;
        }
        decode_cell(g, c, cxb, cyb, czb);
    }
    const bool same = activeA && activeB && cya == cyb && cza == czb && cxb >= cxa;
    const bool straddle = activeB && !same;
    MixAcc2 a;
    a.se = a.ce = a.sx = a.cx = a.sy = a.cy = a.sz = a.cz = a.w = f2(0.f, 0.f);
    a.np = 0;
    {
        int ws[9], wl[9];
        if (activeA) {
            mix_windows2(g, mp, rec, off, n, xa, ua, xb, ub, same, cxa, cxb, cya, cza, ws, wl);
        } else {
#pragma unroll
            for (int r = 0; r < 9; ++r) ws[r] = wl[r] = 0;
        }
#pragma unroll
        for (int r = 0; r < 9; ++r) s_win[r][threadIdx.x] = make_int2(ws[r], wl[r]);
    }
    mix_passes2<kMixThreads>(rec, ka, kb, min(ka, n - 1), activeA, same, f2(-xa, -xb), f2(ua.x, ub.x),
                             f2(ua.y, ub.y), s_win, mp, a);
    if (__any_sync(0xffffffffu, straddle)) {
        {
            int ws[9], wl[9];
            if (straddle) {
                mix_windows2(g, mp, rec, off, n, xb, ub, xb, ub, false, cxb, cxb, cyb, czb, ws, wl);
            } else {
#pragma unroll
                for (int r = 0; r < 9; ++r) ws[r] = wl[r] = 0;
            }
#pragma unroll
            for (int r = 0; r < 9; ++r) s_win[r][threadIdx.x] = make_int2(ws[r], wl[r]);
        }
        mix_passes2<kMixThreads>(rec, kb, kb, min(kb, n - 1), false, straddle, f2(-xb, -xb), f2(ub.x, ub.x),
                                 f2(ub.y, ub.y), s_win, mp, a);
    }
    if (activeA) {
        if (energy) energy[ka] = mp.e4 * (a.se.x + a.ce.x);
        if (force) {
            force[3 * (size_t)ka + 0] = mp.fscale * (a.sx.x + a.cx.x);
            force[3 * (size_t)ka + 1] = mp.fscale * (a.sy.x + a.cy.x);
            force[3 * (size_t)ka + 2] = mp.fscale * (a.sz.x + a.cz.x);
        }
    }
    if (activeB) {
        if (energy) energy[kb] = mp.e4 * (a.se.y + a.ce.y);
        if (force) {
            force[3 * (size_t)kb + 0] = mp.fscale * (a.sx.y + a.cx.y);
            force[3 * (size_t)kb + 1] = mp.fscale * (a.sy.y + a.cy.y);
            force[3 * (size_t)kb + 2] = mp.fscale * (a.sz.y + a.cz.y);
        }
    }
    reduce_totals<kMixThreads>(
        0.5 * (double)mp.e4 * ((double)a.se.x + (double)a.ce.x + (double)a.se.y + (double)a.ce.y),
        0.5 * (double)mp.e24 * ((double)a.w.x + (double)a.w.y), (unsigned long long)a.np, part, counter, totals);
}

}  // namespace ljc

using namespace ljc;

extern "C" lj_status lj_pack_mixed(lj_ctx* ctx, const lj_grid* g, int n, const float* sorted_xyzi,
                                   const int* sorted_cell, float* rec) {
    const NvtxRange nvtx_range("lj_pack_mixed");
    if (!ctx || !g || n < 0 || (n > 0 && (!sorted_xyzi || !sorted_cell || !rec))) return LJ_EINVAL;
    if (!(g->width > 0.0f) || g->dim[0] < 1 || g->dim[1] < 1 || g->dim[2] < 1) return LJ_EINVAL;
    if ((reinterpret_cast<uintptr_t>(sorted_xyzi) & 15) || (reinterpret_cast<uintptr_t>(rec) & 7)) return LJ_EINVAL;
    if (n == 0) return LJ_OK;
    int blocks = (n + 255) / 256;
    if (blocks > ctx->sm_count * 8) blocks = ctx->sm_count * 8;
    k_pack_mixed<<<blocks, 256, 0, ctx->stream>>>(to_dev(*g), reinterpret_cast<const float4*>(sorted_xyzi),
                                                  sorted_cell, n, reinterpret_cast<float2*>(rec));
    return last_launch_status();
}

extern "C" lj_status lj_compute_mixed(lj_ctx* ctx, const lj_grid* g, const lj_params* p, int n, const float* rec,
                                      const int* sorted_cell, const int* offsets, float* energy, float* force,
                                      lj_totals* totals) {
    const NvtxRange nvtx_range("lj_compute_mixed");
    if (!ctx || !g || !p || n < 0 || (n > 0 && (!rec || !sorted_cell || !offsets))) return LJ_EINVAL;
    if (!(g->width > 0.0f) || g->dim[0] < 1 || g->dim[1] < 1 || g->dim[2] < 1) return LJ_EINVAL;
    if (!(p->cutoff > 0.0f) || !(p->cutoff <= g->width) || !(p->sigma > 0.0f)) return LJ_EINVAL;
    if (reinterpret_cast<uintptr_t>(rec) & 7) return LJ_EINVAL;
    if (n == 0) {
        if (totals && cudaMemsetAsync(totals, 0, sizeof(lj_totals), ctx->stream) != cudaSuccess) return LJ_ECUDA;
        return LJ_OK;
    }
    MixParams mp;
    mp.w = g->width;
    mp.invw = 1.0f / g->width;
    const float rc2 = p->cutoff * p->cutoff;
    mp.rc2u = rc2 * mp.invw * mp.invw;
    mp.rc2uw = mp.rc2u * (1.0f + 1e-5f);
    const float sig2 = p->sigma * p->sigma;
    mp.sig2u = sig2 * mp.invw * mp.invw;
    mp.e4 = 4.0f * p->epsilon;
    mp.e24 = 24.0f * p->epsilon;
    mp.fscale = -mp.e24 * g->width / sig2;
    mp.slack = grid_slack(*g);
    const bool two = ctx->tuning.pair_kernel == 0 || ctx->tuning.pair_kernel >= 8;  // two targets per lane
    const int per_block = two ? 2 * kMixThreads : kMixThreads;
    const int blocks = (n + per_block - 1) / per_block;
    const size_t need = 256 + (size_t)blocks * sizeof(Partial);
    if (need > ctx->red_bytes) {
        lj_status s = grow(&ctx->red, &ctx->red_bytes, need);
        if (s != LJ_OK) return s;
        if (cudaMemsetAsync(ctx->red, 0, 256, ctx->stream) != cudaSuccess) return LJ_ECUDA;
    }
    unsigned* counter = static_cast<unsigned*>(ctx->red);
    Partial* part = reinterpret_cast<Partial*>(static_cast<char*>(ctx->red) + 256);
    // row passes with two targets per lane by default (and with the tuning's two-target kernels 8-10);
    // pair_kernel 1 (windows in shared memory) or 2 (windows in registers) asks for a flat walk, the
    // others for row passes with one target per lane
    if (two)
        k_pair_mixed_pass2<<<blocks, kMixThreads, 0, ctx->stream>>>(to_dev(*g), mp,
                                                                    reinterpret_cast<const float2*>(rec), sorted_cell,
                                                                    offsets, n, energy, force, part, counter, totals,
                                                                    ctx->d_status);
    else if (ctx->tuning.pair_kernel != 1 && ctx->tuning.pair_kernel != 2)
        k_pair_mixed_pass<<<blocks, kMixThreads, 0, ctx->stream>>>(to_dev(*g), mp,
                                                                   reinterpret_cast<const float2*>(rec), sorted_cell,
                                                                   offsets, n, energy, force, part, counter, totals,
                                                                   ctx->d_status);
    else if (ctx->tuning.pair_kernel == 2)
        k_pair_mixed_reg<<<blocks, kMixThreads, 0, ctx->stream>>>(to_dev(*g), mp, reinterpret_cast<const float2*>(rec),
                                                                  sorted_cell, offsets, n, energy, force, part,
                                                                  counter, totals, ctx->d_status);
    else
        k_pair_mixed<<<blocks, kMixThreads, 0, ctx->stream>>>(to_dev(*g), mp, reinterpret_cast<const float2*>(rec),
                                                              sorted_cell, offsets, n, energy, force, part, counter,
                                                              totals, ctx->d_status);
    return last_launch_status();
}
