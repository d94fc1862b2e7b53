// pair_common.cuh -- pieces shared by the pair kernels (pair.cu, pair_pass.cu, pair_half.cu, batch.cu).
#pragma once

#include <cfloat>

#include "ljcell_internal.cuh"

namespace ljc {

struct Partial {
    double e;
    double w;
    unsigned long long p;
    unsigned long long pad;
};

struct PairParams {
    float rc2;     // cutoff^2 (float), the distance test threshold
    float rc2w;    // rc2 * (1 + 1e-5): window / row-skip bound, above any rounding of the test
    float sig2;    // sigma^2
    float e4;      // 4 eps
    float e24;     // 24 eps
    float fscale;  // -24 eps / sigma^2: converts the accumulated sum of t * s2 * d into a force
    float slack;   // absolute rounding slack for cell planes and window ends
    int by_index = 0;  // 1: target k's outputs go to its original index (its record's fourth word), not k
};

// Output slot of sorted target k: k, or with pp.by_index the original index stored in its record
// (-1, and the range flag, if that index is outside [0, n)).
__device__ __forceinline__ int out_slot(const PairParams& pp, const float4* __restrict__ p, int k, int n,
                                        unsigned* status) {
    if (!pp.by_index) return k;
    const int o = __float_as_int(__ldg(&p[k].w));
    if (o < 0 || o >= n) {
        atomicOr(status, kFlagRange);
        return -1;
    }
    return o;
}

__device__ __forceinline__ void decode_cell(const GridDev& g, int c, int& cx, int& cy, int& cz) {
    const int gxy = g.gx * g.gy;
    cz = c / gxy;
    const int r = c - cz * gxy;
    cy = r / g.gx;
    cx = r - cy * g.gx;
}

// first j in [lo, hi) with p[j].x >= v (x-sorted range)
__device__ __forceinline__ int lower_x(const float4* __restrict__ p, int lo, int hi, float v) {
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (__ldg(&p[mid].x) < v)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}
// first j in [lo, hi) with p[j].x > v
__device__ __forceinline__ int upper_x(const float4* __restrict__ p, int lo, int hi, float v) {
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (__ldg(&p[mid].x) <= v)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

constexpr int kPairThreads = 128;
constexpr int kMaxWin = 10;

// Block reduction of the totals followed by a last-block final pass.
template <int BLOCK>
__device__ void reduce_totals(double e, double w, unsigned long long np, Partial* part, unsigned* counter,
                              lj_totals* totals) {
    __shared__ double s_e[BLOCK / 32], s_w[BLOCK / 32];
    __shared__ unsigned long long s_p[BLOCK / 32];
    __shared__ bool s_last;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    e = warp_sum(e);
    w = warp_sum(w);
    np = warp_sum(np);
    if (lane == 0) {
        s_e[warp] = e;
        s_w[warp] = w;
        s_p[warp] = np;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double te = 0, tw = 0;
        unsigned long long tp = 0;
        for (int i = 0; i < BLOCK / 32; ++i) {
            te += s_e[i];
            tw += s_w[i];
            tp += s_p[i];
        }
        part[blockIdx.x] = Partial{te, tw, tp, 0ULL};
        __threadfence();
        const unsigned done = atomicAdd(counter, 1u);
        s_last = (done == gridDim.x - 1);
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    // The last block reads every block's partial: eight independent L2 loads in flight per thread,
    // each thread's share in a fixed order, so the totals are the same on every run.
    double te = 0, tw = 0;
    unsigned long long tp = 0;
    const unsigned nb = gridDim.x;
    for (unsigned b0 = 0; b0 < nb; b0 += 8 * blockDim.x) {
        Partial q[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const unsigned b = b0 + u * blockDim.x + threadIdx.x;
            q[u] = Partial{0.0, 0.0, 0ULL, 0ULL};
            if (b < nb) {
                const double2 ew = __ldcg(reinterpret_cast<const double2*>(part + b));
                q[u].e = ew.x;
                q[u].w = ew.y;
                q[u].p = __ldcg(&part[b].p);
            }
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            te += q[u].e;
            tw += q[u].w;
            tp += q[u].p;
        }
    }
    te = warp_sum(te);
    tw = warp_sum(tw);
    tp = warp_sum(tp);
    __syncthreads();
    if (lane == 0) {
        s_e[warp] = te;
        s_w[warp] = tw;
        s_p[warp] = tp;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double fe = 0, fw = 0;
        unsigned long long fp = 0;
        for (int i = 0; i < BLOCK / 32; ++i) {
            fe += s_e[i];
            fw += s_w[i];
            fp += s_p[i];
        }
        if (totals) {
            totals->energy = fe;
            totals->virial = fw;
            totals->pairs = fp;
            totals->pad = 0ULL;
        }
        *counter = 0u;  // ready for the next launch
    }
}


// Per-target work of the truncated law: windows and walk.  `c` is the
// target's cell in grid g, `off` the offsets of that grid (values are indices
// into p), `n` bounds every index.  Shared by the single-system kernel and
// the batched kernel so both produce the same per-target results.
template <bool XWIN, int BLOCK>
__device__ __forceinline__ void pair_target(const GridDev& g, const PairParams& pp, const float4* __restrict__ p,
                                            const int* __restrict__ off, int n, int k, int c,
                                            int2 (*s_win)[BLOCK], float& ea, float& fx, float& fy, float& fz,
                                            float& wa, unsigned& np) {
    const int tid = threadIdx.x;
    const float4 pi = p[k];
    int cx, cy, cz;
    decode_cell(g, c, cx, cy, cz);
    const int xl = max(cx - 1, 0), xh = min(cx + 1, g.gx - 1);
    const float slack = pp.slack + 8.0f * FLT_EPSILON * fmaxf(fabsf(pi.x), fmaxf(fabsf(pi.y), fabsf(pi.z)));
    int nw = 0;
#pragma unroll
    for (int dz = -1; dz <= 1; ++dz) {
        const int z = cz + dz;
        if (z < 0 || z >= g.gz) continue;
        float dzm = 0.f;
        if (XWIN) {
            if (dz < 0) dzm = pi.z - fmaf((float)cz, g.w, g.oz);
            if (dz > 0) dzm = fmaf((float)(cz + 1), g.w, g.oz) - pi.z;
            dzm = fmaxf(dzm - slack, 0.f);
        }
#pragma unroll
        for (int dy = -1; dy <= 1; ++dy) {
            const int y = cy + dy;
            if (y < 0 || y >= g.gy) continue;
            const int rb = (z * g.gy + y) * g.gx;
            int s = min(max(__ldg(&off[rb + xl]), 0), n);
            int e = min(max(__ldg(&off[rb + xh + 1]), s), n);
            if (XWIN) {
                float dym = 0.f;
                if (dy < 0) dym = pi.y - fmaf((float)cy, g.w, g.oy);
                if (dy > 0) dym = fmaf((float)(cy + 1), g.w, g.oy) - pi.y;
                dym = fmaxf(dym - slack, 0.f);
                const float d2 = fmaf(dym, dym, dzm * dzm);
                if (d2 >= pp.rc2w) continue;
                const float h = sqrtf(pp.rc2w - d2) + slack;
                s = lower_x(p, s, e, pi.x - h);
                e = upper_x(p, s, e, pi.x + h);
            }
            if (dz == 0 && dy == 0) {
                s_win[nw++][tid] = make_int2(s, k);
                s_win[nw++][tid] = make_int2(k + 1, e);
            } else {
                s_win[nw++][tid] = make_int2(s, e);
            }
        }
    }
    int w = 0;
    int2 cur = s_win[0][tid];
    const float rc2 = pp.rc2;
    const float2 sig2 = make_float2(pp.sig2, pp.sig2), two2 = make_float2(2.0f, 2.0f);
    const float2 npx = make_float2(-pi.x, -pi.x), npy = make_float2(-pi.y, -pi.y), npz = make_float2(-pi.z, -pi.z);
    float2 S12 = make_float2(0.f, 0.f), S6 = S12, FX = S12, FY = S12, FZ = S12;
    // two candidates per iteration, evaluated together in the paired FP32 instructions without a
    // branch (a miss contributes exact zeros)
    while (true) {
        bool done = false;
        while (cur.x >= cur.y) {
            if (++w >= nw) {
                done = true;
                break;
            }
            cur = s_win[w][tid];
        }
        if (done) break;
        const int j0 = cur.x;
        const bool two = j0 + 1 < cur.y;
        const int j1 = two ? j0 + 1 : j0;
        cur.x = j1 + 1;
        const float4 q0 = __ldg(&p[j0]);
        const float4 q1 = __ldg(&p[j1]);
        const float2 dx = __fadd2_rn(make_float2(q0.x, q1.x), npx);
        const float2 dy = __fadd2_rn(make_float2(q0.y, q1.y), npy);
        const float2 dz = __fadd2_rn(make_float2(q0.z, q1.z), npz);
        const float2 r2 = __ffma2_rn(dz, dz, __ffma2_rn(dy, dy, __fmul2_rn(dx, dx)));
        const bool in0 = r2.x < rc2, in1 = two && r2.y < rc2;
        const float2 ir2 = make_float2(rcp_hit(in0, r2.x), rcp_hit(in1, r2.y));
        const float2 s2 = __fmul2_rn(sig2, ir2);
        const float2 s4 = __fmul2_rn(s2, s2);
        const float2 s6 = __fmul2_rn(s4, s2);
        const float2 s12 = __fmul2_rn(s6, s6);
        S12 = __fadd2_rn(S12, s12);
        S6 = __fadd2_rn(S6, s6);
        const float2 t = __ffma2_rn(two2, s12, make_float2(-s6.x, -s6.y));
        const float2 fs = __fmul2_rn(t, s2);
        FX = __ffma2_rn(fs, dx, FX);
        FY = __ffma2_rn(fs, dy, FY);
        FZ = __ffma2_rn(fs, dz, FZ);
        np += (unsigned)in0 + (unsigned)in1;
    }
    const float s12t = S12.x + S12.y, s6t = S6.x + S6.y;
    ea += s12t - s6t;
    wa += fmaf(2.0f, s12t, -s6t);
    fx += FX.x + FX.y;
    fy += FY.x + FY.y;
    fz += FZ.x + FZ.y;
}

float grid_slack(const lj_grid& g);
// Row-pass walks (pair_pass.cu): one target per lane (kernel 6) or two (kernel 10).
lj_status launch_pair_pass(lj_ctx* ctx, const lj_grid* g, const PairParams& pp, int n, const float* xyzi,
                           const int* cs, const int* off, bool two, float* energy, float* force, lj_totals* totals,
                           int kb, int ke);
// Kernel 12 (pair_pass.cu): targets paired inside their cell, whole rows.
lj_status launch_pair_cellpair(lj_ctx* ctx, const lj_grid* g, const PairParams& pp, int n, const float* xyzi,
                               const int* cs, const int* off, float* energy, float* force, lj_totals* totals,
                               int kb, int ke);
// Exclusive scan of counts[ncells] into offsets[0..ncells] on the context's stream (bin.cu).
lj_status launch_scan(lj_ctx* ctx, const int* counts, long long ncells, int* offsets);
}  // namespace ljc
