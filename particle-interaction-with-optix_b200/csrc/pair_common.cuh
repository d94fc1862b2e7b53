// pair_common.cuh -- pieces shared by the pair kernels (pair.cu, pair_tiled.cu).
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
};

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
    double te = 0, tw = 0;
    unsigned long long tp = 0;
    for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x) {
        const volatile Partial* q = part + b;
        te += q->e;
        tw += q->w;
        tp += q->p;
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


float grid_slack(const lj_grid& g);
lj_status launch_pair_direct(lj_ctx* ctx, const lj_grid* g, const PairParams& pp, int n, const float* xyzi,
                             const int* cs, const int* off, bool compact, float* energy, float* force,
                             lj_totals* totals);
lj_status launch_pair_tiled(lj_ctx* ctx, const lj_grid* g, const PairParams& pp, int n, const float* xyzi,
                            const int* off, float* energy, float* force, lj_totals* totals);

}  // namespace ljc
