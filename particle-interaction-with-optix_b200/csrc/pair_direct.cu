// pair_direct.cu -- the truncated-LJ pair kernel, one thread per target,
// neighbours read through L1 (no shared-memory staging).
//
// Per target: the 9 stencil rows are skipped or cut to an x-window exactly as
// in pair.cu (particles binned with LJ_ORDER_X).  The windows stay in
// registers: slot r holds row r, slot 9 the part of the own row after the
// target, and the walk shifts the slots down (static register indices, no
// local memory), so shared memory is free for the L1 cache.
//
// COMPACT = true splits the walk in two phases.  Phase A streams candidates
// through the distance test only and appends each interacting neighbour's
// (dx, dy, dz, r2) to a per-lane queue in shared memory; when any lane's queue
// is full (and at the end) the warp drains all queues, evaluating the pair
// law only for real partners.  With about one candidate in three passing, the
// pair law is no longer evaluated (predicated) on every step of the warp.
#include "pair_common.cuh"

namespace ljc {

constexpr int kDirThreads = 128;
constexpr int kQueue = 12;  // per-lane queue of interacting neighbours (COMPACT)
constexpr int kBurst = 4;   // candidates a lane tests between two warp votes

struct DirAcc {
    float e, fx, fy, fz, w;
    unsigned np;
};

__device__ __forceinline__ void law(float dx, float dy, float dz, float r2, float sig2, DirAcc& a) {
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

// Evaluates the law for every queued neighbour of every lane of the warp.
__device__ __forceinline__ void drain_queue(float4 (*s_q)[kDirThreads], int qn, float sig2, DirAcc& a) {
    int qmax = qn;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) qmax = max(qmax, __shfl_xor_sync(0xffffffffu, qmax, o));
    for (int i = 0; i < qmax; ++i) {
        if (i < qn) {
            const float4 d = s_q[i][threadIdx.x];
            law(d.x, d.y, d.z, d.w, sig2, a);
        }
    }
}

template <bool COMPACT>
__global__ void __launch_bounds__(kDirThreads) k_pair_direct(GridDev g, PairParams pp, const float4* __restrict__ p,
                                                             const int* __restrict__ cs,
                                                             const int* __restrict__ off, int n, int kb, int ke,
                                                             float* __restrict__ energy, float* __restrict__ force,
                                                             Partial* part, unsigned* counter, lj_totals* totals,
                                                             unsigned* status) {
    __shared__ float4 s_q[COMPACT ? kQueue : 1][kDirThreads];
    const int tid = threadIdx.x;
    const int k = kb + blockIdx.x * kDirThreads + tid;   // targets [kb, ke) of the n sorted particles
    const bool active = k < ke;
    DirAcc a{0.f, 0.f, 0.f, 0.f, 0.f, 0u};
    int2 slot[10];
#pragma unroll
    for (int i = 0; i < 10; ++i) slot[i] = make_int2(0, 0);
    float4 pi = make_float4(0.f, 0.f, 0.f, 0.f);
    if (active) {
        pi = __ldg(&p[k]);
        int c = __ldg(&cs[k]);
        const int ncell = g.gx * g.gy * g.gz;
        if (c < 0 || c >= ncell) {
            atomicOr(status, kFlagRange);
            c = 0;
        }
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
            const int s = min(max(__ldg(&off[rb + xl]), 0), n);
            const int e = min(max(__ldg(&off[rb + xh + 1]), s), n);
            const float h = sqrtf(pp.rc2w - d2) + slack;
            const int lo = lower_x(p, s, e, pi.x - h);
            const int hi = upper_x(p, lo, e, pi.x + h);
            if (r == 4) {
                slot[4] = make_int2(lo, k);
                slot[9] = make_int2(k + 1, hi);
            } else {
                slot[r] = make_int2(lo, hi);
            }
        }
    }
    const float rc2 = pp.rc2, sig2 = pp.sig2;
    int2 cur = slot[0];
    int rem = 10;  // windows left, including cur
    bool more = active;
// Moves `cur` to the next non-empty window (shifting the slots); clears `more` at the end.
#define LJ_ADVANCE()                                                \
    do {                                                            \
        if (--rem == 0) {                                           \
            more = false;                                           \
            break;                                                  \
        }                                                           \
        cur = slot[1];                                              \
        _Pragma("unroll") for (int i_ = 1; i_ < 9; ++i_) slot[i_] = slot[i_ + 1]; \
        slot[9] = make_int2(0, 0);                                  \
    } while (cur.x >= cur.y)
    if constexpr (!COMPACT) {
        while (more) {
            if (cur.x >= cur.y) {
                LJ_ADVANCE();
                if (!more) break;
            }
            const float4 q = __ldg(&p[cur.x]);
            ++cur.x;
            const float dx = q.x - pi.x, dy = q.y - pi.y, dz = q.z - pi.z;
            const float r2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
            if (r2 < rc2) law(dx, dy, dz, r2, sig2, a);
        }
    } else {
        // Lockstep bursts: every lane votes at the top; before a burst each queue
        // holds at most kQueue - kBurst entries, so a burst cannot overflow it.
        int qn = 0;
        while (__any_sync(0xffffffffu, more)) {
            if (more) {
#pragma unroll
                for (int b = 0; b < kBurst; ++b) {
                    if (cur.x >= cur.y) {
                        LJ_ADVANCE();
                        if (!more) break;
                    }
                    const float4 q = __ldg(&p[cur.x]);
                    ++cur.x;
                    const float dx = q.x - pi.x, dy = q.y - pi.y, dz = q.z - pi.z;
                    const float r2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
                    if (r2 < rc2) s_q[qn++][tid] = make_float4(dx, dy, dz, r2);
                }
            }
            if (__any_sync(0xffffffffu, qn > kQueue - kBurst)) {
                drain_queue(s_q, qn, sig2, a);
                qn = 0;
            }
        }
        drain_queue(s_q, qn, sig2, a);
    }
#undef LJ_ADVANCE
    if (active) {
        if (energy) energy[k] = pp.e4 * a.e;
        if (force) {
            force[3 * (size_t)k + 0] = pp.fscale * a.fx;
            force[3 * (size_t)k + 1] = pp.fscale * a.fy;
            force[3 * (size_t)k + 2] = pp.fscale * a.fz;
        }
    }
    reduce_totals<kDirThreads>(0.5 * (double)pp.e4 * (double)a.e, 0.5 * (double)pp.e24 * (double)a.w,
                               (unsigned long long)a.np, part, counter, totals);
}

lj_status launch_pair_direct(lj_ctx* ctx, const lj_grid* g, const PairParams& pp, int n, const float* xyzi,
                             const int* cs, const int* off, bool compact, float* energy, float* force,
                             lj_totals* totals, int kb, int ke) {
    const int blocks = (ke - kb + kDirThreads - 1) / kDirThreads;
    const size_t need = 256 + (size_t)blocks * sizeof(Partial);
    if (need > ctx->red_bytes) {
        lj_status s = grow(&ctx->red, &ctx->red_bytes, need);
        if (s != LJ_OK) return s;
        if (cudaMemsetAsync(ctx->red, 0, 256, ctx->stream) != cudaSuccess) return LJ_ECUDA;
    }
    unsigned* counter = static_cast<unsigned*>(ctx->red);
    Partial* part = reinterpret_cast<Partial*>(static_cast<char*>(ctx->red) + 256);
    const float4* p4 = reinterpret_cast<const float4*>(xyzi);
    if (compact)
        k_pair_direct<true><<<blocks, kDirThreads, 0, ctx->stream>>>(to_dev(*g), pp, p4, cs, off, n, kb, ke, energy,
                                                                     force, part, counter, totals, ctx->d_status);
    else
        k_pair_direct<false><<<blocks, kDirThreads, 0, ctx->stream>>>(to_dev(*g), pp, p4, cs, off, n, kb, ke, energy,
                                                                      force, part, counter, totals, ctx->d_status);
    return last_launch_status();
}

}  // namespace ljc
