// pair_half.cu -- half-shell (Newton's third law) evaluation of the truncated law: lj_compute_half.
//
// The reference evaluates every ordered pair twice, once from each side (the full 27-cell stencil
// of ComputeParticleInterationsParPartNoLoop, cudaLJ.cu:319-337).  Here each unordered pair {i, j}
// is evaluated once, by the cell of i when the cell of j lies in its forward half-stencil (the 13
// neighbours with dz = +1, or dz = 0 and dy = +1, or dz = dy = 0 and dx = +1) or, inside one cell,
// when j > i; the reaction -F_ij, e_ij and the virial term go to j.
//
// Determinism without float atomics:
//  * Phases.  Cells are coloured with period 3 in x and y and 2 in z (18 colours).  A cell writes
//    its own particles and those of its forward half-stencil, a block spanning x in [cx-1, cx+1],
//    y in [cy-1, cy+1] and z in [cz, cz+1], so two cells of one colour never write the same particle.
//    The phases run one after another (one launch each); within a phase every write is a plain
//    read-modify-write with no other writer.
//  * Within a cell (one warp): the cell's targets (up to 32 per round) walk each candidate range in
//    a rotated order, lane l taking candidate (t + l) mod U at step t, so no two lanes touch one
//    candidate in a step; the reactions collect in shared memory (one slot per candidate of the
//    range, __syncwarp between steps) and are added to the particles' accumulators after the range,
//    in slot order.  Every particle's sums therefore come out in one fixed order on every run.
//  * Pair count: the unordered interacting pairs, counted in integers (associative), times 2.
//
// The candidate ranges are whole rows of cells (no x-window: the targets of a cell span it in x, so
// their union window is the row's 3 cells anyway).  Outputs and totals match lj_compute's meaning:
// per-particle energy and force, E = 1/2 sum of the per-particle energies, the virial and the
// ordered pair count, all reduced from the float per-particle sums in FP64 in a fixed order.
#include <algorithm>

#include "pair_common.cuh"

namespace ljc {

namespace {
constexpr int kHalfWarps = 4;     // warps (cells) per block
constexpr int kHalfSeg = 256;     // candidates per shared-memory reaction segment
}  // namespace

// Raw accumulators per particle (law units): e = sum (s^12 - s^6), w = sum (2 s^12 - s^6),
// f = minus sum (2 s^12 - s^6) s^2 (p_j - p_i).
struct HalfRaw {
    float* e;
    float* w;
    float* f;  // 3 per particle
};

__device__ __forceinline__ void half_law(const float4& pi, const float4& q, float rc2, float sig2, bool m,
                                         float& e, float& w, float& fx, float& fy, float& fz, bool& hit) {
    const float dx = q.x - pi.x, dy = q.y - pi.y, dz = q.z - pi.z;
    const float r2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
    hit = m && r2 < rc2;
    const float ir2 = rcp_hit(hit, r2);
    const float s2 = sig2 * ir2;
    const float s6 = s2 * s2 * s2;
    const float s12 = s6 * s6;
    e = s12 - s6;
    w = fmaf(2.0f, s12, -s6);
    const float fs = w * s2;  // force along d in units of 24 eps / sigma^2: minus fs * d for i, plus for j
    fx = fs * dx;
    fy = fs * dy;
    fz = fs * dz;
}

// One candidate range [a, b) for the lane's target i (active: the lane has a target in this
// round; own: only j > i).  U: the segment's length; slots in shared memory.
__device__ __forceinline__ void half_range(const float4* __restrict__ p, int a, int b, int i, bool active, bool own,
                                           int lane0, int rounds_lanes, const float4& pi, float rc2, float sig2,
                                           float* se, float* sw, float* sf, HalfRaw raw, float& ei, float& wi,
                                           float& fxi, float& fyi, float& fzi, unsigned long long& np) {
    const int l = (int)(threadIdx.x & 31u);
    for (int seg = a; seg < b; seg += kHalfSeg) {
        const int U = min(kHalfSeg, b - seg);
        for (int u = l; u < U; u += 32) {
            se[u] = 0.f;
            sw[u] = 0.f;
            sf[3 * u] = sf[3 * u + 1] = sf[3 * u + 2] = 0.f;
        }
        __syncwarp();
        // lanes in rounds of at most U, so the rotation gives distinct slots within a step
        const int G = min(32, U);
        for (int r0 = 0; r0 < rounds_lanes; r0 += G) {
            const bool mine = active && l >= r0 && l < r0 + G;
            const int rot = l - r0;
            for (int t = 0; t < U; ++t) {
                int idx = t + rot;
                idx = idx >= U ? idx - U : idx;
                const int j = seg + idx;
                const bool m = mine && (!own || j > i);
                const float4 q = __ldg(&p[m ? j : lane0]);
                float e, w, fx, fy, fz;
                bool hit;
                half_law(pi, q, rc2, sig2, m, e, w, fx, fy, fz, hit);
                if (hit) {
                    ei += e;
                    wi += w;
                    fxi -= fx;
                    fyi -= fy;
                    fzi -= fz;
                    se[idx] += e;
                    sw[idx] += w;
                    sf[3 * idx] += fx;
                    sf[3 * idx + 1] += fy;
                    sf[3 * idx + 2] += fz;
                    ++np;
                }
                __syncwarp();
            }
        }
        // the segment's reactions to the candidates' accumulators, in slot order
        for (int u = l; u < U; u += 32) {
            const int j = seg + u;
            raw.e[j] += se[u];
            raw.w[j] += sw[u];
            raw.f[3 * (size_t)j + 0] += sf[3 * u];
            raw.f[3 * (size_t)j + 1] += sf[3 * u + 1];
            raw.f[3 * (size_t)j + 2] += sf[3 * u + 2];
        }
        __syncwarp();
    }
}

// One colour (ox, oy, oz): warp w of the launch takes the w-th cell of the colour.
__global__ void __launch_bounds__(32 * kHalfWarps) k_pair_half(GridDev g, PairParams pp, const float4* __restrict__ p,
                                                               const int* __restrict__ off, int n, int ox, int oy,
                                                               int oz, HalfRaw raw, unsigned long long* pairs) {
    __shared__ float s_e[kHalfWarps][kHalfSeg], s_w[kHalfWarps][kHalfSeg], s_f[kHalfWarps][3 * kHalfSeg];
    const int wib = (int)(threadIdx.x >> 5), l = (int)(threadIdx.x & 31u);
    const long long cw = (long long)blockIdx.x * kHalfWarps + wib;
    const int ncx = (g.gx - ox + 2) / 3, ncy = (g.gy - oy + 2) / 3, ncz = (g.gz - oz + 1) / 2;
    if (cw >= (long long)ncx * ncy * ncz) return;  // warp-uniform
    const int ix = (int)(cw % ncx), iy = (int)((cw / ncx) % ncy), iz = (int)(cw / ((long long)ncx * ncy));
    const int cx = ox + 3 * ix, cy = oy + 3 * iy, cz = oz + 2 * iz;
    const int c = (cz * g.gy + cy) * g.gx + cx;
    const int s = min(max(__ldg(&off[c]), 0), n), e = min(max(__ldg(&off[c + 1]), s), n);
    if (s == e) return;  // warp-uniform
    // forward ranges: the own row from this cell through cell cx + 1 (j > i), the row (cy + 1, cz),
    // and the rows (cy - 1 .. cy + 1, cz + 1), each over cells cx - 1 .. cx + 1
    int ra[5], rb[5];
    const int own_end = cx + 1 < g.gx ? min(max(__ldg(&off[c + 2]), e), n) : e;
    ra[0] = s;
    rb[0] = own_end;
#pragma unroll
    for (int k = 1; k < 5; ++k) {
        const int dy = k == 1 ? 1 : k - 3, dz = k == 1 ? 0 : 1;  // (1, 0), (-1, 1), (0, 1), (1, 1)
        const int y = cy + dy, z = cz + dz;
        ra[k] = rb[k] = 0;
        if (y < 0 || y >= g.gy || z >= g.gz) continue;
        const int rbase = (z * g.gy + y) * g.gx;
        ra[k] = min(max(__ldg(&off[rbase + max(cx - 1, 0)]), 0), n);
        rb[k] = min(max(__ldg(&off[rbase + min(cx + 1, g.gx - 1) + 1]), ra[k]), n);
    }
    const float rc2 = pp.rc2, sig2 = pp.sig2;
    unsigned long long np = 0;
    for (int base = s; base < e; base += 32) {
        const int i = base + l;
        const bool active = i < e;
        const int na = min(32, e - base);
        const float4 pi = __ldg(&p[active ? i : s]);
        float ei = 0.f, wi = 0.f, fxi = 0.f, fyi = 0.f, fzi = 0.f;
#pragma unroll 1
        for (int k = 0; k < 5; ++k)
            half_range(p, ra[k], rb[k], i, active, k == 0, s, na, pi, rc2, sig2, s_e[wib], s_w[wib], s_f[wib], raw,
                       ei, wi, fxi, fyi, fzi, np);
        if (active) {  // the target's own forward sums (its cell is written by this warp only)
            raw.e[i] += ei;
            raw.w[i] += wi;
            raw.f[3 * (size_t)i + 0] += fxi;
            raw.f[3 * (size_t)i + 1] += fyi;
            raw.f[3 * (size_t)i + 2] += fzi;
        }
        __syncwarp();
    }
    np = warp_sum(np);
    if (l == 0 && np) atomicAdd(pairs, np);  // integer: the sum does not depend on the order
}

// Outputs and totals from the raw sums: per-particle energy and force, then FP64 totals by block
// partials and a last-block pass in a fixed order (as the full-shell kernels).
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_half_finish(PairParams pp, HalfRaw raw, int n,
                                                       const unsigned long long* pairs, float* __restrict__ energy,
                                                       float* __restrict__ force, Partial* part, unsigned* counter,
                                                       lj_totals* totals) {
    const int k = blockIdx.x * BLOCK + threadIdx.x;
    double e = 0.0, w = 0.0;
    if (k < n) {
        const float ek = pp.e4 * raw.e[k];
        if (energy) energy[k] = ek;
        if (force) {  // F = 24 eps / sigma^2 * raw.f = -fscale * raw.f
            const float nf = -pp.fscale;
            force[3 * (size_t)k + 0] = nf * raw.f[3 * (size_t)k + 0];
            force[3 * (size_t)k + 1] = nf * raw.f[3 * (size_t)k + 1];
            force[3 * (size_t)k + 2] = nf * raw.f[3 * (size_t)k + 2];
        }
        e = 0.5 * (double)ek;
        w = 0.5 * (double)pp.e24 * (double)raw.w[k];
    }
    // pairs: the block holding particle 0 contributes the whole count (ordered = 2 x unordered)
    const unsigned long long np = (k == 0) ? 2ULL * *pairs : 0ULL;
    reduce_totals<BLOCK>(e, w, np, part, counter, totals);
}

}  // namespace ljc

using namespace ljc;

extern "C" lj_status lj_compute_half(lj_ctx* ctx, const lj_grid* g, const lj_params* prm, int n,
                                     const float* sorted_xyzi, const int* offsets, float* energy, float* force,
                                     lj_totals* totals) {
    const NvtxRange nvtx_range("lj_compute_half");
    if (!ctx || !g || !prm || n < 0 || (n > 0 && (!sorted_xyzi || !offsets))) return LJ_EINVAL;
    if (!(g->width > 0.0f) || g->dim[0] < 1 || g->dim[1] < 1 || g->dim[2] < 1) return LJ_EINVAL;
    if (!(prm->cutoff > 0.0f) || !(prm->cutoff <= g->width) || !(prm->sigma > 0.0f)) return LJ_EINVAL;
    if (reinterpret_cast<uintptr_t>(sorted_xyzi) & 15) return LJ_EINVAL;
    const long long nc = (long long)g->dim[0] * g->dim[1] * g->dim[2];
    if (nc > 2147483646LL) return LJ_EINVAL;
    if (n == 0) {
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
    // scratch: raw sums (5 floats per particle) and the pair counter, in the context's step buffer
    const size_t b_e = ((size_t)n * sizeof(float) + 255) & ~(size_t)255;
    const size_t b_f = (3 * (size_t)n * sizeof(float) + 255) & ~(size_t)255;
    const size_t need = 2 * b_e + b_f + 256;
    lj_status s = grow(&ctx->half, &ctx->half_bytes, need);
    if (s != LJ_OK) return s;
    char* base = static_cast<char*>(ctx->half);
    HalfRaw raw{reinterpret_cast<float*>(base), reinterpret_cast<float*>(base + b_e),
                reinterpret_cast<float*>(base + 2 * b_e)};
    unsigned long long* pairs = reinterpret_cast<unsigned long long*>(base + 2 * b_e + b_f);
    if (cudaMemsetAsync(ctx->half, 0, need, ctx->stream) != cudaSuccess) return LJ_ECUDA;
    const GridDev gd = to_dev(*g);
    const float4* p4 = reinterpret_cast<const float4*>(sorted_xyzi);
    for (int oz = 0; oz < 2; ++oz)
        for (int oy = 0; oy < 3; ++oy)
            for (int ox = 0; ox < 3; ++ox) {
                const long long cells = (long long)((gd.gx - ox + 2) / 3) * ((gd.gy - oy + 2) / 3) *
                                        ((gd.gz - oz + 1) / 2);
                if (cells <= 0) continue;
                const long long blocks = (cells + kHalfWarps - 1) / kHalfWarps;
                k_pair_half<<<(unsigned)blocks, 32 * kHalfWarps, 0, ctx->stream>>>(gd, pp, p4, offsets, n, ox, oy, oz,
                                                                                   raw, pairs);
                if ((s = last_launch_status()) != LJ_OK) return s;
            }
    constexpr int kFin = 256;
    const int blocks = (n + kFin - 1) / kFin;
    const size_t rneed = 256 + (size_t)blocks * sizeof(Partial);
    if (rneed > ctx->red_bytes) {
        if ((s = grow(&ctx->red, &ctx->red_bytes, rneed)) != LJ_OK) return s;
        if (cudaMemsetAsync(ctx->red, 0, 256, ctx->stream) != cudaSuccess) return LJ_ECUDA;
    }
    unsigned* counter = static_cast<unsigned*>(ctx->red);
    Partial* part = reinterpret_cast<Partial*>(static_cast<char*>(ctx->red) + 256);
    k_half_finish<kFin><<<blocks, kFin, 0, ctx->stream>>>(pp, raw, n, pairs, energy, force, part, counter, totals);
    return last_launch_status();
}
