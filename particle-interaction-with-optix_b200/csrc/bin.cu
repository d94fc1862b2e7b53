// bin.cu -- the cell-grid build on the device.
//
// Replaces the binning sequence of executeSimulation (cudaLJ.cu:614-634):
//   ComputeNbParticlePerCells (cudaLJ.cu:345-383)  -> k_count   (warp-aggregated
//        per-cell counting; the same atomic hands out each particle's ticket)
//   PrefixFullV2 (prefixsum.hpp:160-215)           -> k_scan    (single-pass
//        decoupled look-back exclusive scan; no recursion, no allocation, no
//        host synchronisation)
//   InitNewCells (cudaLJ.cu:428-439)               -> k_descriptors
//   MoveParticlesToNewCells (cudaLJ.cu:441-471)    -> k_scatter + k_cell_rank (+ k_large_sort)
//        (ticket scatter, then a per-cell sort that makes the order a pure
//        function of the input, repacking positions as float4 x, y, z, index)
// and ComputeNbInteractions (cudaLJ.cu:255-297) -> k_candidates (per cell
// instead of per particle).
#include <algorithm>
#include <climits>

#include "ljcell_internal.cuh"

namespace ljc {

// ---------------------------------------------------------------- counting
// One thread per particle, grid-stride by whole warps.  Lanes that share a
// cell elect a leader (__match_any_sync) which adds the group's size with one
// atomic; each lane's ticket is the leader's old value plus its rank in the
// group.  Tickets give a slot inside the cell; their order is not
// deterministic, which k_cell_rank fixes.
template <bool TICKETS>
__global__ void __launch_bounds__(256) k_count(GridDev g, const float* __restrict__ x, const float* __restrict__ y,
                                               const float* __restrict__ z, int stride, int n,
                                               int* __restrict__ counts, int2* __restrict__ ct,
                                               unsigned* status) {
    const int lane = threadIdx.x & 31;
    const long long gwarp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long base = gwarp * 32; base < n; base += nwarps * 32) {
        const long long i = base + lane;
        const bool valid = i < n;
        int cell = -1 - lane;  // distinct key for inactive lanes
        if (valid) {
            const float px = x[i * stride], py = y[i * stride], pz = z[i * stride];
            if (!(isfinite(px) && isfinite(py) && isfinite(pz))) atomicOr(status, kFlagNonFinite);
            cell = cell_of(g, px, py, pz);
        }
        const unsigned peers = __match_any_sync(0xffffffffu, cell);
        const int leader = __ffs(peers) - 1;
        int first = 0;
        if (valid && lane == leader) first = atomicAdd(&counts[cell], __popc(peers));
        first = __shfl_sync(0xffffffffu, first, leader);
        if (TICKETS && valid) ct[i] = make_int2(cell, first + __popc(peers & lanemask_lt()));
    }
}

// ---------------------------------------------------------------- scan
// Exclusive scan of int counts[n] into offsets[0..n] (offsets[n] = total).
// Tiles of 8192 items (256 threads x 32), tile index taken from an atomic
// counter so every predecessor tile is already running.  Each warp scans 1024
// items in a striped layout (coalesced int4 loads and stores); warp 0 then
// publishes the tile aggregate and looks back over predecessors, 32 tiles at a
// time, until it meets an inclusive prefix.  Tile state = 2-bit flag | 62-bit
// value in one 64-bit word, so flag and value become visible together.  The
// look-back wait is bounded: on timeout it records kFlagTimeout and goes on.
constexpr int kScanThreads = 256;
constexpr int kScanTile = 8192;
constexpr int kScanIters = kScanTile / (kScanThreads * 4);  // int4 loads per thread
constexpr unsigned long long kStAgg = 1ULL << 62;
constexpr unsigned long long kStPre = 2ULL << 62;
constexpr unsigned long long kStVal = (1ULL << 62) - 1ULL;
constexpr unsigned kSpinLimit = 1u << 20;  // polls: well under a second of waiting

__device__ __forceinline__ unsigned long long ld_state(const unsigned long long* p) {
    return *reinterpret_cast<const volatile unsigned long long*>(p);
}
__device__ __forceinline__ void st_state(unsigned long long* p, unsigned long long v) {
    *reinterpret_cast<volatile unsigned long long*>(p) = v;
}

__global__ void __launch_bounds__(kScanThreads) k_scan(const int* __restrict__ counts, int* __restrict__ offsets,
                                                       long long n, long long ntiles,
                                                       unsigned long long* tile_state, unsigned* tile_counter,
                                                       int vec_ok, unsigned* status) {
    __shared__ unsigned s_tile;
    __shared__ long long s_warp[8];
    __shared__ long long s_prefix;
    if (threadIdx.x == 0) s_tile = atomicAdd(tile_counter, 1u);
    __syncthreads();
    const long long tile = s_tile;
    if (tile >= ntiles) return;  // defensive: more CTAs than tiles
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long long tbase = tile * kScanTile;
    const long long wbase = tbase + warp * (kScanIters * 128);
    const bool full = vec_ok && (tbase + kScanTile <= n);
    int v[kScanIters][4];
    if (full) {
#pragma unroll
        for (int it = 0; it < kScanIters; ++it) {
            const int4 q = __ldg(reinterpret_cast<const int4*>(counts + wbase + it * 128 + lane * 4));
            v[it][0] = q.x;
            v[it][1] = q.y;
            v[it][2] = q.z;
            v[it][3] = q.w;
        }
    } else {
#pragma unroll
        for (int it = 0; it < kScanIters; ++it)
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const long long idx = wbase + it * 128 + lane * 4 + e;
                v[it][e] = idx < n ? counts[idx] : 0;
            }
    }
    // warp-local exclusive prefixes (sums stay below 2^31: they are particle counts)
    int carry = 0;
#pragma unroll
    for (int it = 0; it < kScanIters; ++it) {
        const int a0 = v[it][0], a1 = a0 + v[it][1], a2 = a1 + v[it][2], a3 = a2 + v[it][3];
        int inc = a3;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += t;
        }
        const int ex = carry + inc - a3;
        v[it][0] = ex;
        v[it][1] = ex + a0;
        v[it][2] = ex + a1;
        v[it][3] = ex + a2;
        carry += __shfl_sync(0xffffffffu, inc, 31);
    }
    if (lane == 0) s_warp[warp] = carry;
    __syncthreads();
    if (warp == 0) {
        const long long wt = lane < 8 ? s_warp[lane] : 0;
        long long inc = wt;
#pragma unroll
        for (int o = 1; o < 8; o <<= 1) {
            const long long t = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += t;
        }
        const long long agg = __shfl_sync(0xffffffffu, inc, 7);
        __syncwarp();
        if (lane < 8) s_warp[lane] = inc - wt;
        long long prefix = 0;
        if (tile == 0) {
            if (lane == 0) st_state(&tile_state[0], kStPre | (unsigned long long)agg);
        } else {
            if (lane == 0) st_state(&tile_state[tile], kStAgg | (unsigned long long)agg);
            long long pred = tile - 1;
            unsigned spins = 0;
            while (true) {
                const long long t = pred - lane;
                unsigned long long st = kStPre;  // before tile 0: an inclusive prefix of 0
                bool gave_up = false;
                if (t >= 0) {
                    st = ld_state(&tile_state[t]);
                    while ((st >> 62) == 0ULL) {
                        if (++spins > kSpinLimit) {
                            gave_up = true;
                            break;
                        }
                        __nanosleep(32);
                        st = ld_state(&tile_state[t]);
                    }
                }
                if (__any_sync(0xffffffffu, gave_up)) {
                    if (lane == 0) atomicOr(status, kFlagTimeout);
                    break;
                }
                const unsigned pre = __ballot_sync(0xffffffffu, (st >> 62) == 2ULL);
                if (pre) {
                    const int first = __ffs(pre) - 1;
                    const unsigned long long val = lane <= first ? (st & kStVal) : 0ULL;
                    prefix += (long long)warp_sum(val);
                    break;
                }
                prefix += (long long)warp_sum(st & kStVal);
                pred -= 32;
            }
            if (lane == 0) st_state(&tile_state[tile], kStPre | (unsigned long long)(prefix + agg));
        }
        if (lane == 0) {
            s_prefix = prefix;
            if (tile == ntiles - 1) offsets[n] = (int)(prefix + agg);
        }
    }
    __syncthreads();
    const int tp = (int)(s_prefix + s_warp[warp]);
    if (full) {
#pragma unroll
        for (int it = 0; it < kScanIters; ++it)
            *reinterpret_cast<int4*>(offsets + wbase + it * 128 + lane * 4) =
                make_int4(tp + v[it][0], tp + v[it][1], tp + v[it][2], tp + v[it][3]);
    } else {
#pragma unroll
        for (int it = 0; it < kScanIters; ++it)
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const long long idx = wbase + it * 128 + lane * 4 + e;
                if (idx < n) offsets[idx] = tp + v[it][e];
            }
    }
}

// ---------------------------------------------------------------- scatter
// Moves each particle to offsets[cell] + ticket as float4 (x, y, z, index
// bits).  The slot is range-checked so that a corrupted offsets array cannot
// write out of bounds.
// Four particles per thread per round, all loads issued before the stores: the kernel is bound by
// the latency of the offset gather and of the scattered 16-byte writes, not by bandwidth.
// Only particles of cells [c_lo, c_hi) move: bin_finish runs it in passes over cell ranges whose
// slots span a region that fits in L2, so the scattered 16-byte records of a cell meet there and
// leave L2 as whole lines instead of as partial sectors.
__global__ void __launch_bounds__(256) k_scatter(const float* __restrict__ x, const float* __restrict__ y,
                                                 const float* __restrict__ z, int stride, int n,
                                                 const int2* __restrict__ ct, const int* __restrict__ offsets,
                                                 float4* __restrict__ tmp, unsigned* status, int c_lo, int c_hi) {
    constexpr int U = 4;
    const long long step = (long long)gridDim.x * blockDim.x;
    for (long long i0 = (long long)blockIdx.x * blockDim.x + threadIdx.x; i0 < n; i0 += U * step) {
        int2 c[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const long long i = i0 + u * step;
            c[u] = i < n ? __ldg(&ct[i]) : make_int2(0, 0);
        }
        long long slot[U];
        float px[U], py[U], pz[U];
        bool mine[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const long long i = i0 + u * step;
            mine[u] = i < n && c[u].x >= c_lo && c[u].x < c_hi;
            slot[u] = mine[u] ? (long long)__ldg(&offsets[c[u].x]) + c[u].y : -1;
            px[u] = mine[u] ? __ldg(&x[i * stride]) : 0.f;
            py[u] = mine[u] ? __ldg(&y[i * stride]) : 0.f;
            pz[u] = mine[u] ? __ldg(&z[i * stride]) : 0.f;
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const long long i = i0 + u * step;
            if (!mine[u]) continue;
            if (slot[u] >= 0 && slot[u] < n)
                tmp[slot[u]] = make_float4(px[u], py[u], pz[u], __int_as_float((int)i));
            else
                atomicOr(status, kFlagRange);
        }
    }
}

// ---------------------------------------------------------------- within-cell sort
// Keys: LJ_ORDER_INDEX sorts by original index; LJ_ORDER_X by x, then index.
// Indices are unique, so keys are unique and the result is a pure function of
// the input.
template <int ORDER>
__device__ __forceinline__ bool key_less(float xa, int ia, float xb, int ib) {
    if (ORDER == LJ_ORDER_X) return (xa < xb) || (xa == xb && ia < ib);
    return ia < ib;
}

struct SortOut {
    float4* out4;
    int* out_cell;
    float* sx;
    float* sy;
    float* sz;
    int* sidx;
};

__device__ __forceinline__ void emit(const SortOut& o, long long slot, float4 r, int cell) {
    o.out4[slot] = r;
    o.out_cell[slot] = cell;
    if (o.sx) o.sx[slot] = r.x;
    if (o.sy) o.sy[slot] = r.y;
    if (o.sz) o.sz[slot] = r.z;
    if (o.sidx) o.sidx[slot] = __float_as_int(r.w);
}

constexpr long long kScatterRegion = 56LL << 20;  // bytes of tmp4 one scatter pass writes (L2 holds 126 MB)
constexpr int kRankMax = 512;    // cells up to this size are ranked record by record
constexpr int kLargeCapMin = 4096;

// One thread per record of the scattered (cell-grouped, unordered within a cell) array.  The
// record's cell is recomputed from its position with the count kernel's formula (the same float
// operations on the same values, so the same cell; with several systems, the system is found from
// the record's original index); its rank is the number of records of the same cell with a smaller
// key (a loop over the cell's records, which the neighbouring threads read too: L1 hits), and it
// is written at offset + rank.  Every lane is busy whatever the cell sizes.  Cells above kRankMax
// go to a list handled by k_large_sort (registered by the thread of the cell's first slot).
template <int ORDER>
__global__ void __launch_bounds__(256) k_cell_rank(const float4* __restrict__ tmp, const int* __restrict__ offsets,
                                                   GridDev g, const BinSys* __restrict__ sys,
                                                   const int* __restrict__ firsts, int nsys, int n, SortOut so,
                                                   int* large, int large_cap, unsigned* status) {
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
        const float4 r = tmp[s];
        int c;
        if (nsys == 0) {
            c = cell_of(g, r.x, r.y, r.z);
        } else {
            const int i = __float_as_int(r.w);
            int lo = 0, hi = nsys - 1;
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (__ldg(&firsts[mid]) <= i)
                    lo = mid;
                else
                    hi = mid - 1;
            }
            c = sys[lo].cell_base + cell_of(sys[lo].g, r.x, r.y, r.z);
        }
        so.out_cell[s] = c;  // every slot of a cell holds its id, whatever the order inside the cell
        const int o0 = min(max(__ldg(&offsets[c]), 0), n);
        const int o1 = min(max(__ldg(&offsets[c + 1]), o0), n);
        const int m = o1 - o0;
        if (m > kRankMax) {
            if (s == o0) {
                const int slot = atomicAdd(&large[0], 1);
                if (slot < large_cap)
                    large[1 + slot] = c;
                else
                    atomicOr(status, kFlagRange);
            }
            continue;
        }
        const float rx = r.x;
        const int ri = __float_as_int(r.w);
        int rank = 0;
        for (int j = o0; j < o1; ++j) {
            const float4 t = tmp[j];
            rank += key_less<ORDER>(t.x, __float_as_int(t.w), rx, ri) ? 1 : 0;
        }
        const long long slot = (long long)o0 + rank;
        so.out4[slot] = r;
        if (so.sx) so.sx[slot] = r.x;
        if (so.sy) so.sy[slot] = r.y;
        if (so.sz) so.sz[slot] = r.z;
        if (so.sidx) so.sidx[slot] = __float_as_int(r.w);
    }
}

// Cells larger than kRankMax (rare: clustered or degenerate inputs): one
// CTA per cell sorts 2048-record chunks in shared memory (bitonic network),
// then merges runs pairwise, each record finding its place in the partner run
// by binary search; ping-pong between the cell's tmp and out ranges.
template <int ORDER>
__device__ __forceinline__ bool rec_less(const float4& a, const float4& b) {
    return key_less<ORDER>(a.x, __float_as_int(a.w), b.x, __float_as_int(b.w));
}

template <int ORDER>
__global__ void __launch_bounds__(1024) k_large_sort(float4* __restrict__ tmp, const int* __restrict__ offsets,
                                                     int n, SortOut so, const int* __restrict__ large,
                                                     int large_cap) {
    __shared__ float4 sbuf[2048];
    const int count = min(large[0], large_cap);
    const int tid = threadIdx.x;
    for (int li = blockIdx.x; li < count; li += gridDim.x) {
        const int c = large[1 + li];
        int o = min(max(offsets[c], 0), n);
        int e1 = min(max(offsets[c + 1], o), n);
        const int cnt = e1 - o;
        float4* A = tmp + o;
        float4* B = so.out4 + o;
        const float4 sentinel = make_float4(__int_as_float(0x7f800000), 0.f, 0.f, __int_as_float(INT_MAX));
        for (int ch = 0; ch < cnt; ch += 2048) {
            const int len = min(2048, cnt - ch);
            for (int i = tid; i < 2048; i += 1024) sbuf[i] = i < len ? A[ch + i] : sentinel;
            __syncthreads();
            for (int k = 2; k <= 2048; k <<= 1)
                for (int j = k >> 1; j > 0; j >>= 1) {
                    for (int i = tid; i < 2048; i += 1024) {
                        const int p = i ^ j;
                        if (p > i) {
                            const bool up = (i & k) == 0;
                            const float4 a = sbuf[i], b = sbuf[p];
                            if (rec_less<ORDER>(b, a) == up) {
                                sbuf[i] = b;
                                sbuf[p] = a;
                            }
                        }
                    }
                    __syncthreads();
                }
            for (int i = tid; i < len; i += 1024) B[ch + i] = sbuf[i];
            __syncthreads();
        }
        float4* src = B;
        float4* dst = A;
        for (int width = 2048; width < cnt; width *= 2) {
            for (int e = tid; e < cnt; e += 1024) {
                const int run = e / width;
                const int run_start = run * width;
                const int pair_start = (run & ~1) * width;
                const bool left = (run & 1) == 0;
                const int other = left ? run_start + width : run_start - width;
                const int other_len = left ? max(0, min(cnt - other, width)) : width;
                const float4 r = src[e];
                int lo = 0, hi = other_len;
                while (lo < hi) {
                    const int mid = (lo + hi) >> 1;
                    if (rec_less<ORDER>(src[other + mid], r))
                        lo = mid + 1;
                    else
                        hi = mid;
                }
                dst[pair_start + (e - run_start) + lo] = r;
            }
            __syncthreads();
            float4* t = src;
            src = dst;
            dst = t;
        }
        for (int e = tid; e < cnt; e += 1024) emit(so, (long long)o + e, src[e], c);
        __syncthreads();
    }
}

// ---------------------------------------------------------------- descriptors / candidates
__global__ void __launch_bounds__(256) k_descriptors(const int* __restrict__ offsets, long long ncells,
                                                     lj_cell_desc* __restrict__ cells) {
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < ncells;
         c += (long long)gridDim.x * blockDim.x) {
        const int o0 = offsets[c], o1 = offsets[c + 1];
        cells[c] = lj_cell_desc{o1 - o0, o0};
    }
}

// Candidate ordered pairs: sum over cells of count * (stencil occupancy - 1),
// the stencil being the clamped 3x3x3 block read as 9 rows of consecutive
// cells.  Integer atomics make the total order-independent.
__global__ void __launch_bounds__(256) k_candidates(GridDev g, const int* __restrict__ offsets, long long ncells,
                                                    unsigned long long* out) {
    __shared__ unsigned long long s[8];
    unsigned long long acc = 0;
    const long long gxy = (long long)g.gx * g.gy;
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < ncells;
         c += (long long)gridDim.x * blockDim.x) {
        const long long cnt = (long long)__ldg(&offsets[c + 1]) - __ldg(&offsets[c]);
        if (cnt <= 0) continue;
        const int cz = (int)(c / gxy);
        const long long r = c - cz * gxy;
        const int cy = (int)(r / g.gx);
        const int cx = (int)(r - (long long)cy * g.gx);
        const int xl = max(cx - 1, 0), xh = min(cx + 1, g.gx - 1);
        long long s_occ = 0;
        for (int z = max(cz - 1, 0); z <= min(cz + 1, g.gz - 1); ++z)
            for (int y = max(cy - 1, 0); y <= min(cy + 1, g.gy - 1); ++y) {
                const long long rb = ((long long)z * g.gy + y) * g.gx;
                s_occ += (long long)__ldg(&offsets[rb + xh + 1]) - __ldg(&offsets[rb + xl]);
            }
        acc += (unsigned long long)(cnt * (s_occ - 1));
    }
    acc = warp_sum(acc);
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        unsigned long long t = threadIdx.x < (blockDim.x >> 5) ? s[threadIdx.x] : 0ULL;
        t = warp_sum(t);
        if (threadIdx.x == 0 && t) atomicAdd(out, t);
    }
}

#ifdef LJ_CHECKS
// ---------------------------------------------------------------- consistency checks (-DLJ_CHECKS)
// The bounds-checked build (libljcell_checks.so) verifies after each binning stage what the next
// stage relies on; a violation ORs kFlagCheck into the status word, which lj_sync reports as
// LJ_ECHECK.  The checks only read their buffers (and mark one scratch array); none traps.

// Counts are non-negative and offsets[c + 1] - offsets[c] = counts[c], offsets[0] = 0.
__global__ void k_chk_scan(const int* __restrict__ counts, const int* __restrict__ offsets, long long nc,
                           unsigned* status) {
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < nc;
         c += (long long)gridDim.x * blockDim.x) {
        const int k = counts[c], a = offsets[c], b = offsets[c + 1];
        if (k < 0 || b - a != k || (c == 0 && a != 0)) atomicOr(status, kFlagCheck);
    }
}

// Each particle's (cell, ticket): a cell of the grid, a ticket below that cell's count.
__global__ void k_chk_tickets(const int2* __restrict__ ct, const int* __restrict__ counts, int n, long long nc,
                              unsigned* status) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int2 v = ct[i];
        if (v.x < 0 || v.x >= nc || v.y < 0 || v.y >= counts[v.x]) atomicOr(status, kFlagCheck);
    }
}

// Sorted records: original index in [0, n) (marked in seen), cell in [0, nc) with the record inside
// the cell's offset range, cells non-decreasing, the within-cell order strict, and (single system)
// the cell recomputed from the stored position equal to the stored one.
template <int ORDER>
__global__ void k_chk_sorted(GridDev g, int recompute, const float4* __restrict__ xyzi, const int* __restrict__ cell,
                             const int* __restrict__ offsets, int n, long long nc, int* __restrict__ seen,
                             unsigned* status) {
    for (long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x; s < n; s += (long long)gridDim.x * blockDim.x) {
        const float4 r = xyzi[s];
        const int i = __float_as_int(r.w), c = cell[s];
        bool bad = i < 0 || i >= n || c < 0 || c >= nc;
        if (!bad) {
            atomicAdd(&seen[i], 1);
            bad = s < offsets[c] || s >= offsets[c + 1];
        }
        if (!bad && recompute && isfinite(r.x) && isfinite(r.y) && isfinite(r.z)) bad = cell_of(g, r.x, r.y, r.z) != c;
        if (!bad && s > 0) {
            const float4 q = xyzi[s - 1];
            const int cp = cell[s - 1];
            bad = cp > c || (cp == c && key_less<ORDER>(r.x, i, q.x, __float_as_int(q.w)));
        }
        if (bad) atomicOr(status, kFlagCheck);
    }
}

// Every original index seen exactly once: the sorted order is a permutation.
__global__ void k_chk_seen(const int* __restrict__ seen, int n, unsigned* status) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        if (seen[i] != 1) atomicOr(status, kFlagCheck);
}
#endif

// ---------------------------------------------------------------- host side

static lj_status check_grid(const lj_grid* g, long long* ncells) {
    if (!g || !(g->width > 0.0f) || g->dim[0] < 1 || g->dim[1] < 1 || g->dim[2] < 1) return LJ_EINVAL;
    const long long nc = (long long)g->dim[0] * g->dim[1] * g->dim[2];
    if (nc > (long long)INT_MAX - 1) return LJ_EUNSUPPORTED;
    *ncells = nc;
    return LJ_OK;
}

lj_status launch_scan(lj_ctx* ctx, const int* counts, long long ncells, int* offsets) {
    const long long ntiles = (ncells + kScanTile - 1) / kScanTile;
    const size_t need = 256 + (size_t)(ntiles > 0 ? ntiles : 1) * sizeof(unsigned long long);
    lj_status s = grow(&ctx->scan_state, &ctx->scan_state_bytes, need);
    if (s != LJ_OK) return s;
    if (ncells == 0) {
        if (cudaMemsetAsync(offsets, 0, sizeof(int), ctx->stream) != cudaSuccess) return LJ_ECUDA;
        return LJ_OK;
    }
    if (cudaMemsetAsync(ctx->scan_state, 0, need, ctx->stream) != cudaSuccess) return LJ_ECUDA;
    unsigned* counter = reinterpret_cast<unsigned*>(ctx->scan_state);
    unsigned long long* states = reinterpret_cast<unsigned long long*>(static_cast<char*>(ctx->scan_state) + 256);
    const int vec_ok = ((reinterpret_cast<uintptr_t>(counts) | reinterpret_cast<uintptr_t>(offsets)) & 15) == 0;
    k_scan<<<(unsigned)ntiles, kScanThreads, 0, ctx->stream>>>(counts, offsets, ncells, ntiles, states, counter,
                                                              vec_ok, ctx->d_status);
#ifdef LJ_CHECKS
    if ((s = last_launch_status()) != LJ_OK) return s;
    k_chk_scan<<<grid_for(ctx, ncells, 256), 256, 0, ctx->stream>>>(counts, offsets, ncells, ctx->d_status);
#endif
    return last_launch_status();
}

}  // namespace ljc

using namespace ljc;

extern "C" lj_status lj_count_cells(lj_ctx* ctx, const lj_grid* g, int n, const float* x, const float* y,
                                    const float* z, int stride, int* counts) {
    long long nc;
    if (!ctx || n < 0 || !counts || stride < 1) return LJ_EINVAL;
    lj_status s = check_grid(g, &nc);
    if (s != LJ_OK) return s;
    if (n > 0 && (!x || !y || !z)) return LJ_EINVAL;
    if (cudaMemsetAsync(counts, 0, sizeof(int) * (size_t)nc, ctx->stream) != cudaSuccess) return LJ_ECUDA;
    if (n == 0) return LJ_OK;
    k_count<false><<<grid_for(ctx, n, 256), 256, 0, ctx->stream>>>(to_dev(*g), x, y, z, stride, n, counts, nullptr,
                                                                  ctx->d_status);
    return last_launch_status();
}

extern "C" lj_status lj_exclusive_scan(lj_ctx* ctx, const int* counts, long long ncells, int* offsets) {
    const NvtxRange nvtx_range("lj_exclusive_scan");
    if (!ctx || ncells < 0 || !offsets || (ncells > 0 && !counts)) return LJ_EINVAL;
    if (ncells > (long long)INT_MAX - 1) return LJ_EUNSUPPORTED;
    return launch_scan(ctx, counts, ncells, offsets);
}

extern "C" lj_status lj_cell_descriptors(lj_ctx* ctx, const int* offsets, long long ncells, lj_cell_desc* cells) {
    if (!ctx || ncells < 0 || !offsets || !cells) return LJ_EINVAL;
    if (ncells == 0) return LJ_OK;
    k_descriptors<<<grid_for(ctx, ncells, 256), 256, 0, ctx->stream>>>(offsets, ncells, cells);
    return last_launch_status();
}

namespace ljc {

// Stage 1 of a cell-grid build: scratch for n particles, counts zeroed.
lj_status bin_prepare(lj_ctx* ctx, int n, long long nc, int* counts) {
    lj_status s;
    const size_t need = (size_t)(n > 0 ? n : 1);
    if (need > ctx->part_cap) {
        void* p1 = ctx->cell_ticket;
        void* p2 = ctx->tmp4;
        size_t c1 = ctx->part_cap * sizeof(int2), c2 = ctx->part_cap * sizeof(float4);
        // a failed growth has freed its old buffer: record the null pointer and a zero capacity
        // so that no freed buffer is used or freed again
        s = grow(&p1, &c1, need * sizeof(int2));
        ctx->cell_ticket = static_cast<int2*>(p1);
        if (s == LJ_OK) {
            s = grow(&p2, &c2, need * sizeof(float4));
            ctx->tmp4 = static_cast<float4*>(p2);
        }
        if (s != LJ_OK) {
            ctx->part_cap = 0;
            return s;
        }
        ctx->part_cap = need;
    }
    const size_t large_need = (size_t)std::max<long long>(kLargeCapMin, (long long)n / kRankMax + 1);
    if (!ctx->large_cells || ctx->large_cap < large_need) {
        void* p = ctx->large_cells;
        size_t cap = ctx->large_cells ? sizeof(int) * (1 + ctx->large_cap) : 0;
        s = grow(&p, &cap, sizeof(int) * (1 + large_need));
        ctx->large_cells = static_cast<int*>(p);
        ctx->large_cap = s == LJ_OK ? large_need : 0;
        if (s != LJ_OK) return s;
    }
    if (cudaMemsetAsync(counts, 0, sizeof(int) * (size_t)nc, ctx->stream) != cudaSuccess) return LJ_ECUDA;
    if (cudaMemsetAsync(ctx->large_cells, 0, sizeof(int), ctx->stream) != cudaSuccess) return LJ_ECUDA;
    return LJ_OK;
}

// Stages after a count kernel has filled counts and ctx->cell_ticket: scan,
// scatter, within-cell sort (with the descriptor view and SoA outputs).
lj_status bin_finish(lj_ctx* ctx, long long nc, int n, const float* x, const float* y, const float* z, int stride,
                     lj_order order, int* counts, int* offsets, lj_cell_desc* cells, lj_particles* sorted,
                     float* sorted_xyzi, int* sorted_cell, const GridDev& g, const BinSys* sys, const int* firsts,
                     int nsys) {
    lj_status s;
    cudaStream_t st = ctx->stream;
    if ((s = launch_scan(ctx, counts, nc, offsets)) != LJ_OK) return s;
#ifdef LJ_CHECKS
    if (n > 0) {
        k_chk_tickets<<<grid_for(ctx, n, 256), 256, 0, st>>>(ctx->cell_ticket, counts, n, nc, ctx->d_status);
        if ((s = last_launch_status()) != LJ_OK) return s;
    }
#endif
    if (n > 0) {
        // passes: the tuning's scatter_passes, else enough that each pass writes about kScatterRegion bytes
        long long passes = ctx->tuning.scatter_passes;
        if (passes <= 0) passes = ((long long)n * (long long)sizeof(float4) + kScatterRegion - 1) / kScatterRegion;
        passes = std::max(1LL, std::min(passes, std::min(8LL, nc)));
        for (long long q = 0; q < passes; ++q) {
            const int c_lo = (int)(nc * q / passes), c_hi = (int)(nc * (q + 1) / passes);
            k_scatter<<<grid_for(ctx, n, 256), 256, 0, st>>>(x, y, z, stride, n, ctx->cell_ticket, offsets,
                                                             ctx->tmp4, ctx->d_status, c_lo, c_hi);
            if ((s = last_launch_status()) != LJ_OK) return s;
        }
    }
    SortOut so{reinterpret_cast<float4*>(sorted_xyzi), sorted_cell, nullptr, nullptr, nullptr, nullptr};
    if (sorted) {
        so.sx = sorted->x;
        so.sy = sorted->y;
        so.sz = sorted->z;
        so.sidx = sorted->index;
    }
    const int lcap = (int)ctx->large_cap;
    if (n > 0) {
        if (order == LJ_ORDER_X) {
            k_cell_rank<LJ_ORDER_X><<<grid_for(ctx, n, 256), 256, 0, st>>>(ctx->tmp4, offsets, g, sys, firsts, nsys, n,
                                                                           so, ctx->large_cells, lcap, ctx->d_status);
            if ((s = last_launch_status()) != LJ_OK) return s;
            k_large_sort<LJ_ORDER_X><<<ctx->sm_count, 1024, 0, st>>>(ctx->tmp4, offsets, n, so, ctx->large_cells,
                                                                     lcap);
        } else {
            k_cell_rank<LJ_ORDER_INDEX><<<grid_for(ctx, n, 256), 256, 0, st>>>(ctx->tmp4, offsets, g, sys, firsts, nsys,
                                                                               n, so, ctx->large_cells, lcap,
                                                                               ctx->d_status);
            if ((s = last_launch_status()) != LJ_OK) return s;
            k_large_sort<LJ_ORDER_INDEX><<<ctx->sm_count, 1024, 0, st>>>(ctx->tmp4, offsets, n, so,
                                                                         ctx->large_cells, lcap);
        }
        if ((s = last_launch_status()) != LJ_OK) return s;
    }
    if (cells) {
        k_descriptors<<<grid_for(ctx, nc, 256), 256, 0, st>>>(offsets, nc, cells);
    }
#ifdef LJ_CHECKS
    // the permutation check needs scratch, which cannot be allocated while a graph is being captured
    cudaStreamCaptureStatus capturing = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st, &capturing) != cudaSuccess) return LJ_ECUDA;
    if (n > 0 && capturing == cudaStreamCaptureStatusNone) {
        if ((s = grow(&ctx->check, &ctx->check_bytes, (size_t)n * sizeof(int))) != LJ_OK) return s;
        int* seen = static_cast<int*>(ctx->check);
        if (cudaMemsetAsync(seen, 0, (size_t)n * sizeof(int), st) != cudaSuccess) return LJ_ECUDA;
        const float4* x4 = reinterpret_cast<const float4*>(sorted_xyzi);
        if (order == LJ_ORDER_X)
            k_chk_sorted<LJ_ORDER_X><<<grid_for(ctx, n, 256), 256, 0, st>>>(g, sys == nullptr, x4, sorted_cell, offsets,
                                                                            n, nc, seen, ctx->d_status);
        else
            k_chk_sorted<LJ_ORDER_INDEX><<<grid_for(ctx, n, 256), 256, 0, st>>>(g, sys == nullptr, x4, sorted_cell,
                                                                                offsets, n, nc, seen, ctx->d_status);
        if ((s = last_launch_status()) != LJ_OK) return s;
        k_chk_seen<<<grid_for(ctx, n, 256), 256, 0, st>>>(seen, n, ctx->d_status);
    }
#endif
    return last_launch_status();
}

}  // namespace ljc

extern "C" lj_status lj_bin(lj_ctx* ctx, const lj_grid* g, int n, const float* x, const float* y, const float* z,
                            int stride, lj_order order, int* counts, int* offsets, lj_cell_desc* cells,
                            lj_particles* sorted, float* sorted_xyzi, int* sorted_cell) {
    const NvtxRange nvtx_range("lj_bin");
    long long nc;
    if (!ctx || n < 0 || stride < 1 || !counts || !offsets) return LJ_EINVAL;
    if (order != LJ_ORDER_INDEX && order != LJ_ORDER_X) return LJ_EINVAL;
    lj_status s = check_grid(g, &nc);
    if (s != LJ_OK) return s;
    if (n > 0 && (!x || !y || !z || !sorted_xyzi || !sorted_cell)) return LJ_EINVAL;
    if (reinterpret_cast<uintptr_t>(sorted_xyzi) & 15) return LJ_EINVAL;
    if ((s = bin_prepare(ctx, n, nc, counts)) != LJ_OK) return s;
    if (n > 0) {
        k_count<true><<<grid_for(ctx, n, 256), 256, 0, ctx->stream>>>(to_dev(*g), x, y, z, stride, n, counts,
                                                                      ctx->cell_ticket, ctx->d_status);
        if ((s = last_launch_status()) != LJ_OK) return s;
    }
    return bin_finish(ctx, nc, n, x, y, z, stride, order, counts, offsets, cells, sorted, sorted_xyzi, sorted_cell,
                      to_dev(*g), nullptr, nullptr, 0);
}

extern "C" lj_status lj_count_candidates(lj_ctx* ctx, const lj_grid* g, const int* offsets,
                                         unsigned long long* d_count) {
    const NvtxRange nvtx_range("lj_count_candidates");
    long long nc;
    if (!ctx || !offsets || !d_count) return LJ_EINVAL;
    lj_status s = check_grid(g, &nc);
    if (s != LJ_OK) return s;
    if (cudaMemsetAsync(d_count, 0, sizeof(unsigned long long), ctx->stream) != cudaSuccess) return LJ_ECUDA;
    k_candidates<<<grid_for(ctx, nc, 256), 256, 0, ctx->stream>>>(to_dev(*g), offsets, nc, d_count);
    return last_launch_status();
}

// ---------------------------------------------------------------- failure-path test hook
namespace ljc {
__global__ void k_set_u32(unsigned* p, unsigned v) { *p = v; }
}  // namespace ljc

// Runs k_scan with tile 0 withheld: the counter starts at 1, so no CTA ever
// publishes tile 0 and every look-back wait runs out its bounded limit,
// records LJ_ETIMEOUT in the context's status word and returns.  Exercises the
// error path of the bounded waits without faulting or hanging the GPU.
extern "C" lj_status lj_test_scan_withheld_tile(lj_ctx* ctx, const int* counts, long long ncells, int* offsets) {
    if (!ctx || !counts || !offsets || ncells <= kScanTile || ncells > (long long)INT_MAX - 1) return LJ_EINVAL;
    const long long ntiles = (ncells + kScanTile - 1) / kScanTile;
    const size_t need = 256 + (size_t)ntiles * sizeof(unsigned long long);
    lj_status s = grow(&ctx->scan_state, &ctx->scan_state_bytes, need);
    if (s != LJ_OK) return s;
    if (cudaMemsetAsync(ctx->scan_state, 0, need, ctx->stream) != cudaSuccess) return LJ_ECUDA;
    unsigned* counter = reinterpret_cast<unsigned*>(ctx->scan_state);
    unsigned long long* states = reinterpret_cast<unsigned long long*>(static_cast<char*>(ctx->scan_state) + 256);
    k_set_u32<<<1, 1, 0, ctx->stream>>>(counter, 1u);
    k_scan<<<(unsigned)(ntiles - 1), kScanThreads, 0, ctx->stream>>>(counts, offsets, ncells, ntiles, states, counter,
                                                                      0, ctx->d_status);
    return last_launch_status();
}

// ---------------------------------------------------------------- allocation-free scan
// Some callers cannot allocate device memory at all: code running under an
// allocator that forbids cudaMalloc (a memory pool that owns the whole device,
// a pre-sized plugin host) or code that must not stall other streams on the
// implicit synchronisation that cudaMalloc / cudaFree can cause.  For them
// lj_exclusive_scan_noalloc runs k_scan with its look-back scratch (tile
// counter + one 64-bit state per 4096-cell tile) in this file-scope array
// instead of a context's allocation.  Every GPU that loads the library holds
// the array (kNoAllocScratchBytes) until the process exits.
namespace ljc {

constexpr long long kNoAllocMaxCells = 1LL << 26;  // 67,108,864 cells
constexpr long long kNoAllocMaxTiles = kNoAllocMaxCells / kScanTile;
constexpr size_t kNoAllocScratchBytes = 256 + (size_t)kNoAllocMaxTiles * sizeof(unsigned long long);

// [0, 4): tile counter; [4, 8): status word; [256, ...): tile states.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// Device address of the array on the current device.  Looked up on every call (cudaGetSymbolAddress
// allocates nothing): an address kept from an earlier call would go stale if the caller reset the
// device in between.
static lj_status noalloc_scratch(void** out) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) {
        cudaGetLastError();
        return LJ_ECUDA;
    }
    *out = p;
    return LJ_OK;
}

// A look-back that gave up (kFlagTimeout in the array's status word) marks
// the result invalid with offsets[n] = -1; a valid total is never negative.
__global__ void k_noalloc_mark(const unsigned* status, int* offsets, long long n) {
    if (*status) offsets[n] = -1;
}

// The scan on the array.  withhold: tile 0 is never published (the tile counter starts at 1 and one
// CTA fewer runs), so every bounded look-back wait gives up: the failure path, for tests.
static lj_status noalloc_scan(const int* counts, long long ncells, int* offsets, void* stream, bool withhold) {
    if (ncells < 0 || !offsets || (ncells > 0 && !counts)) return LJ_EINVAL;
    if (ncells > kNoAllocMaxCells) return LJ_EUNSUPPORTED;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int cur = -1;
    if (cudaGetDevice(&cur) != cudaSuccess) return LJ_ECUDA;
    if (st) {  // the array resolved below is the current device's: the stream must belong to it
        int sdev = -1;
        if (cudaStreamGetDevice(st, &sdev) != cudaSuccess) {
            cudaGetLastError();
            return LJ_EINVAL;
        }
        if (sdev != cur) return LJ_EINVAL;
    }
    void* scratch = nullptr;
    lj_status s = noalloc_scratch(&scratch);
    if (s != LJ_OK) return s;
    if (ncells == 0) return cudaMemsetAsync(offsets, 0, sizeof(int), st) == cudaSuccess ? LJ_OK : LJ_ECUDA;
    const long long ntiles = (ncells + kScanTile - 1) / kScanTile;
    if (withhold && ntiles < 2) return LJ_EINVAL;
    // the counter, status and the states this call uses must start at zero; the array keeps the last call's values
    const size_t used = 256 + (size_t)ntiles * sizeof(unsigned long long);
    if (cudaMemsetAsync(scratch, 0, used, st) != cudaSuccess) return LJ_ECUDA;
    unsigned* counter = static_cast<unsigned*>(scratch);
    unsigned* status = counter + 1;
    unsigned long long* states = reinterpret_cast<unsigned long long*>(static_cast<char*>(scratch) + 256);
    if (withhold) k_set_u32<<<1, 1, 0, st>>>(counter, 1u);
    const int vec_ok = ((reinterpret_cast<uintptr_t>(counts) | reinterpret_cast<uintptr_t>(offsets)) & 15) == 0;
    k_scan<<<(unsigned)(withhold ? ntiles - 1 : ntiles), kScanThreads, 0, st>>>(counts, offsets, ncells, ntiles,
                                                                                 states, counter, vec_ok, status);
    if ((s = last_launch_status()) != LJ_OK) return s;
    k_noalloc_mark<<<1, 1, 0, st>>>(status, offsets, ncells);
    return last_launch_status();
}

}  // namespace ljc

extern "C" lj_status lj_exclusive_scan_noalloc(const int* counts, long long ncells, int* offsets, void* stream) {
    return noalloc_scan(counts, ncells, offsets, stream, false);
}

extern "C" lj_status lj_test_scan_noalloc_withheld_tile(const int* counts, long long ncells, int* offsets,
                                                        void* stream) {
    return noalloc_scan(counts, ncells, offsets, stream, true);
}

// ---------------------------------------------------------------- spatial sort (lj_reorder)
// The operation of the reference's reorder() (SDK/optixMultiSphereAABB/sort.cu:29-41 with its key
// kernel count_per_cell, :7-18): each float4 point gets the key of its cell, width = int(1 / radius),
// id = int(x / radius) + int(y / radius) * width + int(z / radius) * width^2, stored in .w as float,
// and the points are sorted by .w.  The division is the one the reference's own build performs: its
// SDK compiles sort.cu with --use_fast_math, so x / radius is the fast single-precision division
// (__fdividef here; it and IEEE division can truncate to different cells for a coordinate within a
// couple of ulps of a cell face).  The key is summed in exact integers: stored in .w (one rounding to
// float) it equals the reference's float sum, which the compiler contracts into fused multiply-adds
// (both checked against the reference built from source, on points next to cell faces too).  Here the sort
// is a counting sort over the keys on the binning kernels: count with tickets, scan, ticket scatter
// (k_scatter, reading x, y, z with stride 4), then a rank by original index within each key, so
// points of equal .w keep their input order (the reference's thrust::sort leaves that order open).
// Keys are counted as int(float(id)), the value .w holds, so two ids that round to the same float
// share a bin exactly as they compare equal in the reference.
namespace ljc {

constexpr int kReorderMaxWidth = 512;  // int(1 / radius) <= 512: at most 134,480,385 keys

struct ReorderKey {
    float radius;
    int width;
    int nkeys;
};

__device__ __forceinline__ int reorder_key(const ReorderKey& rk, float x, float y, float z, bool& bad) {
    const int cx = __float2int_rz(__fdividef(x, rk.radius));
    const int cy = __float2int_rz(__fdividef(y, rk.radius));
    const int cz = __float2int_rz(__fdividef(z, rk.radius));
    const long long id = (long long)cx + (long long)cy * rk.width + (long long)cz * rk.width * rk.width;
    bad = !(x == x && y == y && z == z) || id < 0 || id > INT_MAX;
    const int kf = bad ? 0 : __float2int_rz(__int2float_rn((int)id));
    if (kf >= rk.nkeys) {
        bad = true;
        return 0;
    }
    return kf;
}

__global__ void __launch_bounds__(256) k_reorder_count(const float4* __restrict__ pts, int n, ReorderKey rk,
                                                       int* __restrict__ counts, int2* __restrict__ ct,
                                                       unsigned* status) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 p = pts[i];
        bool bad;
        const int key = reorder_key(rk, p.x, p.y, p.z, bad);
        if (bad) atomicOr(status, kFlagRange);
        // one atomic per distinct key in the warp (points of a key often arrive together)
        const unsigned peers = __match_any_sync(__activemask(), key);
        const int leader = __ffs(peers) - 1;
        int base = 0;
        if ((int)lane_id() == leader) base = atomicAdd(&counts[key], __popc(peers));
        base = __shfl_sync(peers, base, leader);
        ct[i] = make_int2(key, base + __popc(peers & lanemask_lt()));
    }
}

// Rank of each scattered record among the records of its key, by original index (as k_cell_rank);
// keys above kRankMax records go to the large list for k_large_sort<LJ_ORDER_INDEX>.
__global__ void __launch_bounds__(256) k_reorder_rank(const float4* __restrict__ tmp, const int2* __restrict__ ct,
                                                      const int* __restrict__ offsets, int n, SortOut so, int* large,
                                                      int large_cap, unsigned* status) {
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
        const float4 r = tmp[s];
        const int i = __float_as_int(r.w);
        const int c = (i >= 0 && i < n) ? __ldg(&ct[i]).x : 0;
        so.out_cell[s] = c;
        const int o0 = min(max(__ldg(&offsets[c]), 0), n);
        const int o1 = min(max(__ldg(&offsets[c + 1]), o0), n);
        const int m = o1 - o0;
        if (m > kRankMax) {
            if (s == o0) {
                const int slot = atomicAdd(&large[0], 1);
                if (slot < large_cap)
                    large[1 + slot] = c;
                else
                    atomicOr(status, kFlagRange);
            }
            continue;
        }
        int rank = 0;
        for (int j = o0; j < o1; ++j) rank += __float_as_int(tmp[j].w) < i ? 1 : 0;
        so.out4[(long long)o0 + rank] = r;
    }
}

__global__ void __launch_bounds__(256) k_reorder_emit(const float4* __restrict__ sorted, const int* __restrict__ key,
                                                      int n, float4* __restrict__ pts) {
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
        const float4 r = sorted[s];
        pts[s] = make_float4(r.x, r.y, r.z, __int2float_rn(key[s]));
    }
}

}  // namespace ljc

extern "C" lj_status lj_reorder(lj_ctx* ctx, int n, float* points, float radius) {
    const NvtxRange nvtx_range("lj_reorder");
    if (!ctx || n < 0 || (n > 0 && !points) || !(radius > 0.0f) || !(radius < 3.4e38f)) return LJ_EINVAL;
    if (reinterpret_cast<uintptr_t>(points) & 15) return LJ_EINVAL;
    if (n == 0) return LJ_OK;
    const float wf = 1.0f / radius;
    if (!(wf < (float)kReorderMaxWidth + 1.0f)) return LJ_EUNSUPPORTED;
    const long long width = (long long)wf;  // the reference's int(1.0f / radius)
    // coordinates in [0, 1] give cell coordinates in [0, width]
    const long long max_id = width + width * width + width * width * width;
    const long long max_key = std::max(max_id, (long long)(float)max_id);
    const long long nkeys = max_key + 1;
    ReorderKey rk{radius, (int)width, (int)nkeys};
    lj_status s;
    // scratch: counts[nkeys], offsets[nkeys + 1] (16-byte aligned), sorted float4[n], keys int[n]
    const size_t cnt_bytes = ((size_t)nkeys * sizeof(int) + 255) & ~(size_t)255;
    const size_t off_bytes = (((size_t)nkeys + 1) * sizeof(int) + 255) & ~(size_t)255;
    const size_t rec_bytes = (size_t)n * sizeof(float4);
    const size_t key_bytes = (size_t)n * sizeof(int);
    if ((s = grow(&ctx->reorder, &ctx->reorder_bytes, cnt_bytes + off_bytes + rec_bytes + key_bytes)) != LJ_OK)
        return s;
    char* base = static_cast<char*>(ctx->reorder);
    int* counts = reinterpret_cast<int*>(base);
    int* offsets = reinterpret_cast<int*>(base + cnt_bytes);
    float4* sorted = reinterpret_cast<float4*>(base + cnt_bytes + off_bytes);
    int* keys = reinterpret_cast<int*>(base + cnt_bytes + off_bytes + rec_bytes);
    cudaStream_t st = ctx->stream;
    if ((s = bin_prepare(ctx, n, nkeys, counts)) != LJ_OK) return s;  // tickets, tmp4, large list; counts zeroed
    const float4* p4 = reinterpret_cast<const float4*>(points);
    k_reorder_count<<<grid_for(ctx, n, 256), 256, 0, st>>>(p4, n, rk, counts, ctx->cell_ticket, ctx->d_status);
    if ((s = last_launch_status()) != LJ_OK) return s;
    if ((s = launch_scan(ctx, counts, nkeys, offsets)) != LJ_OK) return s;
    k_scatter<<<grid_for(ctx, n, 256), 256, 0, st>>>(points, points + 1, points + 2, 4, n, ctx->cell_ticket, offsets,
                                                     ctx->tmp4, ctx->d_status, 0, INT_MAX);
    if ((s = last_launch_status()) != LJ_OK) return s;
    SortOut so{sorted, keys, nullptr, nullptr, nullptr, nullptr};
    const int lcap = (int)ctx->large_cap;
    k_reorder_rank<<<grid_for(ctx, n, 256), 256, 0, st>>>(ctx->tmp4, ctx->cell_ticket, offsets, n, so,
                                                          ctx->large_cells, lcap, ctx->d_status);
    if ((s = last_launch_status()) != LJ_OK) return s;
    k_large_sort<LJ_ORDER_INDEX><<<ctx->sm_count, 1024, 0, st>>>(ctx->tmp4, offsets, n, so, ctx->large_cells, lcap);
    if ((s = last_launch_status()) != LJ_OK) return s;
    k_reorder_emit<<<grid_for(ctx, n, 256), 256, 0, st>>>(sorted, keys, n, reinterpret_cast<float4*>(points));
    return last_launch_status();
}
