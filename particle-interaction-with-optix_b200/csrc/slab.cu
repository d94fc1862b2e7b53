// slab.cu -- the boundary layers of a rank's particles, for the halo exchange of a slab
// decomposition over z (no counterpart in the reference, which runs one system on one GPU):
// lj_select_layers.
//
// A stable two-way compaction in three launches, deterministic (no atomics): k_sel_count counts,
// per block of kSelItems particles, those in the low and in the high layer; k_sel_scan turns the
// block counts into block offsets (one block, chunks of 1024 with a carry); k_sel_write recomputes
// each particle's layer and writes it at its block offset plus its rank among the block's matches
// (warp ballots, then the warps in order), so both outputs keep the input order.  The layer is the
// one lj_bin gives the particle (axis_cell: IEEE subtraction and division, truncation, clamped).
#include "ljcell_internal.cuh"

namespace ljc {

namespace {
constexpr int kSelThreads = 256;
constexpr int kSelPer = 4;                          // particles per thread
constexpr int kSelItems = kSelThreads * kSelPer;    // particles per block
constexpr int kSelWarps = kSelThreads / 32;

__device__ __forceinline__ int layer_of(const GridDev& g, const float* __restrict__ xyz, long long i) {
    return axis_cell(__ldg(&xyz[3 * i + 2]), g.oz, g.w, g.gz);
}
}  // namespace

__global__ void __launch_bounds__(kSelThreads) k_sel_count(GridDev g, const float* __restrict__ xyz, int n, int lo,
                                                            int hi, int2* __restrict__ block_counts) {
    __shared__ int s_lo[kSelWarps], s_hi[kSelWarps];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int c_lo = 0, c_hi = 0;
#pragma unroll
    for (int k = 0; k < kSelPer; ++k) {
        const long long i = (long long)blockIdx.x * kSelItems + k * kSelThreads + threadIdx.x;
        if (i < n) {
            const int layer = layer_of(g, xyz, i);
            c_lo += layer == lo;
            c_hi += layer == hi;
        }
    }
    c_lo = (int)__reduce_add_sync(0xffffffffu, (unsigned)c_lo);
    c_hi = (int)__reduce_add_sync(0xffffffffu, (unsigned)c_hi);
    if (lane == 0) {
        s_lo[warp] = c_lo;
        s_hi[warp] = c_hi;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int a = 0, b = 0;
        for (int w = 0; w < kSelWarps; ++w) {
            a += s_lo[w];
            b += s_hi[w];
        }
        block_counts[blockIdx.x] = make_int2(a, b);
    }
}

// Exclusive scan of the nb block counts in place (one block of 1024 threads); totals[0..1] = sums.
__global__ void __launch_bounds__(1024) k_sel_scan(int2* __restrict__ block_counts, int nb, int* __restrict__ totals) {
    __shared__ int2 s_warp[32];
    __shared__ int2 s_carry;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) s_carry = make_int2(0, 0);
    __syncthreads();
    for (int base = 0; base < nb; base += 1024) {
        const int i = base + threadIdx.x;
        const int2 v = i < nb ? block_counts[i] : make_int2(0, 0);
        int2 inc = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int tx = __shfl_up_sync(0xffffffffu, inc.x, o), ty = __shfl_up_sync(0xffffffffu, inc.y, o);
            if (lane >= o) {
                inc.x += tx;
                inc.y += ty;
            }
        }
        if (lane == 31) s_warp[warp] = inc;
        __syncthreads();
        if (warp == 0) {
            int2 w = s_warp[lane];
            int2 winc = w;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int tx = __shfl_up_sync(0xffffffffu, winc.x, o), ty = __shfl_up_sync(0xffffffffu, winc.y, o);
                if (lane >= o) {
                    winc.x += tx;
                    winc.y += ty;
                }
            }
            s_warp[lane] = make_int2(winc.x - w.x, winc.y - w.y);  // exclusive warp offsets
        }
        __syncthreads();
        const int2 c = s_carry;
        if (i < nb)
            block_counts[i] = make_int2(c.x + s_warp[warp].x + inc.x - v.x, c.y + s_warp[warp].y + inc.y - v.y);
        __syncthreads();
        if (threadIdx.x == 1023) s_carry = make_int2(c.x + s_warp[31].x + inc.x, c.y + s_warp[31].y + inc.y);
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        totals[0] = s_carry.x;
        totals[1] = s_carry.y;
    }
}

__global__ void __launch_bounds__(kSelThreads) k_sel_write(GridDev g, const float* __restrict__ xyz, int n, int lo,
                                                            int hi, const int2* __restrict__ block_offsets,
                                                            float* __restrict__ out_lo, float* __restrict__ out_hi) {
    __shared__ int s_lo[kSelWarps], s_hi[kSelWarps];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int2 bo = block_offsets[blockIdx.x];
    int run_lo = bo.x, run_hi = bo.y;  // matches of the block before this chunk
#pragma unroll 1
    for (int k = 0; k < kSelPer; ++k) {
        const long long i = (long long)blockIdx.x * kSelItems + k * kSelThreads + threadIdx.x;
        int layer = -2;
        if (i < n) layer = layer_of(g, xyz, i);
        const bool m_lo = layer == lo, m_hi = layer == hi;
        const unsigned b_lo = __ballot_sync(0xffffffffu, m_lo), b_hi = __ballot_sync(0xffffffffu, m_hi);
        if (lane == 0) {
            s_lo[warp] = __popc(b_lo);
            s_hi[warp] = __popc(b_hi);
        }
        __syncthreads();
        int w_lo = 0, w_hi = 0, t_lo = 0, t_hi = 0;
#pragma unroll
        for (int w = 0; w < kSelWarps; ++w) {
            if (w < warp) {
                w_lo += s_lo[w];
                w_hi += s_hi[w];
            }
            t_lo += s_lo[w];
            t_hi += s_hi[w];
        }
        if (m_lo) {
            const long long o = run_lo + w_lo + __popc(b_lo & lanemask_lt());
            out_lo[3 * o + 0] = __ldg(&xyz[3 * i + 0]);
            out_lo[3 * o + 1] = __ldg(&xyz[3 * i + 1]);
            out_lo[3 * o + 2] = __ldg(&xyz[3 * i + 2]);
        }
        if (m_hi) {
            const long long o = run_hi + w_hi + __popc(b_hi & lanemask_lt());
            out_hi[3 * o + 0] = __ldg(&xyz[3 * i + 0]);
            out_hi[3 * o + 1] = __ldg(&xyz[3 * i + 1]);
            out_hi[3 * o + 2] = __ldg(&xyz[3 * i + 2]);
        }
        run_lo += t_lo;
        run_hi += t_hi;
        __syncthreads();  // s_lo / s_hi are rewritten by the next chunk
    }
}

}  // namespace ljc

using namespace ljc;

extern "C" lj_status lj_select_layers(lj_ctx* ctx, const lj_grid* g, int n, const float* xyz, int layer_lo,
                                      int layer_hi, float* out_lo, float* out_hi, int* counts) {
    const NvtxRange nvtx_range("lj_select_layers");
    if (!ctx || !g || n < 0 || !counts || (n > 0 && !xyz)) return LJ_EINVAL;
    if (!(g->width > 0.0f) || g->dim[0] < 1 || g->dim[1] < 1 || g->dim[2] < 1) return LJ_EINVAL;
    if ((layer_lo >= 0 && !out_lo) || (layer_hi >= 0 && !out_hi)) return LJ_EINVAL;
    if (n == 0) return cudaMemsetAsync(counts, 0, 2 * sizeof(int), ctx->stream) == cudaSuccess ? LJ_OK : LJ_ECUDA;
    const int nb = (int)(((long long)n + kSelItems - 1) / kSelItems);
    const size_t need = (size_t)nb * sizeof(int2);
    if (need > ctx->sel_bytes) {
        lj_status s = grow(&ctx->sel, &ctx->sel_bytes, need);
        if (s != LJ_OK) return s;
    }
    int2* bc = static_cast<int2*>(ctx->sel);
    // a layer below 0 matches no particle (axis_cell returns 0 .. gz - 1)
    const int lo = layer_lo >= 0 ? layer_lo : -3, hi = layer_hi >= 0 ? layer_hi : -3;
    const GridDev gd = to_dev(*g);
    k_sel_count<<<nb, kSelThreads, 0, ctx->stream>>>(gd, xyz, n, lo, hi, bc);
    lj_status s = last_launch_status();
    if (s != LJ_OK) return s;
    k_sel_scan<<<1, 1024, 0, ctx->stream>>>(bc, nb, counts);
    if ((s = last_launch_status()) != LJ_OK) return s;
    k_sel_write<<<nb, kSelThreads, 0, ctx->stream>>>(gd, xyz, n, lo, hi, bc, out_lo, out_hi);
    return last_launch_status();
}
