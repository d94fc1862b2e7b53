// ljcell_internal.cuh -- device-side shared definitions of the B200 cell-grid path.
#pragma once

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>
#include <stdint.h>

#include "ljcell.h"

namespace ljc {

// An NVTX range around one C-ABI call: the stages of a step show up by name on a profiler's
// timeline (header-only NVTX 3: without a tool attached the calls do nothing).
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};

// Bits of the context's device status word (the kernels OR them in).
enum : unsigned {
    kFlagNonFinite = 1u << 0,  // a coordinate was NaN or Inf
    kFlagTimeout = 1u << 1,    // a bounded spin-wait gave up
    kFlagRange = 1u << 2,      // an index fell outside its buffer (defensive check)
    kFlagCheck = 1u << 3,      // a consistency check of the -DLJ_CHECKS build failed
};

// Grid passed by value to kernels.
struct GridDev {
    float ox, oy, oz, w;
    int gx, gy, gz;
};

inline GridDev to_dev(const lj_grid& g) {
    GridDev d;
    d.ox = g.origin[0];
    d.oy = g.origin[1];
    d.oz = g.origin[2];
    d.w = g.width;
    d.gx = g.dim[0];
    d.gy = g.dim[1];
    d.gz = g.dim[2];
    return d;
}

// Cell coordinate along one axis: int((x - o) / w) with IEEE subtraction and
// division (PosToCellCoord, cudaLJ.cu:110-119), clamped to [0, g-1]; NaN and
// negative quotients land in cell 0.
__device__ __forceinline__ int axis_cell(float x, float o, float w, int g) {
    const float q = __fdiv_rn(__fsub_rn(x, o), w);
    if (q >= (float)g) return g - 1;
    if (q > 0.0f) return __float2int_rz(q);
    return 0;
}

__device__ __forceinline__ int cell_of(const GridDev& g, float x, float y, float z) {
    const int cx = axis_cell(x, g.ox, g.w, g.gx);
    const int cy = axis_cell(y, g.oy, g.w, g.gy);
    const int cz = axis_cell(z, g.oz, g.w, g.gz);
    return (cz * g.gy + cy) * g.gx + cx;
}

__device__ __forceinline__ unsigned lane_id() { return threadIdx.x & 31u; }

__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Approximate reciprocal (PTX rcp.approx.ftz.f32, at most 1 ulp error).
__device__ __forceinline__ float rcp_approx(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// r^-2 of a candidate pair, or an exact 0 when it does not interact (rcp.approx.ftz(+inf) = +0):
// one reciprocal on every lane, with no branch around it.
__device__ __forceinline__ float rcp_hit(bool hit, float r2) {
    return rcp_approx(hit ? r2 : __int_as_float(0x7f800000));
}

// Warp sums.
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ unsigned long long warp_sum(unsigned long long v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

}  // namespace ljc

// Device buffer sets of the queued host-buffer steps.  Three, so that a step's upload never waits
// for a download: with two, the upload of step k + 1 waits for the download of step k - 1, and a
// step whose results go down only after its whole pair stage (the input-order entry) then sets a
// period of (upload + compute + download) / 2 instead of the slowest of the three.
constexpr int kE2EASlots = 3;

// Opaque context (host side).
struct lj_ctx {
    int device;
    cudaStream_t stream;
    int sm_count;
    unsigned* d_status;          // device status word
    // scratch, grown on demand
    void* scan_state;            // tile counter + tile status words
    size_t scan_state_bytes;
    int2* cell_ticket;           // per particle: cell id, ticket
    float4* tmp4;                // scatter target before the within-cell sort
    size_t part_cap;             // capacity (particles) of cell_ticket / tmp4
    int* large_cells;            // [0] = count, [1..] = ids of cells too large for the warp sort
    size_t large_cap;
    void* red;                   // reduction partials + counter
    size_t red_bytes;
    unsigned long long* d_cand;  // candidate-count accumulator
    lj_tuning tuning;            // implementation choices (lj_set_tuning)
    void* reorder;               // lj_reorder: key counts, offsets, sorted records and their keys
    size_t reorder_bytes;
    void* step;                  // lj_step_verlet: moved positions, half-kicked velocities, ids
    size_t step_bytes;
    void* half;                  // lj_compute_half: raw per-particle sums and the pair counter
    size_t half_bytes;
    void* sel;                   // lj_select_layers: per-block counts, then offsets
    size_t sel_bytes;
    void* check;                 // -DLJ_CHECKS build: per-particle marks of the permutation check
    size_t check_bytes;
    void* cellpair;              // pair kernel 12: pair-opening flags, their exclusive scan, the pair list
    size_t cellpair_bytes;
    // end-to-end buffers (lj_simulate_host): device buffers, a second stream for the device-to-host
    // copies and the events that order it after the pair chunks
    void* e2e;
    size_t e2e_bytes;
    cudaStream_t copy_stream;
    cudaEvent_t e2e_ev[8];
    bool e2e_ready;
    // pipelined host-buffer steps (lj_simulate_host_async): kE2EASlots device buffer sets used in
    // turn, an upload stream, and events: [0, S) slot free (its last download done), then at S + 0
    // upload done, S + 1 binning done, S + 2 .. S + 5 pair chunks done, S + 6 totals done
    void* e2ea[kE2EASlots];
    size_t e2ea_bytes[kE2EASlots];
    int e2ea_slot;
    cudaStream_t up_stream;
    cudaEvent_t e2ea_ev[kE2EASlots + 7];
    bool e2ea_ready;
    lj_totals* e2ea_tot;         // pinned staging of the queued calls' totals (kE2EAPending entries)
    lj_totals* e2ea_dst[64];     // caller's totals pointer of each queued call
    int e2ea_pending;
};

namespace ljc {
// Blocks for a grid-stride loop over `items`: enough for every item, at most `waves` per SM.
inline int grid_for(const lj_ctx* ctx, long long items, int per_block, int waves = 8) {
    long long b = (items + per_block - 1) / per_block;
    const long long cap = (long long)ctx->sm_count * waves;
    if (b > cap) b = cap;
    return (int)(b < 1 ? 1 : b);
}
}  // namespace ljc


namespace ljc {
// Host helpers shared by the .cu files (defined in api.cu).
lj_status grow(void** p, size_t* cap, size_t need);
lj_status last_launch_status();
// Cell-grid build stages (bin.cu), shared by lj_bin and the batched step.
lj_status bin_prepare(lj_ctx* ctx, int n, long long nc, int* counts);
// The within-cell sort recomputes each record's cell: from grid g when nsys == 0, else from the
// system table (sys[s] for the last s with firsts[s] <= the record's original index).
struct BinSys {
    GridDev g;
    int cell_base;
    int first;
};
lj_status bin_finish(lj_ctx* ctx, long long nc, int n, const float* x, const float* y, const float* z, int stride,
                     lj_order order, int* counts, int* offsets, lj_cell_desc* cells, lj_particles* sorted,
                     float* sorted_xyzi, int* sorted_cell, const GridDev& g, const BinSys* sys, const int* firsts,
                     int nsys);
// Default pair kernel (lj_tuning numbering) for n particles binned in g with LJ_ORDER_X (pair.cu).
int default_pair_kernel(int n, const lj_grid& g);
// Pair stage of lj_compute over the sorted targets [kb, ke) (pair.cu); totals cover those targets only.
// by_index: each target's energy and force go to its original index instead of its sorted position.
lj_status launch_pair_config(lj_ctx* ctx, const lj_grid* g, const lj_params* prm, int n, const float* xyzi,
                             const int* cs, const int* off, lj_order order, float* energy, float* force,
                             lj_totals* totals, int kb, int ke, bool by_index = false);
}  // namespace ljc
