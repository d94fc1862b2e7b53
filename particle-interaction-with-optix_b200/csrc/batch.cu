// batch.cu -- many independent systems in one step.
//
// The systems' particles sit back to back; system s owns particles
// [first_s, first_s + n_s) and cells [cell_base_s, cell_base_s + ncells_s) of a
// shared cell numbering.  Binning is the single-system build (bin.cu) with a
// count kernel that picks each particle's system and grid, so one launch per
// stage bins every system, and each system's sorted particles land in its own
// range [first_s, first_s + n_s).  The pair kernel is persistent: CTAs take
// (system, block of consecutive sorted targets) tiles from a device work
// queue, largest estimated cost first, and evaluate each target with the same
// per-target routine as the single-system kernel (pair_target), so per-target
// results equal a per-system run bit for bit.  Per-system totals are reduced
// from per-target values in a fixed order (deterministic).  The whole step can
// be captured once in a CUDA graph and replayed.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "pair_pass.cuh"

namespace ljc {

struct SysDev {
    GridDev g;
    PairParams pp;
    int cell_base;
    int first;
    int n;
    int walk;  // 1: one target per lane (kernel 6's walk), 3: two targets per lane (kernel 10's), as the
               // single-system default chooses for the system
};

// ---------------------------------------------------------------- count
// As k_count (bin.cu), with the system of particle i found by binary search
// over the systems' first indices: the last s with firsts[s] <= i (empty
// systems share their first with the next one and are skipped that way).
__global__ void __launch_bounds__(256) k_count_batched(const SysDev* __restrict__ sys,
                                                       const int* __restrict__ firsts, int nsys,
                                                       const float* __restrict__ x, const float* __restrict__ y,
                                                       const float* __restrict__ z, int n, int* __restrict__ counts,
                                                       int2* __restrict__ ct, unsigned* status) {
    const int lane = threadIdx.x & 31;
    const long long gwarp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long base = gwarp * 32; base < n; base += nwarps * 32) {
        const long long i = base + lane;
        const bool valid = i < n;
        int cell = -1 - lane;
        if (valid) {
            int lo = 0, hi = nsys - 1;
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (__ldg(&firsts[mid]) <= (int)i)
                    lo = mid;
                else
                    hi = mid - 1;
            }
            const GridDev g = sys[lo].g;
            const int cb = sys[lo].cell_base;
            const float px = x[i], py = y[i], pz = z[i];
            if (!(isfinite(px) && isfinite(py) && isfinite(pz))) atomicOr(status, kFlagNonFinite);
            cell = cb + cell_of(g, px, py, pz);
        }
        const unsigned peers = __match_any_sync(0xffffffffu, cell);
        const int leader = __ffs(peers) - 1;
        int first = 0;
        if (valid && lane == leader) first = atomicAdd(&counts[cell], __popc(peers));
        first = __shfl_sync(0xffffffffu, first, leader);
        if (valid) ct[i] = make_int2(cell, first + __popc(peers & lanemask_lt()));
    }
}

// ---------------------------------------------------------------- pair (persistent, tile queue)
// Tile = (system, k0, k1): targets [k0, k1) of one system, at most
// BLOCK * PPT of them (2 * BLOCK * PPT for MODE 3).  Each target runs the
// per-target routine of the single-system kernel the default picks for the
// system (MODE 1: pass_target, one target per lane, as kernel 6; MODE 3:
// pass_target2, two targets per lane, as kernel 10), in the system's local
// indices, so per-particle results equal a per-system lj_compute with that
// kernel bit for bit.  One launch per walk mode, over the tiles of the systems
// using it.  Per-target raw sums go to te / tw / tnp for the per-system totals.
template <int BLOCK, int PPT, int MODE>
__global__ void __launch_bounds__(BLOCK) k_pair_batched(const SysDev* __restrict__ sys, const float4* __restrict__ p,
                                                        const int* __restrict__ cs, const int* __restrict__ off,
                                                        const int4* __restrict__ tiles, int ntiles,
                                                        unsigned* tile_counter, float* __restrict__ energy,
                                                        float* __restrict__ force, float* __restrict__ te,
                                                        float* __restrict__ tw, unsigned* __restrict__ tnp,
                                                        unsigned* status) {
    __shared__ int s_t;
    while (true) {
        if (threadIdx.x == 0) s_t = (int)atomicAdd(tile_counter, 1u);
        __syncthreads();
        const int t = s_t;
        if (t >= ntiles) break;
        const int4 d = __ldg(&tiles[t]);
        const SysDev S = sys[d.x];
        const int ncell = S.g.gx * S.g.gy * S.g.gz;
        const float4* ps = p + S.first;
        if (MODE == 3) {
            // two targets per thread (pass_target2): a = k, b = k + 1, windows parked in shared memory
            __shared__ int2 s_win[9][BLOCK];
#pragma unroll
            for (int r = 0; r < PPT; ++r) {
                const int k = d.y + 2 * (r * BLOCK + threadIdx.x);
                const bool activeA = k < d.z, activeB = k + 1 < d.z;
                int ca = 0, cb = 0;
                if (activeA) {
                    ca = __ldg(&cs[k]) - S.cell_base;
                    if (ca < 0 || ca >= ncell) {
                        atomicOr(status, kFlagRange);
                        ca = 0;
                    }
                }
                if (activeB) {
                    cb = __ldg(&cs[k + 1]) - S.cell_base;
                    if (cb < 0 || cb >= ncell) {
                        atomicOr(status, kFlagRange);
                        cb = 0;
                    }
                }
                Pass2Acc a;
                pass_target2<BLOCK>(S.g, S.pp, ps, off + S.cell_base, S.first, S.n, k - S.first, ca, cb, activeA,
                                    activeB, a, s_win);
                const float nf = -S.pp.fscale;
                if (activeA) {
                    if (energy) energy[k] = S.pp.e4 * a.e.x;
                    if (force) {
                        force[3 * (size_t)k + 0] = nf * a.fx.x;
                        force[3 * (size_t)k + 1] = nf * a.fy.x;
                        force[3 * (size_t)k + 2] = nf * a.fz.x;
                    }
                    te[k] = a.e.x;
                    tw[k] = a.w.x;
                    tnp[k] = a.np;  // both targets' pairs: the per-system totals only need their sum
                }
                if (activeB) {
                    if (energy) energy[k + 1] = S.pp.e4 * a.e.y;
                    if (force) {
                        force[3 * (size_t)k + 3] = nf * a.fx.y;
                        force[3 * (size_t)k + 4] = nf * a.fy.y;
                        force[3 * (size_t)k + 5] = nf * a.fz.y;
                    }
                    te[k + 1] = a.e.y;
                    tw[k + 1] = a.w.y;
                    tnp[k + 1] = 0u;
                }
            }
            __syncthreads();  // s_t is reused by the next tile
            continue;
        }
#pragma unroll
        for (int r = 0; r < PPT; ++r) {
            const int k = d.y + r * BLOCK + threadIdx.x;
            const bool active = k < d.z;
            int c = 0;
            if (active) {
                c = __ldg(&cs[k]) - S.cell_base;
                if (c < 0 || c >= ncell) {
                    atomicOr(status, kFlagRange);
                    c = 0;
                }
            }
            PassAcc a;
            pass_target(S.g, S.pp, ps, off + S.cell_base, S.first, S.n, k - S.first, c, active, a);
            if (active) {
                const float ea = a.e.x + a.e.y;
                if (energy) energy[k] = S.pp.e4 * ea;
                if (force) {
                    const float nf = -S.pp.fscale;
                    force[3 * (size_t)k + 0] = nf * (a.fx.x + a.fx.y);
                    force[3 * (size_t)k + 1] = nf * (a.fy.x + a.fy.y);
                    force[3 * (size_t)k + 2] = nf * (a.fz.x + a.fz.y);
                }
                te[k] = ea;
                tw[k] = a.w.x + a.w.y;
                tnp[k] = a.np;
            }
        }
        __syncthreads();  // s_t is reused by the next tile
    }
}


// One block per system: totals from the per-target sums, in index order.
__global__ void __launch_bounds__(256) k_sys_totals(const SysDev* __restrict__ sys, const float* __restrict__ te,
                                                    const float* __restrict__ tw, const unsigned* __restrict__ tnp,
                                                    lj_totals* __restrict__ totals) {
    __shared__ double s_e[8], s_w[8];
    __shared__ unsigned long long s_p[8];
    const SysDev S = sys[blockIdx.x];
    double e = 0.0, w = 0.0;
    unsigned long long np = 0;
    for (int k = S.first + threadIdx.x; k < S.first + S.n; k += blockDim.x) {
        e += 0.5 * (double)S.pp.e4 * (double)te[k];
        w += 0.5 * (double)S.pp.e24 * (double)tw[k];
        np += tnp[k];
    }
    e = warp_sum(e);
    w = warp_sum(w);
    np = warp_sum(np);
    const int warp = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
        s_e[warp] = e;
        s_w[warp] = w;
        s_p[warp] = np;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double fe = 0.0, fw = 0.0;
        unsigned long long fp = 0;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) {
            fe += s_e[i];
            fw += s_w[i];
            fp += s_p[i];
        }
        totals[blockIdx.x] = lj_totals{fe, fw, fp, 0ULL};
    }
}

// Adds `delta` to n ints (batch-wide indices for the per-system path).
__global__ void k_add_offset(int* __restrict__ v, int n, int delta) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) v[i] += delta;
}

}  // namespace ljc

// ---------------------------------------------------------------- plan (host)
struct lj_batch {
    int device = 0;
    int nsys = 0;
    int ntotal = 0;
    lj_batch_config cfg{};
    unsigned version = 0;  // bumped when the plan changes (graph key)
    std::vector<lj_system> sys;
    std::vector<ljc::SysDev> sd;
    std::vector<lj_grid> grids;
    long long total_cells = 0;
    ljc::SysDev* d_sys = nullptr;
    ljc::BinSys* d_binsys = nullptr;  // grids and cell bases for the within-cell sort
    int* d_firsts = nullptr;
    int4* d_tiles = nullptr;
    int ntiles = 0;
    int ntiles1 = 0;  // tiles [0, ntiles1) use walk mode 1, the rest mode 3
    size_t tiles_cap = 0;
    unsigned* d_counter = nullptr;
    int* counts = nullptr;
    int* offsets = nullptr;
    size_t cells_cap = 0;
    float4* xyzi = nullptr;
    int* cell = nullptr;
    float* te = nullptr;
    float* tw = nullptr;
    unsigned* tnp = nullptr;
    int persistent_blocks[3] = {0, 0, 0};  // grid of the persistent pair kernel per walk mode
    // graph replay
    cudaStream_t gstream = nullptr;
    cudaEvent_t ev_in = nullptr, ev_out = nullptr;
    cudaGraphExec_t exec = nullptr;
    const void* gkey[7] = {};
    unsigned gversion = ~0u;
};

namespace ljc {

static void free_plan_buffers(lj_batch* b) {
    cudaFree(b->d_sys);
    cudaFree(b->d_binsys);
    cudaFree(b->d_firsts);
    cudaFree(b->d_tiles);
    cudaFree(b->d_counter);
    cudaFree(b->counts);
    cudaFree(b->offsets);
    cudaFree(b->xyzi);
    cudaFree(b->cell);
    cudaFree(b->te);
    cudaFree(b->tw);
    cudaFree(b->tnp);
    b->d_sys = nullptr;
    b->d_binsys = nullptr;
    b->d_firsts = nullptr;
    b->d_tiles = nullptr;
    b->d_counter = nullptr;
    b->counts = b->offsets = nullptr;
    b->xyzi = nullptr;
    b->cell = nullptr;
    b->te = b->tw = nullptr;
    b->tnp = nullptr;
    b->tiles_cap = b->cells_cap = 0;
}

static bool valid_config(const lj_batch_config& c) {
    return c.cell_multiple >= 1.0f && c.cell_multiple <= 8.0f &&
           (c.threads == 64 || c.threads == 128 || c.threads == 256) && (c.per_thread == 1 || c.per_thread == 2);
}

// Grids, cell numbering and system table for the cell multiple of cfg.
static lj_status build_grids(lj_batch* b) {
    b->grids.resize(b->nsys);
    b->sd.resize(b->nsys);
    long long base = 0;
    for (int s = 0; s < b->nsys; ++s) {
        const lj_system& y = b->sys[s];
        const float w = y.params.cutoff * b->cfg.cell_multiple;
        lj_status st = lj_grid_from_box(y.lo, y.hi, w, &b->grids[s]);
        if (st != LJ_OK) return st;
        const lj_grid& g = b->grids[s];
        SysDev& d = b->sd[s];
        d.g = to_dev(g);
        d.pp.rc2 = y.params.cutoff * y.params.cutoff;
        d.pp.rc2w = d.pp.rc2 * (1.0f + 1e-5f);
        d.pp.sig2 = y.params.sigma * y.params.sigma;
        d.pp.e4 = 4.0f * y.params.epsilon;
        d.pp.e24 = 24.0f * y.params.epsilon;
        d.pp.fscale = -d.pp.e24 / d.pp.sig2;
        d.pp.slack = grid_slack(g);
        d.cell_base = (int)base;
        d.first = y.first;
        d.n = y.n;
        // the two-target walk where the single-system default takes kernel 10, else one target per
        // lane (kernel 6's walk; the persistent tile queue has no pair list for kernel 12)
        d.walk = default_pair_kernel(y.n, g) == 10 ? 3 : 1;
        base += (long long)g.dim[0] * g.dim[1] * g.dim[2];
        if (base > 2147483646LL) return LJ_EUNSUPPORTED;
    }
    b->total_cells = base;
    return LJ_OK;
}

// Tiles of T = threads * per_thread consecutive targets per system (2T for systems on the two-target
// walk): first those of the systems walked with mode 1, then mode 3, each group ordered by estimated
// cost (targets x expected candidates: n / box volume x cutoff^3), largest first.
static std::vector<int4> build_tiles(const lj_batch* b) {
    const int T = b->cfg.threads * b->cfg.per_thread;
    std::vector<std::pair<double, int4>> v;
    for (int s = 0; s < b->nsys; ++s) {
        const lj_system& y = b->sys[s];
        double vol = 1.0;
        for (int d = 0; d < 3; ++d) vol *= (double)y.hi[d] - (double)y.lo[d];
        const double rc = y.params.cutoff;
        const double per_target = (double)y.n / (vol > 0 ? vol : 1.0) * rc * rc * rc;
        const int Ts = b->sd[s].walk == 3 ? 2 * T : T;  // the two-target walk takes 2 targets per thread
        for (int k0 = 0; k0 < y.n; k0 += Ts) {
            const int k1 = std::min(y.n, k0 + Ts);
            v.push_back({per_target * (k1 - k0), make_int4(s, y.first + k0, y.first + k1, 0)});
        }
    }
    std::stable_sort(v.begin(), v.end(), [b](const auto& a, const auto& c) {
        const int wa = b->sd[a.second.x].walk, wc = b->sd[c.second.x].walk;
        return wa != wc ? wa < wc : a.first > c.first;
    });
    std::vector<int4> out;
    out.reserve(v.size());
    for (auto& e : v) out.push_back(e.second);
    return out;
}

static int count_tiles_below(const lj_batch* b, const std::vector<int4>& tiles, int walk) {
    int m = 0;
    while (m < (int)tiles.size() && b->sd[tiles[m].x].walk < walk) ++m;
    return m;
}

template <class T>
static lj_status dev_alloc(T** p, size_t count) {
    if (cudaMalloc(reinterpret_cast<void**>(p), sizeof(T) * (count > 0 ? count : 1)) != cudaSuccess) {
        cudaGetLastError();
        *p = nullptr;
        return LJ_ENOMEM;
    }
    return LJ_OK;
}

static int batched_occupancy(int threads, int ppt, int mode);

// (Re)builds the device side of the plan for b->cfg.  Synchronous.
static lj_status build_plan(lj_ctx* ctx, lj_batch* b) {
    lj_status st = build_grids(b);
    if (st != LJ_OK) return st;
    const std::vector<int4> tiles = build_tiles(b);
    const size_t N = (size_t)(b->ntotal > 0 ? b->ntotal : 1);
    if (!b->xyzi) {
        if ((st = dev_alloc(&b->xyzi, N)) != LJ_OK || (st = dev_alloc(&b->cell, N)) != LJ_OK ||
            (st = dev_alloc(&b->te, N)) != LJ_OK || (st = dev_alloc(&b->tw, N)) != LJ_OK ||
            (st = dev_alloc(&b->tnp, N)) != LJ_OK || (st = dev_alloc(&b->d_sys, (size_t)b->nsys)) != LJ_OK ||
            (st = dev_alloc(&b->d_firsts, (size_t)b->nsys)) != LJ_OK ||
            (st = dev_alloc(&b->d_binsys, (size_t)b->nsys)) != LJ_OK ||
            (st = dev_alloc(&b->d_counter, (size_t)64)) != LJ_OK)
            return st;
    }
    if ((size_t)b->total_cells + 1 > b->cells_cap) {
        cudaFree(b->counts);
        cudaFree(b->offsets);
        b->counts = b->offsets = nullptr;
        const size_t cap = (size_t)b->total_cells + 1;
        if ((st = dev_alloc(&b->counts, cap)) != LJ_OK || (st = dev_alloc(&b->offsets, cap)) != LJ_OK) return st;
        b->cells_cap = cap;
    }
    if (tiles.size() > b->tiles_cap) {
        cudaFree(b->d_tiles);
        b->d_tiles = nullptr;
        if ((st = dev_alloc(&b->d_tiles, tiles.size())) != LJ_OK) return st;
        b->tiles_cap = tiles.size();
    }
    std::vector<int> firsts(b->nsys);
    std::vector<BinSys> binsys(b->nsys);
    for (int s = 0; s < b->nsys; ++s) {
        firsts[s] = b->sys[s].first;
        binsys[s] = BinSys{b->sd[s].g, b->sd[s].cell_base, b->sd[s].first};
    }
    if (cudaMemcpy(b->d_sys, b->sd.data(), sizeof(SysDev) * b->nsys, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(b->d_firsts, firsts.data(), sizeof(int) * b->nsys, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(b->d_binsys, binsys.data(), sizeof(BinSys) * b->nsys, cudaMemcpyHostToDevice) != cudaSuccess ||
        (!tiles.empty() && cudaMemcpy(b->d_tiles, tiles.data(), sizeof(int4) * tiles.size(),
                                      cudaMemcpyHostToDevice) != cudaSuccess))
        return LJ_ECUDA;
    b->ntiles = (int)tiles.size();
    b->ntiles1 = count_tiles_below(b, tiles, 3);
    b->persistent_blocks[0] = ctx->sm_count * batched_occupancy(b->cfg.threads, b->cfg.per_thread, 1);
    b->persistent_blocks[2] = ctx->sm_count * batched_occupancy(b->cfg.threads, b->cfg.per_thread, 3);
    ++b->version;
    return LJ_OK;
}

}  // namespace ljc

namespace ljc {

template <int BLOCK, int PPT, int MODE>
static int occ_of() {
    int per = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_pair_batched<BLOCK, PPT, MODE>, BLOCK, 0) !=
            cudaSuccess ||
        per < 1) {
        cudaGetLastError();
        per = 1;
    }
    return per;
}

template <int MODE>
static int occ_mode(int threads, int ppt) {
    if (threads == 64) return ppt == 1 ? occ_of<64, 1, MODE>() : occ_of<64, 2, MODE>();
    if (threads == 256) return ppt == 1 ? occ_of<256, 1, MODE>() : occ_of<256, 2, MODE>();
    return ppt == 1 ? occ_of<128, 1, MODE>() : occ_of<128, 2, MODE>();
}

static int batched_occupancy(int threads, int ppt, int mode) {
    return mode == 3 ? occ_mode<3>(threads, ppt) : occ_mode<1>(threads, ppt);
}

// Tiles [t0, t1) with walk MODE; the persistent grid never exceeds the tile count.
template <int BLOCK, int PPT, int MODE>
static void launch_batched_mode(lj_ctx* ctx, lj_batch* b, const float* p4, float* energy, float* force, int t0,
                                int t1) {
    if (t1 <= t0) return;
    const int grid = std::min(b->persistent_blocks[MODE - 1], t1 - t0);
    k_pair_batched<BLOCK, PPT, MODE><<<grid, BLOCK, 0, ctx->stream>>>(
        b->d_sys, reinterpret_cast<const float4*>(p4), b->cell, b->offsets, b->d_tiles + t0,
        t1 - t0, b->d_counter + (MODE - 1), energy, force, b->te, b->tw, b->tnp, ctx->d_status);
}

template <int BLOCK, int PPT>
static void launch_batched_pair(lj_ctx* ctx, lj_batch* b, const float* p4, float* energy, float* force) {
    launch_batched_mode<BLOCK, PPT, 3>(ctx, b, p4, energy, force, b->ntiles1, b->ntiles);
    launch_batched_mode<BLOCK, PPT, 1>(ctx, b, p4, energy, force, 0, b->ntiles1);
}

// The batched step on ctx->stream (no synchronisation, no allocation once the
// context's scratch has grown to the batch size).
static lj_status batch_step(lj_ctx* ctx, lj_batch* b, const float* x, const float* y, const float* z, float* energy,
                            float* force, int* index, lj_totals* totals) {
    lj_status st;
    const int n = b->ntotal;
    cudaStream_t s = ctx->stream;
    if ((st = bin_prepare(ctx, n, b->total_cells, b->counts)) != LJ_OK) return st;
    if (n > 0) {
        long long blocks = ((long long)n + 255) / 256;
        if (blocks > (long long)ctx->sm_count * 8) blocks = (long long)ctx->sm_count * 8;
        k_count_batched<<<(int)blocks, 256, 0, s>>>(b->d_sys, b->d_firsts, b->nsys, x, y, z, n, b->counts,
                                                    ctx->cell_ticket, ctx->d_status);
        if ((st = last_launch_status()) != LJ_OK) return st;
    }
    lj_particles sorted{};
    sorted.index = index;
    float* xyzi = reinterpret_cast<float*>(b->xyzi);
    if ((st = bin_finish(ctx, b->total_cells, n, x, y, z, 1, LJ_ORDER_X, b->counts, b->offsets, nullptr,
                         index ? &sorted : nullptr, xyzi, b->cell, GridDev{}, b->d_binsys, b->d_firsts, b->nsys)) !=
        LJ_OK)
        return st;
    if (cudaMemsetAsync(b->d_counter, 0, 3 * sizeof(unsigned), s) != cudaSuccess) return LJ_ECUDA;
    const int T = b->cfg.threads, P = b->cfg.per_thread;
    if (T == 64)
        P == 1 ? launch_batched_pair<64, 1>(ctx, b, xyzi, energy, force)
               : launch_batched_pair<64, 2>(ctx, b, xyzi, energy, force);
    else if (T == 256)
        P == 1 ? launch_batched_pair<256, 1>(ctx, b, xyzi, energy, force)
               : launch_batched_pair<256, 2>(ctx, b, xyzi, energy, force);
    else
        P == 1 ? launch_batched_pair<128, 1>(ctx, b, xyzi, energy, force)
               : launch_batched_pair<128, 2>(ctx, b, xyzi, energy, force);
    if ((st = last_launch_status()) != LJ_OK) return st;
    if (totals) {
        k_sys_totals<<<b->nsys, 256, 0, s>>>(b->d_sys, b->te, b->tw, b->tnp, totals);
        if ((st = last_launch_status()) != LJ_OK) return st;
    }
    return LJ_OK;
}

static lj_status batch_graph(lj_ctx* ctx, lj_batch* b, const float* x, const float* y, const float* z, float* energy,
                             float* force, int* index, lj_totals* totals) {
    const void* key[7] = {x, y, z, energy, force, index, totals};
    if (!b->gstream) {
        if (cudaStreamCreateWithFlags(&b->gstream, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&b->ev_in, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&b->ev_out, cudaEventDisableTiming) != cudaSuccess)
            return LJ_ECUDA;
    }
    if (!b->exec || b->gversion != b->version || std::memcmp(key, b->gkey, sizeof(key)) != 0) {
        if (b->exec) {
            cudaGraphExecDestroy(b->exec);
            b->exec = nullptr;
        }
        // one plain run sizes the context's scratch, so nothing allocates while capturing
        lj_status st = batch_step(ctx, b, x, y, z, energy, force, index, totals);
        if (st != LJ_OK) return st;
        if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) return LJ_ECUDA;
        cudaStream_t saved = ctx->stream;
        ctx->stream = b->gstream;
        if (cudaStreamBeginCapture(b->gstream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
            ctx->stream = saved;
            return LJ_ECUDA;
        }
        st = batch_step(ctx, b, x, y, z, energy, force, index, totals);
        cudaGraph_t graph = nullptr;
        const cudaError_t ec = cudaStreamEndCapture(b->gstream, &graph);
        ctx->stream = saved;
        if (st != LJ_OK || ec != cudaSuccess) {
            if (graph) cudaGraphDestroy(graph);
            cudaGetLastError();
            return st != LJ_OK ? st : LJ_ECUDA;
        }
        const cudaError_t ei = cudaGraphInstantiate(&b->exec, graph, 0);
        cudaGraphDestroy(graph);
        if (ei != cudaSuccess) {
            b->exec = nullptr;
            return LJ_ECUDA;
        }
        std::memcpy(b->gkey, key, sizeof(key));
        b->gversion = b->version;
    }
    if (cudaEventRecord(b->ev_in, ctx->stream) != cudaSuccess ||
        cudaStreamWaitEvent(b->gstream, b->ev_in, 0) != cudaSuccess ||
        cudaGraphLaunch(b->exec, b->gstream) != cudaSuccess || cudaEventRecord(b->ev_out, b->gstream) != cudaSuccess ||
        cudaStreamWaitEvent(ctx->stream, b->ev_out, 0) != cudaSuccess)
        return LJ_ECUDA;
    return LJ_OK;
}

// One plain lj_bin + lj_compute per system (the path the batched step replaces), each with the
// single-system kernel of the walk the batched kernel takes for it (6: one target per lane, 10: two
// targets per lane), so per-particle results are equal bit for bit.
static lj_status batch_separate_one(lj_ctx* ctx, lj_batch* b, int s, const float* x, const float* y, const float* z,
                                    float* energy, float* force, int* index, lj_totals* totals);

static lj_status batch_separate(lj_ctx* ctx, lj_batch* b, const float* x, const float* y, const float* z,
                                float* energy, float* force, int* index, lj_totals* totals) {
    const lj_tuning saved = ctx->tuning;
    lj_status st = LJ_OK;
    for (int s = 0; s < b->nsys && st == LJ_OK; ++s) {
        ctx->tuning.pair_kernel = b->sd[s].walk == 3 ? 10 : 6;
        st = batch_separate_one(ctx, b, s, x, y, z, energy, force, index, totals);
    }
    ctx->tuning = saved;
    return st;
}

static lj_status batch_separate_one(lj_ctx* ctx, lj_batch* b, int s, const float* x, const float* y, const float* z,
                                    float* energy, float* force, int* index, lj_totals* totals) {
    {
        const lj_system& sy = b->sys[s];
        const SysDev& d = b->sd[s];
        const int f = sy.first;
        int* off_s = b->offsets + d.cell_base;
        lj_particles sorted{};
        sorted.index = index ? index + f : nullptr;
        lj_status st = lj_bin(ctx, &b->grids[s], sy.n, x + f, y + f, z + f, 1, LJ_ORDER_X, b->counts + d.cell_base,
                              off_s, nullptr, index ? &sorted : nullptr, reinterpret_cast<float*>(b->xyzi + f),
                              b->cell + f);
        if (st != LJ_OK) return st;
        if (index && f != 0 && sy.n > 0) {
            k_add_offset<<<(sy.n + 255) / 256, 256, 0, ctx->stream>>>(index + f, sy.n, f);
            if ((st = last_launch_status()) != LJ_OK) return st;
        }
        st = lj_compute(ctx, &b->grids[s], &sy.params, sy.n, reinterpret_cast<const float*>(b->xyzi + f),
                        b->cell + f, off_s, LJ_ORDER_X, energy ? energy + f : nullptr,
                        force ? force + 3 * (size_t)f : nullptr, totals ? totals + s : nullptr);
        if (st != LJ_OK) return st;
    }
    return LJ_OK;
}

}  // namespace ljc

using namespace ljc;

extern "C" lj_status lj_batch_create(lj_ctx* ctx, int nsys, const lj_system* systems, const lj_batch_config* cfg,
                                     lj_batch** out) {
    if (!ctx || !out || nsys < 1 || !systems) return LJ_EINVAL;
    *out = nullptr;
    long long next = 0;
    for (int s = 0; s < nsys; ++s) {
        const lj_system& y = systems[s];
        if (y.n < 0 || y.first != next || !(y.params.cutoff > 0.0f) || !(y.params.sigma > 0.0f)) return LJ_EINVAL;
        next += y.n;
        if (next > 2147483646LL) return LJ_EUNSUPPORTED;
    }
    lj_batch_config c{1.0f, 128, 1, {0, 0, 0, 0, 0}};
    if (cfg) c = *cfg;
    if (!valid_config(c)) return LJ_EINVAL;
    lj_batch* b = new (std::nothrow) lj_batch();
    if (!b) return LJ_ENOMEM;
    b->device = ctx->device;
    b->nsys = nsys;
    b->ntotal = (int)next;
    b->cfg = c;
    b->sys.assign(systems, systems + nsys);
    const lj_status st = build_plan(ctx, b);
    if (st != LJ_OK) {
        free_plan_buffers(b);
        delete b;
        return st;
    }
    *out = b;
    return LJ_OK;
}

extern "C" lj_status lj_batch_destroy(lj_batch* b) {
    if (!b) return LJ_EINVAL;
    if (b->gstream) cudaStreamSynchronize(b->gstream);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->ev_in) cudaEventDestroy(b->ev_in);
    if (b->ev_out) cudaEventDestroy(b->ev_out);
    if (b->gstream) cudaStreamDestroy(b->gstream);
    free_plan_buffers(b);
    delete b;
    return LJ_OK;
}

extern "C" lj_status lj_batch_get_config(const lj_batch* b, lj_batch_config* cfg) {
    if (!b || !cfg) return LJ_EINVAL;
    *cfg = b->cfg;
    return LJ_OK;
}

extern "C" lj_status lj_batch_grid(const lj_batch* b, int s, lj_grid* g) {
    if (!b || !g || s < 0 || s >= b->nsys) return LJ_EINVAL;
    *g = b->grids[s];
    return LJ_OK;
}

static bool batch_args_ok(lj_ctx* ctx, lj_batch* b, const float* x, const float* y, const float* z, float* force) {
    if (!ctx || !b || (b->ntotal > 0 && (!x || !y || !z))) return false;
    return true;
}

extern "C" lj_status lj_batch_run(lj_ctx* ctx, lj_batch* b, const float* x, const float* y, const float* z,
                                  float* energy, float* force, int* index, lj_totals* totals) {
    const NvtxRange nvtx_range("lj_batch_run");
    if (!batch_args_ok(ctx, b, x, y, z, force)) return LJ_EINVAL;
    return batch_step(ctx, b, x, y, z, energy, force, index, totals);
}

extern "C" lj_status lj_batch_run_graph(lj_ctx* ctx, lj_batch* b, const float* x, const float* y, const float* z,
                                        float* energy, float* force, int* index, lj_totals* totals) {
    const NvtxRange nvtx_range("lj_batch_run_graph");
    if (!batch_args_ok(ctx, b, x, y, z, force)) return LJ_EINVAL;
    return batch_graph(ctx, b, x, y, z, energy, force, index, totals);
}

extern "C" lj_status lj_batch_run_separate(lj_ctx* ctx, lj_batch* b, const float* x, const float* y, const float* z,
                                           float* energy, float* force, int* index, lj_totals* totals) {
    const NvtxRange nvtx_range("lj_batch_run_separate");
    if (!batch_args_ok(ctx, b, x, y, z, force)) return LJ_EINVAL;
    return batch_separate(ctx, b, x, y, z, energy, force, index, totals);
}

extern "C" lj_status lj_batch_autotune(lj_ctx* ctx, lj_batch* b, const float* x, const float* y, const float* z,
                                       lj_batch_config* best, float* best_ms) {
    if (!batch_args_ok(ctx, b, x, y, z, nullptr)) return LJ_EINVAL;
    const float multiples[3] = {1.0f, 1.5f, 2.0f};
    const int shapes[3] = {64, 128, 256};
    const int ppts[2] = {1, 2};
    cudaEvent_t e0, e1;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) return LJ_ECUDA;
    lj_batch_config bestc = b->cfg;
    float bestt = 3.4e38f;
    lj_status st = LJ_OK;
    for (float m : multiples) {
        for (int t : shapes) {
            for (int p : ppts) {
                b->cfg.cell_multiple = m;
                b->cfg.threads = t;
                b->cfg.per_thread = p;
                if ((st = build_plan(ctx, b)) != LJ_OK) break;
                // graph replays of the step without the optional outputs
                if ((st = batch_graph(ctx, b, x, y, z, nullptr, nullptr, nullptr, nullptr)) != LJ_OK) break;
                if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) {
                    st = LJ_ECUDA;
                    break;
                }
                float ms = 3.4e38f;
                for (int r = 0; r < 3; ++r) {
                    float one = 0.f;
                    if (cudaEventRecord(e0, ctx->stream) != cudaSuccess ||
                        (st = batch_graph(ctx, b, x, y, z, nullptr, nullptr, nullptr, nullptr)) != LJ_OK ||
                        cudaEventRecord(e1, ctx->stream) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
                        cudaEventElapsedTime(&one, e0, e1) != cudaSuccess) {
                        if (st == LJ_OK) st = LJ_ECUDA;
                        break;
                    }
                    ms = one < ms ? one : ms;
                }
                if (st != LJ_OK) break;
                if (ms < bestt) {
                    bestt = ms;
                    bestc = b->cfg;
                }
            }
            if (st != LJ_OK) break;
        }
        if (st != LJ_OK) break;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    b->cfg = bestc;
    const lj_status st2 = build_plan(ctx, b);
    if (st == LJ_OK) st = st2;
    if (st != LJ_OK) return st;
    if (best) *best = bestc;
    if (best_ms) *best_ms = bestt;
    return lj_sync(ctx);
}
