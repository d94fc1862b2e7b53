/*
 * ljcell.h -- C ABI of the B200 cell-grid Lennard-Jones path.
 *
 * Drop-in boundary for the cell-grid path of OptixLJ (Cuda-version/cudaLJ.cu).
 * The reference has no library API: its de facto interface is the set of
 * stage kernels called by executeSimulation() (cudaLJ.cu:515-677) on a
 * ParticlesContainer<float> (cudaLJ.cu:60-67) and CellDescriptor array
 * (cudaLJ.cu:91-94).  Each entry point below replaces one of those stages and
 * cites it.
 *
 * Conventions
 *  - Plain pointers and sizes only.  Pointers documented as "device" are CUDA
 *    device pointers; "host" pointers are ordinary memory.
 *  - Every call that launches work is asynchronous on the context's stream
 *    (lj_set_stream; 0 = legacy default stream).  Scalar results are written to
 *    device memory; lj_sync() waits and reports errors that kernels recorded
 *    in the context's device status word (LJ_ERANGE for non-finite positions,
 *    LJ_ETIMEOUT for a bounded wait that gave up).
 *  - Errors are returned, never exit(): the reference's CUDA_ASSERT called
 *    exit(1) (cudaLJ.cu:17-26).
 *  - One context per host thread; contexts are not shared between threads.
 *  - The context owns its scratch memory (scan tile states, tickets, reduction
 *    partials) and reuses it across calls; the caller owns every buffer it
 *    passes in.
 */
#ifndef LJCELL_H
#define LJCELL_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LJCELL_ABI_VERSION 1

#if defined(__GNUC__)
#define LJ_API __attribute__((visibility("default")))
#else
#define LJ_API
#endif

typedef enum {
    LJ_OK = 0,
    LJ_EINVAL = 1,       /* bad argument (NULL pointer, size, cutoff <= 0, ...) */
    LJ_ENOMEM = 2,       /* device allocation of context scratch failed */
    LJ_ECUDA = 3,        /* a CUDA runtime call failed */
    LJ_ETIMEOUT = 4,     /* a bounded device-side wait gave up */
    LJ_ERANGE = 5,       /* non-finite particle coordinate seen by the binning */
    LJ_EUNSUPPORTED = 6, /* size or mode outside what this build supports */
    LJ_ECHECK = 7        /* a consistency check of the bounds-checked build (libljcell_checks.so,
                            compiled with -DLJ_CHECKS) failed: negative count, offsets that do not
                            match the counts, a ticket outside its cell, a sorted record outside its
                            cell's range, out of order, or a permutation that is not a bijection */
} lj_status;

/* Within-cell order of the sorted particles.  The reference's order comes
 * from atomic tickets (cudaLJ.cu:462) and changes run to run; both orders
 * here are deterministic functions of the input. */
typedef enum {
    LJ_ORDER_INDEX = 0, /* ascending original index: a stable scatter on the cell key */
    LJ_ORDER_X = 1      /* ascending x, ties by original index (enables x-windowed pair search) */
} lj_order;

typedef struct lj_ctx lj_ctx;

/* == ParticlesContainer<float> (cudaLJ.cu:60-67): device SoA arrays. */
typedef struct {
    float* x;
    float* y;
    float* z;
    float* v;
    int* index;
    int nbParticles;
} lj_particles;

/* == CellDescriptor (cudaLJ.cu:91-94). */
typedef struct {
    int nbParticleInCell;
    int offsetInContainer;
} lj_cell_desc;

/* Regular cell grid: cell (cx,cy,cz) covers origin + [c, c+1) * width per
 * axis; linear index (cz * dim[1] + cy) * dim[0] + cx as CellCoordToIndex
 * (cudaLJ.cu:128-134).  The reference fixes origin = 0 (cudaLJ.cu:525). */
typedef struct {
    float origin[3];
    float width;
    int dim[3];
} lj_grid;

/* Truncated LJ parameters: V = 4 eps [(sigma/r)^12 - (sigma/r)^6], r < cutoff. */
typedef struct {
    float cutoff;
    float epsilon;
    float sigma;
} lj_params;

/* Global results of a compute call (device or host memory as documented). */
typedef struct {
    double energy;            /* E = 1/2 sum_i e_i */
    double virial;            /* W = sum_{i<j} r_ij . F_ij */
    unsigned long long pairs; /* interacting ordered pairs (i != j, r < cutoff) */
    unsigned long long pad;
} lj_totals;

/* ------------------------------------------------------------------ context */
LJ_API int lj_abi_version(void);
LJ_API const char* lj_status_str(lj_status s);

/* Creates a context on `device` issuing work on `stream` (a cudaStream_t,
 * NULL = legacy default stream). */
LJ_API lj_status lj_create(lj_ctx** out, int device, void* stream);
LJ_API lj_status lj_destroy(lj_ctx* ctx);
LJ_API lj_status lj_set_stream(lj_ctx* ctx, void* stream);
/* Waits for the context's stream, then returns (and clears) the first error
 * recorded by its kernels. */
LJ_API lj_status lj_sync(lj_ctx* ctx);

/* --------------------------------------------------------------- generation
 * Replaces InitRandStates + InitParticles / InitParticlesSphere
 * (cudaLJ.cu:98-105, 174-220).  The generator is the POSIX drand48 LCG with
 * srand48(seed) semantics, drawn in the order of the reference's host
 * generator (SDK/optixMultiSphere/optixSphere.cpp:132-155), evaluated on the
 * device by jump-ahead.  Outputs: SoA x, y, z (device), index[i] = i and
 * v[i] = -1 as InitParticles does (each of x/y/z/index/v may be NULL), and
 * optionally an AoS point3d array xyz[3n] (device, may be NULL). */
LJ_API lj_status lj_generate_uniform(lj_ctx* ctx, uint64_t seed, int n, const float lo[3], const float hi[3],
                              lj_particles* out, float* xyz);
LJ_API lj_status lj_generate_sphere(lj_ctx* ctx, uint64_t seed, int n, const float centre[3], float radius,
                             lj_particles* out, float* xyz);

/* ------------------------------------------------------------------- grid
 * Host-only.  dim = int(extent / cutoff) in float, at least 1, as
 * executeSimulation computes GridDim (cudaLJ.cu:528-530). */
LJ_API lj_status lj_grid_from_box(const float lo[3], const float hi[3], float cutoff, lj_grid* out);
/* The reference's grid: origin 0, box [0, box_width)^3 (cudaLJ.cu:525-530). */
LJ_API lj_status lj_grid_compat(float box_width, float cutoff, lj_grid* out);

/* ----------------------------------------------------------------- binning */
/* Per-cell counts, replaces ComputeNbParticlePerCells (cudaLJ.cu:345-383).
 * Positions are read as x[i*stride], y[i*stride], z[i*stride] (stride 1 for
 * SoA, 3 for an AoS point3d array with y = x + 1, z = x + 2).  counts[ncells]
 * (device) is overwritten. */
LJ_API lj_status lj_count_cells(lj_ctx* ctx, const lj_grid* g, int n, const float* x, const float* y, const float* z,
                         int stride, int* counts);

/* Exclusive scan offsets[0..ncells] (offsets[0] = 0, offsets[ncells] = total),
 * replaces PrefixFullV2 (prefixsum.hpp:160-215) as called at cudaLJ.cu:621-622
 * (memset prefix, scan into prefix + 1).  Single pass, decoupled look-back,
 * no per-call allocation, no host synchronisation.  Device pointers. */
LJ_API lj_status lj_exclusive_scan(lj_ctx* ctx, const int* counts, long long ncells, int* offsets);

/* Allocation-free exclusive scan (no counterpart in the reference).  For
 * callers that cannot allocate device memory -- code inside a host that owns
 * every byte of the device through its own pool, or code that must not pay
 * the device-wide synchronisation cudaMalloc/cudaFree can cause -- and so
 * cannot create an lj_ctx.  Same result as lj_exclusive_scan, computed by the
 * same kernel; its look-back scratch is a fixed array inside the library
 * (256 bytes + 8 bytes per 8192 cells, 64 KiB), which every GPU that loads
 * the library holds until the process exits.
 *   - ncells <= 67,108,864 (2^26); larger returns LJ_EUNSUPPORTED.
 *   - No cudaMalloc / cudaFree and no allocating library call.
 *   - Every call looks up the array's device address on the current device
 *     (cudaGetSymbolAddress, which allocates nothing), so a device reset
 *     between calls is harmless; the first call on a device may load the
 *     library's device code there, so make it before any stream capture
 *     begins.
 *   - `stream` must belong to the current device (LJ_EINVAL otherwise): the
 *     array used is the current device's.
 *   - Every call uses the same array: calls that may overlap on the GPU
 *     (different streams, no ordering between them) race and must not be
 *     issued.  Each call clears the part it uses before the scan.
 *   - Asynchronous on `stream` (a cudaStream_t, NULL = legacy default).  A
 *     bounded look-back wait that gave up (never expected) sets
 *     offsets[ncells] = -1 instead of the total. */
LJ_API lj_status lj_exclusive_scan_noalloc(const int* counts, long long ncells, int* offsets, void* stream);

/* Cell descriptors from offsets, replaces InitNewCells (cudaLJ.cu:428-439). */
LJ_API lj_status lj_cell_descriptors(lj_ctx* ctx, const int* offsets, long long ncells, lj_cell_desc* cells);

/* The whole cell-grid build, replaces the binning sequence of
 * executeSimulation (cudaLJ.cu:614-634): count, scan, descriptors and the
 * scatter of MoveParticlesToNewCells (cudaLJ.cu:441-471), made deterministic
 * (`order`).  Device pointers:
 *   in            positions as for lj_count_cells (stride 1 or 3)
 *   counts        [ncells]        per-cell occupancy                (required)
 *   offsets       [ncells + 1]    exclusive prefix of counts        (required)
 *   cells         [ncells]        CellDescriptor view               (may be NULL)
 *   sorted        SoA x, y, z, index of the particles in cell order  (may be NULL;
 *                 any member may be NULL; v is not touched, as in the reference)
 *   sorted_xyzi   [4n] float4 per particle: x, y, z, original index bit-cast
 *                 to float; 16-byte aligned                        (required)
 *   sorted_cell   [n] cell id per sorted particle                   (required) */
LJ_API lj_status lj_bin(lj_ctx* ctx, const lj_grid* g, int n, const float* x, const float* y, const float* z, int stride,
                 lj_order order, int* counts, int* offsets, lj_cell_desc* cells, lj_particles* sorted,
                 float* sorted_xyzi, int* sorted_cell);

/* ----------------------------------------------------------- interactions */
/* Candidate ordered pairs of the clamped 27-cell stencil, no distance test:
 * replaces ComputeNbInteractions (cudaLJ.cu:255-297).  *d_count (device) is
 * overwritten. */
LJ_API lj_status lj_count_candidates(lj_ctx* ctx, const lj_grid* g, const int* offsets, unsigned long long* d_count);

/* Reference pair law ("compat"): per-particle energy v[k] of sorted particle
 * k, summed over every particle of the clamped 27-cell stencil except itself,
 * with 4 eps ((s/r)^12 - (s/r)^6), eps = s = 1, r = sqrt(d.d + 1e-5) and no
 * cutoff test: replaces ComputeParticleInterationsParPartNoLoop
 * (cudaLJ.cu:299-341).  s/r comes from the approximate reciprocal square
 * root (at most 2 ulp) where the reference divides by an IEEE square root:
 * each particle's energy is within about 3e-6 relative of the reference's law
 * for stencils narrower than 1/sqrt(3) (the reference's own check allows
 * 1e-5, cudaLJ.cu:246-250).  Any within-cell order.  Device pointers from
 * lj_bin. */
LJ_API lj_status lj_compute_compat(lj_ctx* ctx, const lj_grid* g, int n, const float* sorted_xyzi, const int* sorted_cell,
                            const int* offsets, float* v);

/* Truncated LJ with forces (the configuration law; not in the reference):
 * for i != j and r < cutoff, e_k = 4 eps sum (s^12 - s^6) and
 * F_k = 24 eps sum r^-2 (2 s^12 - s^6) (p_k - p_j), s = sigma / r, built from
 * r^-2.  The distance test is d = p_j - p_k (float), r2 = fmaf(dz, dz,
 * fmaf(dy, dy, dx * dx)), interacting iff r2 < cutoff * cutoff.  `order` must
 * be the order the particles were binned with (LJ_ORDER_X enables the
 * x-windowed search).  Outputs in sorted order (device, each may be NULL):
 * energy[n], force[3n] (point3d), totals (one lj_totals). */
LJ_API lj_status lj_compute(lj_ctx* ctx, const lj_grid* g, const lj_params* p, int n, const float* sorted_xyzi,
                     const int* sorted_cell, const int* offsets, lj_order order, float* energy, float* force,
                     lj_totals* totals);

/* lj_compute for the targets [kb, ke) of the n sorted particles only (the candidates are all n):
 * energy and force written at those indices, totals over those targets.  The piece a
 * domain-decomposed step needs (no counterpart in the reference, which is single-GPU): a rank bins
 * its own particles and a one-cell halo received from its neighbours, and evaluates its own
 * particles, one contiguous sorted range when the domain is a range of z layers.  Each target's
 * results carry the bits lj_compute gives it with the same pair kernel.  With the tuning's
 * pair_kernel 0 the kernel is chosen, as by lj_compute, from n over the whole grid's cell count;
 * a caller whose particles fill only part of the grid sets the kernel (lj_set_tuning). */
LJ_API lj_status lj_compute_range(lj_ctx* ctx, const lj_grid* g, const lj_params* p, int n, const float* sorted_xyzi,
                                  const int* sorted_cell, const int* offsets, lj_order order, int kb, int ke,
                                  float* energy, float* force, lj_totals* totals);

/* Half-shell form of lj_compute (Newton's third law; the reference evaluates every
 * ordered pair twice, cudaLJ.cu:319-337): each unordered pair {i, j} of the
 * 27-cell stencil is evaluated once, by the cell of i when the cell of j is in
 * its forward half-stencil (or, in one cell, j > i), and the reaction goes to j.
 * Deterministic without float atomics: cells in 18 colours (period 3 in x and y,
 * 2 in z) run one colour per launch, so no two concurrent cells write one
 * particle, and within a cell the reactions collect in a fixed order.  Same
 * distance test and outputs as lj_compute (energy[n], force[3n], totals with
 * E = 1/2 sum of the per-particle energies and the ordered pair count, exactly
 * twice the unordered one); any within-cell order (no x-windows).  Scratch:
 * 20 bytes per particle in the context.  Asynchronous on the context's stream. */
LJ_API lj_status lj_compute_half(lj_ctx* ctx, const lj_grid* g, const lj_params* p, int n, const float* sorted_xyzi,
                                 const int* offsets, float* energy, float* force, lj_totals* totals);

/* ------------------------------------------------------------- tuning
 * Implementation choices of the context (no counterpart in the reference,
 * whose launch shape is fixed at 128 threads per particle, cudaLJ.cu:519-520).
 * Results do not depend on them except in the last bits of floating-point
 * sums.  pair_kernel, for particles binned with LJ_ORDER_X:
 *   0 = default: 10 when the grid averages 2 or more particles per cell, else 12,
 *   1 = one thread per target, neighbours through L1, its windows in shared
 *       memory (also the kernel of LJ_ORDER_INDEX),
 *   6 = row passes: the 9 stencil rows walked in 5 warp-synchronous passes
 *       (opposite rows paired), coalesced neighbour loads, two candidates per
 *       step in paired FP32 instructions,
 *  10 = row passes with two consecutive targets per lane: their windows
 *       merged, each candidate loaded once and tested against both targets in
 *       one paired FP32 evaluation, registers capped at 64 per thread, the
 *       windows parked in shared memory during the walk,
 *  11 = as 1 with the 9 rows walked whole (no row culling, no x-window
 *       searches): on sparse grids such as a sphere shell, where a row holds
 *       few particles, the searches cost more than the candidates they remove.
 *  12 = targets paired inside their cell (a pair list built on the device:
 *       flags, their scan, the list; 12 bytes per target of scratch in the
 *       context): both targets of a lane share one 27-cell stencil, whose
 *       non-empty rows are walked whole, end to end, all lanes in lockstep,
 *       each candidate loaded once for both; for sparse grids (no window
 *       searches, no lane whose targets need two stencils; the autotuner's
 *       pick on a sphere shell and on a uniform grid of 0.5 particles per
 *       cell).  A target's results do not depend on its partner, so
 *       lj_compute_range gives the bits of lj_compute.
 * The values 2-5 and 7-9 named variants that never won on any benchmark
 * workload (per-lane queues, register windows, cell-block tiles staged by TMA
 * bulk copies, scalar passes, SoA pairs); they are kept as aliases of the kernel
 * of their family: 2, 3, 4 run 1; 5, 7 run 6; 8, 9 run 10.
 * With a non-finite coordinate (reported as LJ_ERANGE) the outputs of the
 * particles whose windows hold it are unspecified under 6 and 10. */
typedef struct {
    int pair_kernel;
    int scatter_passes; /* binning scatter in this many passes over cell ranges (0 = one pass per
                           56 MiB of scattered records, so each pass's writes meet in L2); 1-8 */
    int reserved[6];
} lj_tuning;

LJ_API lj_status lj_set_tuning(lj_ctx* ctx, const lj_tuning* t);
/* Autotuner for one system: times the pair kernels 1, 6, 10, 11 and 12 on
 * these binned (LJ_ORDER_X) particles and keeps the fastest in the context's
 * tuning.  Synchronises. */
LJ_API lj_status lj_autotune_compute(lj_ctx* ctx, const lj_grid* g, const lj_params* p, int n,
                                     const float* sorted_xyzi, const int* sorted_cell, const int* offsets,
                                     int* best_kernel, float* best_ms);
LJ_API lj_status lj_get_tuning(lj_ctx* ctx, lj_tuning* t);

/* ------------------------------------------------------------- batched systems
 * Many independent systems of uneven sizes and cutoffs evaluated as one step
 * (no counterpart in the reference, which runs one system per
 * executeSimulation call).  The systems' particles sit back to back in one
 * SoA array: system s owns [first, first + n).  All systems are binned by one
 * launch per stage over a shared cell numbering, and the pair kernel is
 * persistent: its CTAs take (system, cell-block) tiles from a device work
 * queue, largest first. */
typedef struct {
    float lo[3];        /* box covered by the system's grid */
    float hi[3];
    lj_params params;   /* truncated law of the system (cutoff, epsilon, sigma) */
    int first;          /* first particle of the system in the batch arrays */
    int n;              /* particle count */
} lj_system;

typedef struct {
    float cell_multiple; /* cell width = cell_multiple * cutoff (>= 1; default 1) */
    int threads;         /* CTA size of the batched pair kernel: 64, 128 or 256 (default 128) */
    int per_thread;      /* targets per thread in a tile: 1 or 2 (default 1) */
    int reserved[5];
} lj_batch_config;

typedef struct lj_batch lj_batch;

/* Plans a batch: takes host copies of `systems`, allocates the device tables
 * and the batch's working buffers.  cfg may be NULL (defaults). */
LJ_API lj_status lj_batch_create(lj_ctx* ctx, int nsys, const lj_system* systems, const lj_batch_config* cfg,
                                 lj_batch** out);
LJ_API lj_status lj_batch_destroy(lj_batch* b);
LJ_API lj_status lj_batch_get_config(const lj_batch* b, lj_batch_config* cfg);
/* Grid of system s under the batch's current configuration. */
LJ_API lj_status lj_batch_grid(const lj_batch* b, int s, lj_grid* g);

/* One step for every system: binning (LJ_ORDER_X) and the truncated law.
 * x, y, z: device, all systems back to back.  Outputs (device, each may be
 * NULL), per system in its own range [first, first + n) and in that system's
 * cell order: energy, force (3 floats per particle), index (the batch-wide
 * index of each sorted particle); totals[nsys]: each system's lj_totals. */
LJ_API lj_status lj_batch_run(lj_ctx* ctx, lj_batch* b, const float* x, const float* y, const float* z,
                              float* energy, float* force, int* index, lj_totals* totals);
/* The same step captured once in a CUDA graph for a given set of pointers and
 * replayed; ordered after earlier work on the context's stream. */
LJ_API lj_status lj_batch_run_graph(lj_ctx* ctx, lj_batch* b, const float* x, const float* y, const float* z,
                                    float* energy, float* force, int* index, lj_totals* totals);
/* The same results computed with one lj_bin + lj_compute per system: the
 * per-system plain launches the batched step replaces. */
LJ_API lj_status lj_batch_run_separate(lj_ctx* ctx, lj_batch* b, const float* x, const float* y, const float* z,
                                       float* energy, float* force, int* index, lj_totals* totals);
/* Autotuner: times every combination of cell_multiple {1, 1.5, 2}, threads
 * {64, 128, 256} and per_thread {1, 2} on these inputs (graph replays), keeps
 * the fastest in the plan and returns it with its time per step in ms.
 * Synchronises. */
LJ_API lj_status lj_batch_autotune(lj_ctx* ctx, lj_batch* b, const float* x, const float* y, const float* z,
                                   lj_batch_config* best, float* best_ms);

/* ------------------------------------------------------------- mixed precision
 * The mixed-precision form of the truncated law (no counterpart in the
 * reference).  Storage: one 8-byte record per sorted particle, FP32 x and the
 * y, z offsets from the particle's cell origin in cell widths as binary16
 * (stored position = (x, oy + (cy + uy) w, oz + (cz + uz) w)): half the bytes
 * of the float4 layout per neighbour load.  Pair math in FP32 (cell units),
 * each particle's energy and force summed per stencil window (or per pass of
 * the row-pass walks) and those sums added with compensation (TwoSum), totals
 * reduced in FP64.  Results
 * are those of the stored positions: binary16 rounds the y, z offsets to
 * 2^-11 .. 2^-12 of a cell width, and the pair count follows the mixed
 * distance test (d in cell units, r2 < (cutoff / w)^2), restated exactly by
 * the oracle. */

/* Records from binned particles (LJ_ORDER_X).  rec: 2n floats, 8-byte aligned. */
LJ_API lj_status lj_pack_mixed(lj_ctx* ctx, const lj_grid* g, int n, const float* sorted_xyzi,
                               const int* sorted_cell, float* rec);
/* Energy, force (sorted order) and totals from the records; as lj_compute.
 * Walk by the tuning's pair_kernel: 0 (default) and 8-10 row passes with two
 * targets per lane; 1 flat walk, windows in shared memory; 2 flat walk,
 * windows in registers; any other value row passes with one target per lane. */
LJ_API lj_status lj_compute_mixed(lj_ctx* ctx, const lj_grid* g, const lj_params* p, int n, const float* rec,
                                  const int* sorted_cell, const int* offsets, float* energy, float* force,
                                  lj_totals* totals);

/* ------------------------------------------------------------- test hook
 * Failure-path check (no counterpart in the reference): runs the scan with
 * its first tile withheld, so every bounded look-back wait gives up; the next
 * lj_sync returns LJ_ETIMEOUT and the context stays usable.  ncells > 8192. */
LJ_API lj_status lj_test_scan_withheld_tile(lj_ctx* ctx, const int* counts, long long ncells, int* offsets);
/* The same failure path for lj_exclusive_scan_noalloc, on its fixed array: every bounded look-back
 * wait gives up and the call marks its result invalid with offsets[ncells] = -1.  ncells > 8192. */
LJ_API lj_status lj_test_scan_noalloc_withheld_tile(const int* counts, long long ncells, int* offsets, void* stream);
/* Allocation-failure injection (no counterpart in the reference): the k-th next
 * growth of a context's scratch memory, in any context of the process, fails
 * as a cudaMalloc failure would (the call returns LJ_ENOMEM, the context stays
 * usable); k = 0 turns the hook off.  For tests; not for concurrent use. */
LJ_API lj_status lj_test_fail_alloc(int k);

/* ------------------------------------------------------------- time step
 * One velocity-Verlet step of the truncated law with rebinning (no stage of
 * the reference, whose ParticlesContainer swap and per-particle cuRAND state,
 * cudaLJ.cu:69-76 and :96-97, anticipate particles moving between steps).
 * State, all device, in sorted order as lj_bin (LJ_ORDER_X) leaves it:
 *   xyzi[4n]      records (x, y, z, caller's particle id bits), 16-byte aligned
 *   vel[3n]       velocities
 *   force[3n]     forces of the current positions (lj_compute, or the last step)
 *   sorted_cell[n], counts[ncells], offsets[ncells + 1]  the cell grid of g
 * The step: v += h F (h = dt / (2 mass)); x += dt v; rebin the moved particles
 * from the current order; carry v and the ids to the new order; F = forces of
 * the new positions; v += h F.  Each update is one IEEE multiply and one add
 * (no fused multiply-add), in single precision.  On return every state array
 * holds the new sorted state; energy[n] (optional) and totals (optional) are
 * those of the new positions, as lj_compute writes them.  Scratch: 28 bytes
 * per particle in the context.  Asynchronous on the context's stream. */
LJ_API lj_status lj_step_verlet(lj_ctx* ctx, const lj_grid* g, const lj_params* p, int n, float dt, float mass,
                                float* xyzi, float* vel, float* force, int* sorted_cell, int* counts, int* offsets,
                                float* energy, lj_totals* totals);

/* ------------------------------------------------------------- spatial sort
 * Replaces reorder(N, points, radius) (SDK/optixMultiSphereAABB/sort.cu:29-41,
 * key kernel count_per_cell :7-18): sorts n float4 points in place by the key
 * of their cell and stores the key in .w as float.  width = int(1.0f/radius);
 * key = int(x/radius) + int(y/radius)*width + int(z/radius)*width*width as
 * the reference's own build computes it: its SDK compiles sort.cu with
 * --use_fast_math, so the divisions are the fast single-precision division
 * (which can put a coordinate within a couple of ulps of a cell face in the
 * neighbouring cell, unlike IEEE division), truncated; the stored key is the
 * exact integer sum rounded once to float, equal to the reference's
 * contracted float sum.  Points with equal .w keep their input order (the
 * reference's thrust::sort leaves that order unspecified).  points: device,
 * 16-byte aligned.  The domain is the reference's, coordinates in [0, 1]: a
 * point whose key falls outside it (or a NaN coordinate) is reported as
 * LJ_ERANGE by lj_sync and sorted as key 0.  width <= 512 (radius > 1/513),
 * else LJ_EUNSUPPORTED.  Scratch is the context's; asynchronous on its stream. */
LJ_API lj_status lj_reorder(lj_ctx* ctx, int n, float* points, float radius);

/* ------------------------------------------------------- slab decomposition
 * Boundary layers of a rank's particles for the halo exchange of a spatial
 * decomposition over z layers (no counterpart in the reference, which runs one
 * system on one GPU).  Of the n AoS positions xyz[3n] (device), the particles
 * whose z layer -- as lj_bin computes it for grid g -- equals layer_lo are
 * copied, in input order, to out_lo[3 * counts[0]], and those in layer_hi to
 * out_hi[3 * counts[1]] (device; room for n points each, or for as many as the
 * layer can hold).  A negative layer selects nothing (its output may be NULL).
 * counts: device int[2].  Deterministic (no atomics); three launches on the
 * context's stream; scratch 8 bytes per 1024 particles in the context. */
LJ_API lj_status lj_select_layers(lj_ctx* ctx, const lj_grid* g, int n, const float* xyz, int layer_lo,
                                  int layer_hi, float* out_lo, float* out_hi, int* counts);

/* ------------------------------------------------------------- end to end
 * One call with HOST buffers, the shape of executeSimulation's step
 * (cudaLJ.cu:613-653) without the generation: copies positions to the device,
 * bins (LJ_ORDER_X), computes the truncated law and copies back, in sorted
 * order, energy[n], force[3n] and index[n] (original index of each sorted
 * particle), plus the totals.  Device buffers are owned by the context and
 * reused.  Output pointers may be NULL.  Synchronises before returning. */
LJ_API lj_status lj_simulate_host(lj_ctx* ctx, const lj_grid* g, const lj_params* p, int n, const float* hx,
                           const float* hy, const float* hz, float* h_energy, float* h_force, int* h_index,
                           lj_totals* h_totals);

/* The same step without the final synchronisation, for a caller that runs
 * steps back to back (no counterpart in the reference): the call returns once
 * the work is queued, and consecutive calls overlap -- the next call's
 * positions go up on an upload stream while the previous call's results come
 * down on the copy stream (PCIe carries both directions at once).  Three device
 * buffer sets in the context are used in turn.  Host buffers must be pinned
 * for the copies to overlap; the caller must leave the input buffers unchanged,
 * keep every output buffer and h_totals valid, and not read them until
 * lj_simulate_host_wait returns (h_totals is written by that call, from pinned
 * staging in the context: at most 64 calls are staged, a 65th first waits for
 * the queued ones).  Errors recorded by kernels are reported by
 * lj_simulate_host_wait. */
LJ_API lj_status lj_simulate_host_async(lj_ctx* ctx, const lj_grid* g, const lj_params* p, int n, const float* hx,
                                        const float* hy, const float* hz, float* h_energy, float* h_force,
                                        int* h_index, lj_totals* h_totals);
/* Waits for every lj_simulate_host_async call queued so far, then as lj_sync. */
LJ_API lj_status lj_simulate_host_wait(lj_ctx* ctx);

/* The same step with energy[n] and force[3n] returned in the caller's input
 * order (particle i's results at index i), so no index array comes back: 16 B
 * per particle down instead of 20.  The pair kernel writes each particle's
 * results at its input index; they are copied down while the next queued step
 * uploads and computes.  Queued like lj_simulate_host_async
 * (same buffer rules, completed by lj_simulate_host_wait); the two kinds of
 * call may be mixed in one queue.  Per-particle results carry the same bits as
 * lj_simulate_host's, permuted by its index. */
LJ_API lj_status lj_simulate_host_inorder_async(lj_ctx* ctx, const lj_grid* g, const lj_params* p, int n,
                                                const float* hx, const float* hy, const float* hz, float* h_energy,
                                                float* h_force, lj_totals* h_totals);
/* lj_simulate_host_inorder_async followed by lj_simulate_host_wait (which also
 * completes any step queued before it). */
LJ_API lj_status lj_simulate_host_inorder(lj_ctx* ctx, const lj_grid* g, const lj_params* p, int n, const float* hx,
                                          const float* hy, const float* hz, float* h_energy, float* h_force,
                                          lj_totals* h_totals);

#ifdef __cplusplus
}
#endif

#endif /* LJCELL_H */
