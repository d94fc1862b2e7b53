/*
 * ljoracle.c -- CPU oracle for the cell-grid Lennard-Jones path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: the GPU product path
 * never links, loads or calls it.  Only tests/, __graft_entry__.smoke() and
 * the CPU-baseline legs of bench.py use it.
 *
 * It restates, in plain C, the algorithm of the reference's cell-grid path
 * (OptixLJ, Cuda-version/cudaLJ.cu) plus the truncated-LJ ("config") law
 * the new implementation adds.  Each function cites the reference lines it
 * follows.  Floating-point discipline: compiled with -ffp-contract=off, so
 * every a*b+c below is two roundings unless written as fmaf()/fma().
 *
 * Parity pins: the drand48 generator is checked against the C library's
 * drand48(); the compat pair law against the reference's own host-callable
 * lennardJonesPotential<float>() (built from the reference sources into
 * oracle/_ref); binning, candidate count and compat energies against the
 * reference kernels run on the GPU (golden fixtures under tests/golden).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define LJO_EXPORT __attribute__((visibility("default")))

/* ------------------------------------------------------------------------ */
/* drand48 (POSIX): X_{n+1} = (a X_n + c) mod 2^48, a = 0x5DEECE66D, c = 0xB. */
/* srand48(s) sets X_0 = (low 32 bits of s) << 16 | 0x330E; drand48() steps   */
/* first and returns X_{n+1} / 2^48.  The reference draws with drand48() in   */
/* SDK/optixMultiSphere/optixSphere.cpp:132-155.                              */
/* ------------------------------------------------------------------------ */
#define LJO_A 0x5DEECE66DULL
#define LJO_C 0xBULL
#define LJO_M48 ((1ULL << 48) - 1ULL)

LJO_EXPORT uint64_t ljo_srand48_state(uint64_t seed) {
    return ((uint64_t)(uint32_t)seed << 16) | 0x330EULL;
}

static inline double ljo_drand48_step(uint64_t* st) {
    *st = (LJO_A * *st + LJO_C) & LJO_M48;
    return ldexp((double)*st, -48);
}

LJO_EXPORT void ljo_drand48_fill(uint64_t seed, int64_t count, double* out) {
    uint64_t st = ljo_srand48_state(seed);
    for (int64_t i = 0; i < count; ++i) out[i] = ljo_drand48_step(&st);
}

/* Uniform box: per particle draw x, y, z in that order
 * (optixSphere.cpp:150-152); coordinate = (float)(lo + (hi - lo) * u) in
 * double, which for lo = 0, hi = 1 is exactly the reference's
 * make_float3(1.0f * drand48(), ...). */
LJO_EXPORT void ljo_generate_uniform(uint64_t seed, int64_t n, const float lo[3], const float hi[3],
                                     float* x, float* y, float* z) {
    uint64_t st = ljo_srand48_state(seed);
    const double l0 = lo[0], l1 = lo[1], l2 = lo[2];
    const double e0 = (double)hi[0] - l0, e1 = (double)hi[1] - l1, e2 = (double)hi[2] - l2;
    for (int64_t i = 0; i < n; ++i) {
        const double ux = ljo_drand48_step(&st);
        const double uy = ljo_drand48_step(&st);
        const double uz = ljo_drand48_step(&st);
        x[i] = (float)(l0 + e0 * ux);
        y[i] = (float)(l1 + e1 * uy);
        z[i] = (float)(l2 + e2 * uz);
    }
}

/* Sphere surface: theta = 2 pi u1, phi = acos(1 - 2 u2), in double
 * (optixSphere.cpp:135-145), centre c and radius r (the reference uses
 * r = 1, c = 0.5 on the OptiX path and c = 1 in cudaLJ.cu:198-220). */
LJO_EXPORT void ljo_generate_sphere(uint64_t seed, int64_t n, const float centre[3], float radius,
                                    float* x, float* y, float* z) {
    uint64_t st = ljo_srand48_state(seed);
    const double r = radius;
    for (int64_t i = 0; i < n; ++i) {
        const double theta = 2.0 * M_PI * ljo_drand48_step(&st);
        const double phi = acos(1.0 - 2.0 * ljo_drand48_step(&st));
        x[i] = (float)(r * sin(phi) * cos(theta) + (double)centre[0]);
        y[i] = (float)(r * sin(phi) * sin(theta) + (double)centre[1]);
        z[i] = (float)(r * cos(phi) + (double)centre[2]);
    }
}

/* ------------------------------------------------------------------------ */
/* Grid.  Dims = int(extent / cutoff) in float (cudaLJ.cu:528-530), origin  */
/* lo (the reference fixes it at 0, cudaLJ.cu:525).                          */
/* ------------------------------------------------------------------------ */
typedef struct {
    float origin[3];
    float width;
    int dim[3];
} ljo_grid;

LJO_EXPORT int ljo_grid_from_box(const float lo[3], const float hi[3], float cutoff, ljo_grid* g) {
    if (!(cutoff > 0.0f)) return -1;
    for (int d = 0; d < 3; ++d) {
        const float ext = hi[d] - lo[d];
        if (!(ext > 0.0f)) return -1;
        const float q = ext / cutoff;
        if (!(q < 2147483647.0f)) return -1;
        int G = (int)q;
        g->dim[d] = G < 1 ? 1 : G;
        g->origin[d] = lo[d];
    }
    g->width = cutoff;
    return 0;
}

/* Cell coordinate along one axis: int((x - origin) / width) with IEEE float
 * division and truncation, as PosToCellCoord (cudaLJ.cu:110-119).  Values
 * below 0 (or NaN) go to cell 0 and values at or past dim go to dim-1; the
 * reference has no such clamp and asserts instead (cudaLJ.cu:130-132). */
static inline int ljo_axis_cell(float x, float origin, float width, int dim) {
    const float q = (x - origin) / width;
    if (q >= (float)dim) return dim - 1;
    if (q > 0.0f) return (int)q;
    return 0;
}

/* Linear index (z * Gy + y) * Gx + x, CellCoordToIndex (cudaLJ.cu:128-134). */
static inline int64_t ljo_cell_of(const ljo_grid* g, float x, float y, float z) {
    const int cx = ljo_axis_cell(x, g->origin[0], g->width, g->dim[0]);
    const int cy = ljo_axis_cell(y, g->origin[1], g->width, g->dim[1]);
    const int cz = ljo_axis_cell(z, g->origin[2], g->width, g->dim[2]);
    return ((int64_t)cz * g->dim[1] + cy) * g->dim[0] + cx;
}

LJO_EXPORT void ljo_cells_of(const ljo_grid* g, int64_t n, const float* x, const float* y, const float* z,
                             int* cell) {
    for (int64_t i = 0; i < n; ++i) cell[i] = (int)ljo_cell_of(g, x[i], y[i], z[i]);
}

/* ------------------------------------------------------------------------ */
/* Binning: counts (ComputeNbParticlePerCells, cudaLJ.cu:345-383), exclusive */
/* scan into offsets[ncells+1] with offsets[0] = 0 (PrefixFullV2 written at  */
/* prefix+1 after a memset, cudaLJ.cu:621-622 and prefixsum.hpp:160-215),    */
/* scatter to cell order (MoveParticlesToNewCells, cudaLJ.cu:441-471).       */
/* The reference's within-cell order comes from atomic tickets and is not    */
/* deterministic; this oracle defines it:                                    */
/*   order 0: ascending original index (a stable scatter on the cell key);   */
/*   order 1: ascending x, ties by ascending original index.                 */
/* ------------------------------------------------------------------------ */
static const float* g_sort_x;
static int ljo_cmp_x_then_idx(const void* a, const void* b) {
    const int ia = *(const int*)a, ib = *(const int*)b;
    const float xa = g_sort_x[ia], xb = g_sort_x[ib];
    if (xa < xb) return -1;
    if (xb < xa) return 1;
    return (ia > ib) - (ia < ib);
}

LJO_EXPORT int ljo_bin(const ljo_grid* g, int64_t n, const float* x, const float* y, const float* z, int order,
                       int* counts, int* offsets, int* perm, int* cell_sorted) {
    const int64_t ncells = (int64_t)g->dim[0] * g->dim[1] * g->dim[2];
    int* cell = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    int* fill = (int*)calloc((size_t)ncells, sizeof(int));
    if (!cell || !fill) { free(cell); free(fill); return -1; }
    memset(counts, 0, sizeof(int) * (size_t)ncells);
    for (int64_t i = 0; i < n; ++i) {
        cell[i] = (int)ljo_cell_of(g, x[i], y[i], z[i]);
        counts[cell[i]]++;
    }
    int64_t run = 0;
    for (int64_t c = 0; c < ncells; ++c) { offsets[c] = (int)run; run += counts[c]; }
    offsets[ncells] = (int)run;
    for (int64_t i = 0; i < n; ++i) {
        const int c = cell[i];
        const int slot = offsets[c] + fill[c]++;
        perm[slot] = (int)i;
        cell_sorted[slot] = c;
    }
    if (order == 1) {
        g_sort_x = x;
        for (int64_t c = 0; c < ncells; ++c)
            if (counts[c] > 1) qsort(perm + offsets[c], (size_t)counts[c], sizeof(int), ljo_cmp_x_then_idx);
    }
    free(cell);
    free(fill);
    return 0;
}

/* Candidate ordered pairs, ComputeNbInteractions (cudaLJ.cu:255-297): each
 * particle counts (own cell - 1) plus the occupancy of the other cells of
 * its clamped 3x3x3 stencil, with no distance test. */
LJO_EXPORT uint64_t ljo_count_candidates(const ljo_grid* g, const int* offsets) {
    const int gx = g->dim[0], gy = g->dim[1], gz = g->dim[2];
    uint64_t total = 0;
#pragma omp parallel for reduction(+ : total) schedule(static)
    for (int cz = 0; cz < gz; ++cz) {
        for (int cy = 0; cy < gy; ++cy) {
            for (int cx = 0; cx < gx; ++cx) {
                const int64_t c = ((int64_t)cz * gy + cy) * gx + cx;
                const int64_t nc = offsets[c + 1] - offsets[c];
                if (nc == 0) continue;
                int64_t s = 0;
                for (int z = cz > 0 ? cz - 1 : 0; z <= (cz + 1 < gz ? cz + 1 : gz - 1); ++z)
                    for (int y = cy > 0 ? cy - 1 : 0; y <= (cy + 1 < gy ? cy + 1 : gy - 1); ++y) {
                        const int xl = cx > 0 ? cx - 1 : 0, xh = cx + 1 < gx ? cx + 1 : gx - 1;
                        const int64_t rb = ((int64_t)z * gy + y) * gx;
                        s += offsets[rb + xh + 1] - offsets[rb + xl];
                    }
                total += (uint64_t)(nc * (s - 1));
            }
        }
    }
    return total;
}

/* ------------------------------------------------------------------------ */
/* Compat pair law: distance() and lennardJonesPotential() of                */
/* cudaLJ.cu:28-56 with epsilon = sigma = 1 (call site cudaLJ.cu:332):       */
/*   r = sqrt(dx^2 + dy^2 + dz^2 + 1e-5), s = sigma / r,                     */
/*   r6 = (s s)(s s)(s s), r12 = r6 r6, V = (4 eps)(r12 - r6).               */
/* ------------------------------------------------------------------------ */
LJO_EXPORT float ljo_lj_compat(float x1, float y1, float z1, float x2, float y2, float z2, float epsilon,
                               float sigma) {
    const float softening = 1e-5f;
    const float dx = x2 - x1, dy = y2 - y1, dz = z2 - z1;
    const float r = sqrtf(dx * dx + dy * dy + dz * dz + softening);
    const float sdr = sigma / r;
    const float r6 = (sdr * sdr) * (sdr * sdr) * (sdr * sdr);
    const float r12 = r6 * r6;
    return 4.0f * epsilon * (r12 - r6);
}

static inline void ljo_coords(const ljo_grid* g, int64_t c, int* cx, int* cy, int* cz) {
    const int64_t gxy = (int64_t)g->dim[0] * g->dim[1];
    *cz = (int)(c / gxy);
    const int64_t r = c - (int64_t)(*cz) * gxy;
    *cy = (int)(r / g->dim[0]);
    *cx = (int)(r - (int64_t)(*cy) * g->dim[0]);
}

/* Per-particle compat energy over the clamped 27-cell stencil, loop order
 * z, y, x and j ascending, self excluded by sorted index: the hot loop of
 * ComputeParticleInterationsParPartNoLoop (cudaLJ.cu:299-341).  Inputs are
 * in sorted (cell) order; v[k] is the energy of sorted particle k. */
LJO_EXPORT void ljo_compat_energy(const ljo_grid* g, int64_t n, const float* sx, const float* sy, const float* sz,
                                  const int* cell_sorted, const int* offsets, float* v) {
    const int gx = g->dim[0], gy = g->dim[1], gz = g->dim[2];
#pragma omp parallel for schedule(dynamic, 1024)
    for (int64_t k = 0; k < n; ++k) {
        int cx, cy, cz;
        ljo_coords(g, cell_sorted[k], &cx, &cy, &cz);
        float pot = 0.0f;
        for (int z = cz > 0 ? cz - 1 : 0; z <= (cz + 1 < gz ? cz + 1 : gz - 1); ++z)
            for (int y = cy > 0 ? cy - 1 : 0; y <= (cy + 1 < gy ? cy + 1 : gy - 1); ++y)
                for (int x = cx > 0 ? cx - 1 : 0; x <= (cx + 1 < gx ? cx + 1 : gx - 1); ++x) {
                    const int64_t c = ((int64_t)z * gy + y) * gx + x;
                    for (int j = offsets[c]; j < offsets[c + 1]; ++j)
                        if (j != k) pot += ljo_lj_compat(sx[k], sy[k], sz[k], sx[j], sy[j], sz[j], 1.0f, 1.0f);
                }
        v[k] = pot;
    }
}

/* ------------------------------------------------------------------------ */
/* Config law (new; not in the reference): truncated, unshifted LJ           */
/*   V(r) = 4 eps [(sigma/r)^12 - (sigma/r)^6]  for i != j and r < rc,       */
/* built from r^-2.  The distance test is the single definition shared with  */
/* the GPU kernels, so the interacting-pair count is bit-exact:              */
/*   d = p_j - p_i (float), r2 = fmaf(dz, dz, fmaf(dy, dy, dx*dx)),          */
/*   interacting iff r2 < rc*rc (both float).                                */
/* Per-particle outputs (sorted order): e_i = 4 eps sum_j s^12 - s^6 and     */
/* (optional) the conditioning scales 4 eps sum_j (s^12 + s^6) and          */
/* 24 eps sum_j (2 s^12 + s^6) / r: each pair term taken before the          */
/* cancellation between its repulsive and attractive parts.                  */
/* F_i = 24 eps sum_j r^-2 (2 s^12 - s^6) (p_i - p_j).  Totals:              */
/* E = 1/2 sum_i e_i, virial W = 1/2 sum_i sum_j 24 eps (2 s^12 - s^6),      */
/* pairs = number of interacting ordered pairs.                              */
/* The float force is accumulated as sum (2 s^12 - s^6) s^2 d and scaled by */
/* -24 eps / sigma^2 once, as the GPU kernel does (no overflow of r^-2 t).   */
/* nnb[k] (optional) = interacting neighbours of particle k.                 */
/* The loop visits the reference's full 27-cell stencil (cudaLJ.cu:319-337). */
/* ------------------------------------------------------------------------ */
static inline int ljo_interacts(float xi, float yi, float zi, float xj, float yj, float zj, float rc2, float* dx,
                                float* dy, float* dz, float* r2) {
    *dx = xj - xi;
    *dy = yj - yi;
    *dz = zj - zi;
    *r2 = fmaf(*dz, *dz, fmaf(*dy, *dy, *dx * *dx));
    return *r2 < rc2;
}

LJO_EXPORT void ljo_config_forces(const ljo_grid* g, int64_t n, const float* sx, const float* sy, const float* sz,
                                  const int* cell_sorted, const int* offsets, float rc, float eps, float sigma,
                                  float* e32, float* f32, double* e64, double* f64, uint64_t* pairs_out,
                                  double* etot_out, double* vir_out, double* escale64, double* fscale64,
                                  int* nnb) {
    const int gx = g->dim[0], gy = g->dim[1], gz = g->dim[2];
    const float rc2 = rc * rc;
    const float sig2 = sigma * sigma;
    const double sig2d = (double)sigma * (double)sigma;
    uint64_t pairs = 0;
    double etot = 0.0, vir = 0.0;
#pragma omp parallel for schedule(dynamic, 1024) reduction(+ : pairs, etot, vir)
    for (int64_t k = 0; k < n; ++k) {
        int cx, cy, cz;
        ljo_coords(g, cell_sorted[k], &cx, &cy, &cz);
        const float xi = sx[k], yi = sy[k], zi = sz[k];
        float ea = 0.0f, fxa = 0.0f, fya = 0.0f, fza = 0.0f;
        double ed = 0.0, fxd = 0.0, fyd = 0.0, fzd = 0.0, wd = 0.0, esd = 0.0, fsd = 0.0;
        uint64_t np = 0;
        for (int z = cz > 0 ? cz - 1 : 0; z <= (cz + 1 < gz ? cz + 1 : gz - 1); ++z)
            for (int y = cy > 0 ? cy - 1 : 0; y <= (cy + 1 < gy ? cy + 1 : gy - 1); ++y)
                for (int x = cx > 0 ? cx - 1 : 0; x <= (cx + 1 < gx ? cx + 1 : gx - 1); ++x) {
                    const int64_t c = ((int64_t)z * gy + y) * gx + x;
                    for (int j = offsets[c]; j < offsets[c + 1]; ++j) {
                        if (j == k) continue;
                        float dx, dy, dz, r2;
                        if (!ljo_interacts(xi, yi, zi, sx[j], sy[j], sz[j], rc2, &dx, &dy, &dz, &r2)) continue;
                        ++np;
                        if (e32 || f32) {
                            const float ir2 = 1.0f / r2;
                            const float s2 = sig2 * ir2;
                            const float s6 = s2 * s2 * s2;
                            const float s12 = s6 * s6;
                            ea += s12 - s6;
                            const float fs = (2.0f * s12 - s6) * s2;
                            fxa += fs * dx;
                            fya += fs * dy;
                            fza += fs * dz;
                        }
                        if (e64 || f64 || etot_out || vir_out || escale64 || fscale64) {
                            const double ddx = (double)sx[j] - (double)xi;
                            const double ddy = (double)sy[j] - (double)yi;
                            const double ddz = (double)sz[j] - (double)zi;
                            const double rr2 = ddx * ddx + ddy * ddy + ddz * ddz;
                            const double ir2 = 1.0 / rr2;
                            const double s2 = sig2d * ir2;
                            const double s6 = s2 * s2 * s2;
                            const double s12 = s6 * s6;
                            ed += s12 - s6;
                            const double w = 2.0 * s12 - s6;
                            wd += w;
                            const double fs = ir2 * w;
                            fxd += fs * ddx;
                            fyd += fs * ddy;
                            fzd += fs * ddz;
                            esd += s12 + s6;
                            fsd += ir2 * (2.0 * s12 + s6) * sqrt(rr2);
                        }
                    }
                }
        pairs += np;
        if (e32) e32[k] = 4.0f * eps * ea;
        if (f32) {
            const float fsc = -24.0f * eps / sig2;
            f32[3 * k + 0] = fsc * fxa;
            f32[3 * k + 1] = fsc * fya;
            f32[3 * k + 2] = fsc * fza;
        }
        if (nnb) nnb[k] = (int)np;
        const double e4 = 4.0 * (double)eps, e24 = 24.0 * (double)eps;
        if (e64) e64[k] = e4 * ed;
        if (f64) {
            f64[3 * k + 0] = -e24 * fxd;
            f64[3 * k + 1] = -e24 * fyd;
            f64[3 * k + 2] = -e24 * fzd;
        }
        if (escale64) escale64[k] = e4 * esd;
        if (fscale64) fscale64[k] = e24 * fsd;
        etot += 0.5 * e4 * ed;
        vir += 0.5 * e24 * wd;
    }
    if (pairs_out) *pairs_out = pairs;
    if (etot_out) *etot_out = etot;
    if (vir_out) *vir_out = vir;
}

/* CPU baseline entry: the reference's cell-grid loop (27-cell stencil per
 * particle, cudaLJ.cu:299-341) with the config law in float only, over a
 * contiguous block of targets [k0, k1) so that a bounded sample can be
 * timed.  Returns the interacting-pair count of the block. */
LJO_EXPORT uint64_t ljo_config_forces_f32_range(const ljo_grid* g, int64_t k0, int64_t k1, const float* sx,
                                                const float* sy, const float* sz, const int* cell_sorted,
                                                const int* offsets, float rc, float eps, float sigma, float* e32,
                                                float* f32, int nthreads) {
    const int gx = g->dim[0], gy = g->dim[1], gz = g->dim[2];
    const float rc2 = rc * rc;
    const float sig2 = sigma * sigma;
    uint64_t pairs = 0;
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
#pragma omp parallel for schedule(dynamic, 1024) reduction(+ : pairs)
    for (int64_t k = k0; k < k1; ++k) {
        int cx, cy, cz;
        ljo_coords(g, cell_sorted[k], &cx, &cy, &cz);
        const float xi = sx[k], yi = sy[k], zi = sz[k];
        float ea = 0.0f, fxa = 0.0f, fya = 0.0f, fza = 0.0f;
        uint64_t np = 0;
        for (int z = cz > 0 ? cz - 1 : 0; z <= (cz + 1 < gz ? cz + 1 : gz - 1); ++z)
            for (int y = cy > 0 ? cy - 1 : 0; y <= (cy + 1 < gy ? cy + 1 : gy - 1); ++y)
                for (int x = cx > 0 ? cx - 1 : 0; x <= (cx + 1 < gx ? cx + 1 : gx - 1); ++x) {
                    const int64_t c = ((int64_t)z * gy + y) * gx + x;
                    for (int j = offsets[c]; j < offsets[c + 1]; ++j) {
                        if (j == k) continue;
                        float dx, dy, dz, r2;
                        if (!ljo_interacts(xi, yi, zi, sx[j], sy[j], sz[j], rc2, &dx, &dy, &dz, &r2)) continue;
                        ++np;
                        const float ir2 = 1.0f / r2;
                        const float s2 = sig2 * ir2;
                        const float s6 = s2 * s2 * s2;
                        const float s12 = s6 * s6;
                        ea += s12 - s6;
                        const float fs = (2.0f * s12 - s6) * s2;
                        fxa += fs * dx;
                        fya += fs * dy;
                        fza += fs * dz;
                    }
                }
        pairs += np;
        e32[k] = 4.0f * eps * ea;
        const float fsc = -24.0f * eps / sig2;
        f32[3 * k + 0] = fsc * fxa;
        f32[3 * k + 1] = fsc * fya;
        f32[3 * k + 2] = fsc * fza;
    }
    return pairs;
}

LJO_EXPORT int ljo_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* Vectorised ljo_lj_compat over n pairs (a[3i..], b[3i..]), epsilon = sigma = 1. */
LJO_EXPORT void ljo_lj_compat_many(int64_t n, const float* a, const float* b, float* out) {
    for (int64_t i = 0; i < n; ++i)
        out[i] = ljo_lj_compat(a[3 * i], a[3 * i + 1], a[3 * i + 2], b[3 * i], b[3 * i + 1], b[3 * i + 2], 1.0f,
                               1.0f);
}

/* All-pairs O(n^2) evaluation of the config law with the same float distance
 * test, in FP64 (no grid).  Checks that the cell-list loops find every
 * interacting pair.  Outputs in input order. */
LJO_EXPORT uint64_t ljo_brute_force(int64_t n, const float* x, const float* y, const float* z, float rc, float eps,
                                    float sigma, double* e64, double* f64) {
    const float rc2 = rc * rc;
    const double sig2d = (double)sigma * (double)sigma;
    uint64_t pairs = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : pairs)
    for (int64_t i = 0; i < n; ++i) {
        double ed = 0, fxd = 0, fyd = 0, fzd = 0;
        for (int64_t j = 0; j < n; ++j) {
            if (j == i) continue;
            float dx, dy, dz, r2;
            if (!ljo_interacts(x[i], y[i], z[i], x[j], y[j], z[j], rc2, &dx, &dy, &dz, &r2)) continue;
            ++pairs;
            const double ddx = (double)x[j] - (double)x[i];
            const double ddy = (double)y[j] - (double)y[i];
            const double ddz = (double)z[j] - (double)z[i];
            const double ir2 = 1.0 / (ddx * ddx + ddy * ddy + ddz * ddz);
            const double s2 = sig2d * ir2, s6 = s2 * s2 * s2, s12 = s6 * s6;
            ed += s12 - s6;
            const double fs = ir2 * (2.0 * s12 - s6);
            fxd += fs * ddx;
            fyd += fs * ddy;
            fzd += fs * ddz;
        }
        if (e64) e64[i] = 4.0 * (double)eps * ed;
        if (f64) {
            f64[3 * i + 0] = -24.0 * (double)eps * fxd;
            f64[3 * i + 1] = -24.0 * (double)eps * fyd;
            f64[3 * i + 2] = -24.0 * (double)eps * fzd;
        }
    }
    return pairs;
}

/* ------------------------------------------------------------------------ */
/* Mixed-precision form (new; not in the reference).  Records: x in float,  */
/* y and z as binary16 offsets from the particle's cell origin in cell       */
/* widths: u = (y - fmaf(cy, w, oy)) / w rounded to binary16.  The distance  */
/* test is the kernel's, in cell units: dx = (xj - xi) * (1/w),              */
/* dy = uyj - (uyi - (cyj - cyi)), dz likewise, r2 = fmaf(dz, dz, fmaf(dy,   */
/* dy, dx*dx)) < (rc*rc) * (1/w) * (1/w).  The FP64 law runs on the stored   */
/* positions (x, oy + (cy + uy) w, oz + (cz + uz) w).                        */
/* ------------------------------------------------------------------------ */
LJO_EXPORT void ljo_pack_mixed(const ljo_grid* g, int64_t n, const float* sy, const float* sz, const int* cell_sorted,
                               float* uy, float* uz) {
    for (int64_t k = 0; k < n; ++k) {
        int cx, cy, cz;
        ljo_coords(g, cell_sorted[k], &cx, &cy, &cz);
        const float py = fmaf((float)cy, g->width, g->origin[1]);
        const float pz = fmaf((float)cz, g->width, g->origin[2]);
        uy[k] = (float)(_Float16)((sy[k] - py) / g->width);
        uz[k] = (float)(_Float16)((sz[k] - pz) / g->width);
    }
}

LJO_EXPORT void ljo_mixed_forces(const ljo_grid* g, int64_t k0, int64_t k1, const float* sx, const float* uy,
                                 const float* uz, const int* cell_sorted, const int* offsets, float rc, float eps,
                                 float sigma, double* e64, double* f64, uint64_t* pairs_out, double* etot_out,
                                 double* vir_out, double* escale64, double* fscale64, int* nnb) {
    const int gx = g->dim[0], gy = g->dim[1], gz = g->dim[2];
    const float w = g->width;
    const float invw = 1.0f / w;
    const float rc2u = rc * rc * invw * invw;
    const double wd = w, sig2d = (double)sigma * (double)sigma;
    uint64_t pairs = 0;
    double etot = 0.0, vir = 0.0;
#pragma omp parallel for schedule(dynamic, 1024) reduction(+ : pairs, etot, vir)
    for (int64_t k = k0; k < k1; ++k) {
        int cx, cy, cz;
        ljo_coords(g, cell_sorted[k], &cx, &cy, &cz);
        double ed = 0, fxd = 0, fyd = 0, fzd = 0, wd2 = 0, esd = 0, fsd = 0;
        uint64_t np = 0;
        for (int z = cz > 0 ? cz - 1 : 0; z <= (cz + 1 < gz ? cz + 1 : gz - 1); ++z)
            for (int y = cy > 0 ? cy - 1 : 0; y <= (cy + 1 < gy ? cy + 1 : gy - 1); ++y) {
                const float ty = uy[k] - (float)(y - cy);
                const float tz = uz[k] - (float)(z - cz);
                for (int x = cx > 0 ? cx - 1 : 0; x <= (cx + 1 < gx ? cx + 1 : gx - 1); ++x) {
                    const int64_t c = ((int64_t)z * gy + y) * gx + x;
                    for (int j = offsets[c]; j < offsets[c + 1]; ++j) {
                        if (j == k) continue;
                        const float dx = (sx[j] - sx[k]) * invw;
                        const float dy = uy[j] - ty;
                        const float dz = uz[j] - tz;
                        const float r2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
                        if (!(r2 < rc2u)) continue;
                        ++np;
                        /* stored positions in double */
                        const double ddx = (double)sx[j] - (double)sx[k];
                        const double ddy = ((double)(y - cy) + (double)uy[j] - (double)uy[k]) * wd;
                        const double ddz = ((double)(z - cz) + (double)uz[j] - (double)uz[k]) * wd;
                        const double rr2 = ddx * ddx + ddy * ddy + ddz * ddz;
                        const double ir2 = 1.0 / rr2;
                        const double s2 = sig2d * ir2, s6 = s2 * s2 * s2, s12 = s6 * s6;
                        ed += s12 - s6;
                        const double t = 2.0 * s12 - s6;
                        wd2 += t;
                        const double fs = ir2 * t;
                        fxd += fs * ddx;
                        fyd += fs * ddy;
                        fzd += fs * ddz;
                        esd += s12 + s6;
                        fsd += ir2 * (2.0 * s12 + s6) * sqrt(rr2);
                    }
                }
            }
        pairs += np;
        const double e4 = 4.0 * (double)eps, e24 = 24.0 * (double)eps;
        if (e64) e64[k] = e4 * ed;
        if (f64) {
            f64[3 * k + 0] = -e24 * fxd;
            f64[3 * k + 1] = -e24 * fyd;
            f64[3 * k + 2] = -e24 * fzd;
        }
        if (escale64) escale64[k] = e4 * esd;
        if (fscale64) fscale64[k] = e24 * fsd;
        if (nnb) nnb[k] = (int)np;
        etot += 0.5 * e4 * ed;
        vir += 0.5 * e24 * wd2;
    }
    if (pairs_out) *pairs_out = pairs;
    if (etot_out) *etot_out = etot;
    if (vir_out) *vir_out = vir;
}
