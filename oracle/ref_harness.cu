// ref_harness.cu -- drives the REFERENCE's own cell-grid kernels.
//
// TEST INFRASTRUCTURE ONLY (the checker, never the product).  The Makefile in
// this directory compiles this file against the read-only reference sources
// (Cuda-version/cudaLJ.cu, prefixsum.hpp, point3d.hpp, SpTimer.hpp) where they
// lie, into oracle/_ref/libljref.so.  No reference source is copied here.
//
// Two uses:
//  * CPU: the reference's host-callable pair law (distance() and
//    lennardJonesPotential<float>(), cudaLJ.cu:28-56) pins the oracle's compat
//    law bit for bit.
//  * GPU: ljref_run() injects positions into a ParticlesContainer<float> and
//    runs the reference's stage kernels in executeSimulation's order
//    (cudaLJ.cu:613-653): count, PrefixFullV2, InitNewCells, ticket scatter,
//    ComputeNbInteractions, ComputeParticleInterationsParPartNoLoop.  It
//    bypasses cuRAND (InitRandStates/InitParticles) by design.
//
// Safety: the reference kernels index cells without clamping; with -DNDEBUG
// their asserts are compiled out, so an out-of-box position would write out of
// bounds.  ljref_run() therefore checks every position on the host with the
// same float arithmetic (x >= 0 and int(x / w) < dim) and refuses the input
// before any launch.  CUDA errors are recorded, never exit() the process.
#include <cstdio>
#include <cstdint>
#include <cmath>
#include <vector>

static int g_ljref_first_error = 0;
static int g_ljref_error_line = 0;
static inline void ljref_record(cudaError_t e, int line) {
    if (e != cudaSuccess && g_ljref_first_error == 0) {
        g_ljref_first_error = (int)e;
        g_ljref_error_line = line;
    }
}
#define CUDA_ASSERT(X) ljref_record((X), __LINE__)

#define main ljref_reference_main_unused
#include "cudaLJ.cu"
#undef main

extern "C" {

float ljref_lj_potential_host(float x1, float y1, float z1, float x2, float y2, float z2, float epsilon,
                              float sigma) {
    const Point3D<float> p1(x1, y1, z1), p2(x2, y2, z2);
    return lennardJonesPotential<float>(p1, p2, epsilon, sigma);
}

void ljref_lj_potential_host_many(int64_t n, const float* a, const float* b, float* out) {
    for (int64_t i = 0; i < n; ++i) {
        const Point3D<float> p1(a[3 * i], a[3 * i + 1], a[3 * i + 2]);
        const Point3D<float> p2(b[3 * i], b[3 * i + 1], b[3 * i + 2]);
        out[i] = lennardJonesPotential<float>(p1, p2, 1.0f, 1.0f);
    }
}

int ljref_last_error(int* line) {
    if (line) *line = g_ljref_error_line;
    return g_ljref_first_error;
}

// Grid dims exactly as executeSimulation computes them (cudaLJ.cu:528-530).
int ljref_grid_dim(float box_width, float cutoff) { return static_cast<int>(box_width / cutoff); }

// Runs the reference stages `reps` times on the same injected positions.
// Outputs (host buffers, from the last repetition):
//   counts[ncells], prefix[ncells+1], cells[2*ncells] (CellDescriptor pairs),
//   sorted x/y/z/index[n] and v[n] in the reference's (ticket) order,
//   nbinter = ComputeNbInteractions total.
// stage_ms[7] receives the minimum over repetitions of: count, scan,
//   descriptors, scatter, candidate count, pair kernel, and the sum of the
//   binning stages (count..scatter) measured as one span.
// Returns 0, -1 on bad arguments, -2 if a position is outside the grid the
// reference kernels can index, -3 on a CUDA error (see ljref_last_error).
int ljref_run(int n, const float* hx, const float* hy, const float* hz, float box_width, float cutoff, int* counts,
              int* prefix, int* cells, float* sx, float* sy, float* sz, int* sidx, float* v,
              unsigned long long* nbinter, float* stage_ms, int reps) {
    if (n <= 0 || !hx || !hy || !hz || !(cutoff > 0.0f) || reps < 1) return -1;
    const Point3D<float> CellWidth{cutoff, cutoff, cutoff};
    const int G = static_cast<int>(box_width / cutoff);
    if (G < 1) return -1;
    const Point3D<int> GridDim{G, G, G};
    const long long int NbCells = (long long int)G * G * G;
    const float* axes[3] = {hx, hy, hz};
    for (int a = 0; a < 3; ++a)
        for (int i = 0; i < n; ++i) {
            const float p = axes[a][i];
            if (!(p >= 0.0f)) return -2;
            const float q = p / cutoff;
            if (!(q < (float)G) || static_cast<int>(q) >= G) return -2;
        }
    g_ljref_first_error = 0;

    const int DefaultNbThreads = 128;
    const int DefaultNbBlocks = std::max(int((n + DefaultNbThreads - 1) / DefaultNbThreads), 1);
    std::list<void*> ptrs;
    ParticlesContainer<float> particles = AllocateParticles<float>(n, ptrs);
    ParticlesContainer<float> particlesSwap = AllocateParticles<float>(n, ptrs);
    ParticlesContainer<float> pristine = AllocateParticles<float>(n, ptrs);
    int* particlePerCells = nullptr;
    int* prefixParCell = nullptr;
    CellDescriptor* dcells = nullptr;
    unsigned long long* cuNb = nullptr;
    CUDA_ASSERT(cudaMalloc(&particlePerCells, NbCells * sizeof(int)));
    CUDA_ASSERT(cudaMalloc(&prefixParCell, (NbCells + 1) * sizeof(int)));
    CUDA_ASSERT(cudaMalloc(&dcells, NbCells * sizeof(CellDescriptor)));
    CUDA_ASSERT(cudaMalloc(&cuNb, sizeof(unsigned long long)));
    ptrs.push_back(particlePerCells);
    ptrs.push_back(prefixParCell);
    ptrs.push_back(dcells);
    ptrs.push_back(cuNb);
    if (g_ljref_first_error) { deletePtrs(ptrs); return -3; }

    std::vector<int> idx(n);
    std::vector<float> minus1(n, -1.0f);
    for (int i = 0; i < n; ++i) idx[i] = i;
    CUDA_ASSERT(cudaMemcpy(pristine.x, hx, n * sizeof(float), cudaMemcpyHostToDevice));
    CUDA_ASSERT(cudaMemcpy(pristine.y, hy, n * sizeof(float), cudaMemcpyHostToDevice));
    CUDA_ASSERT(cudaMemcpy(pristine.z, hz, n * sizeof(float), cudaMemcpyHostToDevice));
    CUDA_ASSERT(cudaMemcpy(pristine.index, idx.data(), n * sizeof(int), cudaMemcpyHostToDevice));
    CUDA_ASSERT(cudaMemcpy(pristine.v, minus1.data(), n * sizeof(float), cudaMemcpyHostToDevice));

    cudaStream_t stream;
    CUDA_ASSERT(cudaStreamCreate(&stream));
    cudaEvent_t ev[8];
    for (auto& e : ev) CUDA_ASSERT(cudaEventCreate(&e));
    float best[7];
    for (float& b : best) b = 1e30f;

    for (int rep = 0; rep < reps && !g_ljref_first_error; ++rep) {
        particles.copy(pristine);
        CUDA_ASSERT(cudaDeviceSynchronize());
        CUDA_ASSERT(cudaEventRecord(ev[0]));
        CUDA_ASSERT(cudaMemset(particlePerCells, 0, NbCells * sizeof(int)));
        ComputeNbParticlePerCells<float>
            <<<DefaultNbBlocks, DefaultNbThreads>>>(CellWidth, GridDim, particles, particlePerCells);
        CUDA_ASSERT(cudaEventRecord(ev[1]));
        CUDA_ASSERT(cudaMemset(prefixParCell, 0, (NbCells + 1) * sizeof(int)));
        PrefixFullV2(particlePerCells, prefixParCell + 1, NbCells, stream);
        CUDA_ASSERT(cudaEventRecord(ev[2]));
        CUDA_ASSERT(cudaMemset(dcells, 0, NbCells * sizeof(CellDescriptor)));
        InitNewCells<float><<<DefaultNbBlocks, DefaultNbThreads>>>(prefixParCell, dcells, NbCells);
        CUDA_ASSERT(cudaEventRecord(ev[3]));
        CUDA_ASSERT(cudaMemset(particlePerCells, 0, NbCells * sizeof(int)));
        MoveParticlesToNewCells<float><<<DefaultNbBlocks, DefaultNbThreads>>>(CellWidth, GridDim, particles,
                                                                             particlesSwap, particlePerCells, dcells);
        CUDA_ASSERT(cudaEventRecord(ev[4]));
        CUDA_ASSERT(cudaMemset(cuNb, 0, sizeof(unsigned long long)));
        ComputeNbInteractions<float>
            <<<DefaultNbBlocks, DefaultNbThreads>>>(CellWidth, GridDim, particlesSwap, dcells, cuNb);
        CUDA_ASSERT(cudaEventRecord(ev[5]));
        ComputeParticleInterationsParPartNoLoop<float>
            <<<DefaultNbBlocks, DefaultNbThreads>>>(CellWidth, GridDim, particlesSwap, dcells);
        CUDA_ASSERT(cudaEventRecord(ev[6]));
        CUDA_ASSERT(cudaGetLastError());
        CUDA_ASSERT(cudaDeviceSynchronize());
        if (g_ljref_first_error) break;
        float ms;
        for (int s = 0; s < 6; ++s) {
            CUDA_ASSERT(cudaEventElapsedTime(&ms, ev[s], ev[s + 1]));
            if (ms < best[s]) best[s] = ms;
        }
        CUDA_ASSERT(cudaEventElapsedTime(&ms, ev[0], ev[4]));
        if (ms < best[6]) best[6] = ms;
    }
    if (!g_ljref_first_error) {
        if (counts) {
            // counts were reused as tickets by the scatter (cudaLJ.cu:631); recover them from the prefix
            std::vector<int> p(NbCells + 1);
            CUDA_ASSERT(cudaMemcpy(p.data(), prefixParCell, (NbCells + 1) * sizeof(int), cudaMemcpyDeviceToHost));
            for (long long c = 0; c < NbCells; ++c) counts[c] = p[c + 1] - p[c];
        }
        if (prefix)
            CUDA_ASSERT(cudaMemcpy(prefix, prefixParCell, (NbCells + 1) * sizeof(int), cudaMemcpyDeviceToHost));
        if (cells)
            CUDA_ASSERT(cudaMemcpy(cells, dcells, NbCells * sizeof(CellDescriptor), cudaMemcpyDeviceToHost));
        if (sx) CUDA_ASSERT(cudaMemcpy(sx, particlesSwap.x, n * sizeof(float), cudaMemcpyDeviceToHost));
        if (sy) CUDA_ASSERT(cudaMemcpy(sy, particlesSwap.y, n * sizeof(float), cudaMemcpyDeviceToHost));
        if (sz) CUDA_ASSERT(cudaMemcpy(sz, particlesSwap.z, n * sizeof(float), cudaMemcpyDeviceToHost));
        if (sidx) CUDA_ASSERT(cudaMemcpy(sidx, particlesSwap.index, n * sizeof(int), cudaMemcpyDeviceToHost));
        if (v) CUDA_ASSERT(cudaMemcpy(v, particlesSwap.v, n * sizeof(float), cudaMemcpyDeviceToHost));
        if (nbinter) CUDA_ASSERT(cudaMemcpy(nbinter, cuNb, sizeof(unsigned long long), cudaMemcpyDeviceToHost));
        if (stage_ms)
            for (int s = 0; s < 7; ++s) stage_ms[s] = best[s];
    }
    for (auto& e : ev) cudaEventDestroy(e);
    cudaStreamDestroy(stream);
    deletePtrs(ptrs);
    return g_ljref_first_error ? -3 : 0;
}

}  // extern "C"
