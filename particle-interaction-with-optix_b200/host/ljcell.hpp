// ljcell.hpp -- C++17 host layer over the C ABI (include/ljcell.h).
//
// Mirrors the host-side interface of the reference's cell-grid path
// (OptixLJ Cuda-version/cudaLJ.cu) so that C++ callers of that code find the
// same shapes:
//   ljcell::ParticlesContainer<float>  == ParticlesContainer<float>  (cudaLJ.cu:60-86)
//   ljcell::CellDescriptor             == CellDescriptor             (cudaLJ.cu:91-94)
//   ljcell::executeSimulation<float>() == executeSimulation<float>() (cudaLJ.cu:515-677),
//       same arguments and return value (candidate-interaction count and the
//       per-loop init / compute / total times), same console report.
// Differences, by design: errors throw ljcell::Error instead of exit(1)
// (cudaLJ.cu:17-26); timings are CUDA events on the context stream; the init
// time includes the scatter kernel that the reference's timer misses
// (cudaLJ.cu:632-635); positions come from the drand48 generator of
// include/ljcell.h instead of cuRAND.
#pragma once

#include <cuda_runtime.h>

#include <cstdio>
#include <iostream>
#include <stdexcept>
#include <string>
#include <tuple>
#include <utility>
#include <vector>

#include "ljcell.h"

namespace ljcell {

struct Error : std::runtime_error {
    lj_status status;
    Error(lj_status s, const std::string& where)
        : std::runtime_error(where + ": " + lj_status_str(s)), status(s) {}
};

inline void check(lj_status s, const char* where) {
    if (s != LJ_OK) throw Error(s, where);
}

inline void check_cuda(cudaError_t e, const char* where) {
    if (e != cudaSuccess) throw std::runtime_error(std::string(where) + ": " + cudaGetErrorString(e));
}

// Owning device allocation.
template <class T>
class DeviceBuffer {
   public:
    DeviceBuffer() = default;
    explicit DeviceBuffer(size_t n) : n_(n) {
        if (n) check_cuda(cudaMalloc(&p_, n * sizeof(T)), "cudaMalloc");
    }
    ~DeviceBuffer() {
        if (p_) cudaFree(p_);
    }
    DeviceBuffer(DeviceBuffer&& o) noexcept : p_(o.p_), n_(o.n_) { o.p_ = nullptr, o.n_ = 0; }
    DeviceBuffer& operator=(DeviceBuffer&& o) noexcept {
        std::swap(p_, o.p_);
        std::swap(n_, o.n_);
        return *this;
    }
    DeviceBuffer(const DeviceBuffer&) = delete;
    DeviceBuffer& operator=(const DeviceBuffer&) = delete;
    T* get() const { return p_; }
    size_t size() const { return n_; }

   private:
    T* p_ = nullptr;
    size_t n_ = 0;
};

// == ParticlesContainer<FloatType> (cudaLJ.cu:60-86), owning its arrays.
template <typename FloatType>
struct ParticlesContainer;

template <>
struct ParticlesContainer<float> {
    float* x = nullptr;
    float* y = nullptr;
    float* z = nullptr;
    float* v = nullptr;
    int* index = nullptr;
    int nbParticles = 0;

    void swap(ParticlesContainer& o) {
        std::swap(x, o.x);
        std::swap(y, o.y);
        std::swap(z, o.z);
        std::swap(v, o.v);
        std::swap(index, o.index);
        std::swap(nbParticles, o.nbParticles);
        std::swap(storage_, o.storage_);
    }
    lj_particles view() const { return lj_particles{x, y, z, v, index, nbParticles}; }

    static ParticlesContainer allocate(int n) {
        ParticlesContainer p;
        p.storage_ = DeviceBuffer<float>((size_t)5 * (n > 0 ? n : 1));
        float* b = p.storage_.get();
        const size_t s = (size_t)(n > 0 ? n : 1);
        p.x = b;
        p.y = b + s;
        p.z = b + 2 * s;
        p.v = b + 3 * s;
        p.index = reinterpret_cast<int*>(b + 4 * s);
        p.nbParticles = n;
        return p;
    }

   private:
    DeviceBuffer<float> storage_;
};

using CellDescriptor = lj_cell_desc;

// RAII context.
class Context {
   public:
    explicit Context(int device = 0, cudaStream_t stream = nullptr) {
        check(lj_create(&ctx_, device, stream), "lj_create");
    }
    ~Context() {
        if (ctx_) lj_destroy(ctx_);
    }
    Context(const Context&) = delete;
    Context& operator=(const Context&) = delete;
    lj_ctx* get() const { return ctx_; }
    void sync() const { check(lj_sync(ctx_), "lj_sync"); }

   private:
    lj_ctx* ctx_ = nullptr;
};

// One binned system on the device: the product of the cell-grid build.
struct CellGrid {
    lj_grid grid{};
    long long ncells = 0;
    DeviceBuffer<int> counts, offsets, sorted_cell;
    DeviceBuffer<CellDescriptor> cells;
    DeviceBuffer<float> xyzi;  // 4 floats per particle

    CellGrid(const lj_grid& g, int n) : grid(g) {
        ncells = (long long)g.dim[0] * g.dim[1] * g.dim[2];
        counts = DeviceBuffer<int>((size_t)ncells);
        offsets = DeviceBuffer<int>((size_t)ncells + 1);
        cells = DeviceBuffer<CellDescriptor>((size_t)ncells);
        sorted_cell = DeviceBuffer<int>((size_t)(n > 0 ? n : 1));
        xyzi = DeviceBuffer<float>((size_t)4 * (n > 0 ? n : 1));
    }
};

struct AResult {
    double timeInit;
    double timeCompute;
    double timeTotal;
};

// Seconds between two events recorded on one stream.
class StageTimer {
   public:
    StageTimer() {
        check_cuda(cudaEventCreate(&a_), "cudaEventCreate");
        check_cuda(cudaEventCreate(&b_), "cudaEventCreate");
    }
    ~StageTimer() {
        cudaEventDestroy(a_);
        cudaEventDestroy(b_);
    }
    void start(cudaStream_t s) { check_cuda(cudaEventRecord(a_, s), "cudaEventRecord"); }
    void stop(cudaStream_t s) { check_cuda(cudaEventRecord(b_, s), "cudaEventRecord"); }
    double seconds() {
        check_cuda(cudaEventSynchronize(b_), "cudaEventSynchronize");
        float ms = 0;
        check_cuda(cudaEventElapsedTime(&ms, a_, b_), "cudaEventElapsedTime");
        return ms * 1e-3;
    }

   private:
    cudaEvent_t a_, b_;
};

// The reference's experiment (cudaLJ.cu:515-677): `inNbLoops` times generate
// particles, build the cell grid (timed as init), count candidate
// interactions (untimed), evaluate the reference law (timed as compute).
// Returns the summed candidate-interaction count and one AResult per loop.
// `inCheckResult` compares the binning to the CPU rule it restates
// (per-cell counts sum to N) -- the reference accepted and ignored it.
template <typename NumType = float>
std::tuple<unsigned long long, std::vector<AResult>> executeSimulation(const int inNbParticles, const int inNbLoops,
                                                                       const NumType boxWidth1Dim,
                                                                       const NumType inCutoff,
                                                                       const bool inCheckResult,
                                                                       const bool gensurface, int device = 0,
                                                                       bool verbose = true) {
    static_assert(std::is_same<NumType, float>::value, "the B200 path computes in float");
    Context ctx(device);
    lj_grid g;
    check(lj_grid_compat(boxWidth1Dim, inCutoff, &g), "lj_grid_compat");
    const long long NbCells = (long long)g.dim[0] * g.dim[1] * g.dim[2];
    if (verbose) {
        std::cout << "Start Execution" << std::endl;
        std::cout << " - gensurface: " << gensurface << std::endl;
        std::cout << " - NbParticles: " << inNbParticles << std::endl;
        std::cout << " - NbLoops: " << inNbLoops << std::endl;
        std::cout << " - Cutoff: " << inCutoff << std::endl;
        std::cout << " - Space box dimension: " << boxWidth1Dim << std::endl;
        std::cout << " - Space grid dimension: " << g.dim[0] << " / " << g.dim[1] << " / " << g.dim[2] << std::endl;
        std::cout << " - Number of cells: " << NbCells << std::endl;
        std::cout << " - Avergage particles per cell: " << double(inNbParticles) / NbCells << std::endl;
    }
    const int NbFlopsPerInteraction = 18;  // the reference's constant, cudaLJ.cu:550
    ParticlesContainer<float> particles = ParticlesContainer<float>::allocate(inNbParticles);
    ParticlesContainer<float> particlesSwap = ParticlesContainer<float>::allocate(inNbParticles);
    CellGrid grid(g, inNbParticles);
    DeviceBuffer<unsigned long long> cuNb(1);
    std::vector<AResult> results;
    unsigned long long NbInteractions = 0;
    StageTimer initTimer, computeTimer;
    double cumInit = 0, cumCompute = 0;
    for (int loop = 0; loop < inNbLoops; ++loop) {
        lj_particles pv = particles.view();
        if (gensurface) {
            // the reference's sphere: unit radius, centre (1, 1, 1) in [0, 2)^3 (cudaLJ.cu:197-220)
            const float centre[3] = {1.f, 1.f, 1.f};
            check(lj_generate_sphere(ctx.get(), 1234 + loop, inNbParticles, centre, 1.0f, &pv, nullptr),
                  "lj_generate_sphere");
        } else {
            const float lo[3] = {0.f, 0.f, 0.f};
            const float hi[3] = {boxWidth1Dim, boxWidth1Dim, boxWidth1Dim};
            check(lj_generate_uniform(ctx.get(), 1234 + loop, inNbParticles, lo, hi, &pv, nullptr),
                  "lj_generate_uniform");
        }
        ctx.sync();
        initTimer.start(nullptr);
        lj_particles sv = particlesSwap.view();
        check(lj_bin(ctx.get(), &g, inNbParticles, particles.x, particles.y, particles.z, 1, LJ_ORDER_INDEX,
                     grid.counts.get(), grid.offsets.get(), grid.cells.get(), &sv, grid.xyzi.get(),
                     grid.sorted_cell.get()),
              "lj_bin");
        initTimer.stop(nullptr);
        particlesSwap.swap(particles);
        check(lj_count_candidates(ctx.get(), &g, grid.offsets.get(), cuNb.get()), "lj_count_candidates");
        unsigned long long newNb = 0;
        check_cuda(cudaMemcpy(&newNb, cuNb.get(), sizeof(newNb), cudaMemcpyDeviceToHost), "cudaMemcpy");
        NbInteractions += newNb;
        computeTimer.start(nullptr);
        check(lj_compute_compat(ctx.get(), &g, inNbParticles, grid.xyzi.get(), grid.sorted_cell.get(),
                                grid.offsets.get(), particles.v),
              "lj_compute_compat");
        computeTimer.stop(nullptr);
        ctx.sync();
        const double ti = initTimer.seconds(), tc = computeTimer.seconds();
        cumInit += ti;
        cumCompute += tc;
        results.push_back(AResult{ti, tc, ti + tc});
        if (inCheckResult) {
            std::vector<int> off((size_t)NbCells + 1);
            check_cuda(cudaMemcpy(off.data(), grid.offsets.get(), off.size() * sizeof(int), cudaMemcpyDeviceToHost),
                       "cudaMemcpy");
            if (off[0] != 0 || off[NbCells] != inNbParticles) throw Error(LJ_ERANGE, "binning check");
        }
    }
    if (verbose) {
        std::cout << " - Nb interactions: " << NbInteractions << std::endl;
        std::cout << " - Time init: " << cumInit << "s" << std::endl;
        std::cout << " - Time compute: " << cumCompute << "s" << std::endl;
        std::cout << " - Total: " << (cumInit + cumCompute) << "s" << std::endl;
        std::cout << " - GFlops/s: " << (NbInteractions * double(NbFlopsPerInteraction)) / (cumInit + cumCompute) / 1e9
                  << std::endl;
        std::cout << "     - Compute only GFlops/s: "
                  << (NbInteractions * double(NbFlopsPerInteraction)) / cumCompute / 1e9 << std::endl;
        std::cout << " - Interactions/s: " << NbInteractions / (cumInit + cumCompute) << std::endl;
    }
    return std::make_tuple(NbInteractions, std::move(results));
}

}  // namespace ljcell
