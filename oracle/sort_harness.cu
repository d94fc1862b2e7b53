// sort_harness.cu -- drives the REFERENCE's own spatial sort, reorder() and its key kernel
// count_per_cell (SDK/optixMultiSphereAABB/sort.cu:7-41).
//
// TEST INFRASTRUCTURE ONLY (the checker, never the product).  The Makefile in this directory
// compiles this file against the read-only reference source where it lies, with the flags the
// reference's own build gives it (the SDK's CUDA flags: --use_fast_math -lineinfo), into
// oracle/_ref/libljsortref.so.  No reference source is copied here.
//
// Both entries take host arrays, copy them to the device, run the reference's code and copy the
// result back; CUDA errors are returned, never exit() the process.  count_per_cell writes only the
// .w of the points it is given and thrust sorts a copy, so no input can make them index out of
// bounds.
#include <cstdint>
#include <cstdlib>

#include "sort.cu"

extern "C" {

// The reference's key of every point, in input order: count_per_cell with reorder()'s width
// (int(1.0f / radius), sort.cu:30), without the sort.
int ljsr_keys(int n, const float* host_points, float radius, float* keys) {
    if (n <= 0) return 0;
    float4* h = static_cast<float4*>(std::malloc((size_t)n * sizeof(float4)));
    if (!h) return -1;
    float4* d = nullptr;
    cudaError_t e = cudaMalloc(&d, (size_t)n * sizeof(float4));
    if (e == cudaSuccess) e = cudaMemcpy(d, host_points, (size_t)n * sizeof(float4), cudaMemcpyHostToDevice);
    const int width = 1.0f / radius;
    if (e == cudaSuccess) {
        count_per_cell<<<(n + 255) / 256, 256>>>(n, d, radius, width);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemcpy(h, d, (size_t)n * sizeof(float4), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess)
        for (int i = 0; i < n; ++i) keys[i] = h[i].w;
    cudaFree(d);
    std::free(h);
    return (int)e;
}

// reorder(n, points, radius) on a device copy of host_points; the sorted points come back in place.
int ljsr_reorder(int n, float* host_points, float radius) {
    if (n <= 0) return 0;
    float4* d = nullptr;
    cudaError_t e = cudaMalloc(&d, (size_t)n * sizeof(float4));
    if (e != cudaSuccess) return (int)e;
    e = cudaMemcpy(d, host_points, (size_t)n * sizeof(float4), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        reorder(n, d, radius);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemcpy(host_points, d, (size_t)n * sizeof(float4), cudaMemcpyDeviceToHost);
    cudaFree(d);
    return (int)e;
}

}  // extern "C"
