// step.cu -- one velocity-Verlet time step of the truncated law, rebinning from the previous sorted
// order (lj_step_verlet).
//
// The reference never moves particles, but its data structures anticipate it: the
// ParticlesContainer swap (cudaLJ.cu:69-76) and the per-particle cuRAND state kept "because we move
// particles randomly" (cudaLJ.cu:96-97).  Here a step is
//
//     v <- v + h F          (h = dt / (2 m), F the forces of the current positions)
//     x <- x + dt v
//     rebin the moved particles, read in the current sorted order (lj_bin, LJ_ORDER_X)
//     carry v and the caller's ids to the new order
//     F <- forces of the new positions (lj_compute)
//     v <- v + h F
//
// Every update is a separate IEEE multiply and add (no contraction), so the drift is reproducible
// bit for bit by a host restatement.  Particles move little between steps, so the previous sorted
// order is nearly the new one and the scatter of the rebinning writes nearly in order.
#include <algorithm>

#include "pair_common.cuh"

namespace ljc {

// Half kick and drift in the current sorted order: new positions into px / py / pz, half-kicked
// velocities into vh, the caller's ids (the .w bits of the records) into ids.
__global__ void __launch_bounds__(256) k_verlet_drift(const float4* __restrict__ rec, const float* __restrict__ vel,
                                                      const float* __restrict__ force, int n, float h, float dt,
                                                      float* __restrict__ px, float* __restrict__ py,
                                                      float* __restrict__ pz, float* __restrict__ vh,
                                                      int* __restrict__ ids) {
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
        const float4 r = rec[s];
        const size_t b = 3 * (size_t)s;
        const float vx = __fadd_rn(vel[b + 0], __fmul_rn(h, force[b + 0]));
        const float vy = __fadd_rn(vel[b + 1], __fmul_rn(h, force[b + 1]));
        const float vz = __fadd_rn(vel[b + 2], __fmul_rn(h, force[b + 2]));
        px[s] = __fadd_rn(r.x, __fmul_rn(dt, vx));
        py[s] = __fadd_rn(r.y, __fmul_rn(dt, vy));
        pz[s] = __fadd_rn(r.z, __fmul_rn(dt, vz));
        vh[b + 0] = vx;
        vh[b + 1] = vy;
        vh[b + 2] = vz;
        ids[s] = __float_as_int(r.w);
    }
}

// After the rebinning, record s' holds in .w the slot o it came from: carry vh[o] and ids[o] over.
__global__ void __launch_bounds__(256) k_verlet_carry(float4* __restrict__ rec, const float* __restrict__ vh,
                                                      const int* __restrict__ ids, int n, float* __restrict__ vel,
                                                      unsigned* status) {
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
        float4 r = rec[s];
        int o = __float_as_int(r.w);
        if (o < 0 || o >= n) {
            atomicOr(status, kFlagRange);
            o = 0;
        }
        const size_t a = 3 * (size_t)s, b = 3 * (size_t)o;
        vel[a + 0] = vh[b + 0];
        vel[a + 1] = vh[b + 1];
        vel[a + 2] = vh[b + 2];
        r.w = __int_as_float(ids[o]);
        rec[s] = r;
    }
}

// Second half kick with the new forces.
__global__ void __launch_bounds__(256) k_verlet_kick(const float* __restrict__ force, int n3, float h,
                                                     float* __restrict__ vel) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n3; i += gridDim.x * blockDim.x)
        vel[i] = __fadd_rn(vel[i], __fmul_rn(h, force[i]));
}

}  // namespace ljc

using namespace ljc;

extern "C" lj_status lj_step_verlet(lj_ctx* ctx, const lj_grid* g, const lj_params* p, int n, float dt, float mass,
                                    float* xyzi, float* vel, float* force, int* sorted_cell, int* counts, int* offsets,
                                    float* energy, lj_totals* totals) {
    const NvtxRange nvtx_range("lj_step_verlet");
    if (!ctx || !g || !p || n < 0 || !counts || !offsets) return LJ_EINVAL;
    if (n > 0 && (!xyzi || !vel || !force || !sorted_cell)) return LJ_EINVAL;
    if (!(dt > 0.0f) || !(mass > 0.0f) || !(dt < 3.4e38f) || !(mass < 3.4e38f)) return LJ_EINVAL;
    if (reinterpret_cast<uintptr_t>(xyzi) & 15) return LJ_EINVAL;
    const float h = 0.5f * dt / mass;
    lj_status s;
    // scratch: px, py, pz (3n floats), vh (3n floats), ids (n ints)
    const size_t nn = (size_t)(n > 0 ? n : 1);
    if ((s = grow(&ctx->step, &ctx->step_bytes, nn * 7 * sizeof(float))) != LJ_OK) return s;
    float* px = static_cast<float*>(ctx->step);
    float* py = px + nn;
    float* pz = py + nn;
    float* vh = pz + nn;
    int* ids = reinterpret_cast<int*>(vh + 3 * nn);
    float4* rec = reinterpret_cast<float4*>(xyzi);
    const int blocks = std::max(1, std::min((n + 255) / 256, ctx->sm_count * 8));
    if (n > 0) {
        k_verlet_drift<<<blocks, 256, 0, ctx->stream>>>(rec, vel, force, n, h, dt, px, py, pz, vh, ids);
        if ((s = last_launch_status()) != LJ_OK) return s;
    }
    if ((s = lj_bin(ctx, g, n, px, py, pz, 1, LJ_ORDER_X, counts, offsets, nullptr, nullptr, xyzi, sorted_cell)) !=
        LJ_OK)
        return s;
    if (n > 0) {
        k_verlet_carry<<<blocks, 256, 0, ctx->stream>>>(rec, vh, ids, n, vel, ctx->d_status);
        if ((s = last_launch_status()) != LJ_OK) return s;
    }
    if ((s = lj_compute(ctx, g, p, n, xyzi, sorted_cell, offsets, LJ_ORDER_X, energy, force, totals)) != LJ_OK)
        return s;
    if (n > 0) {
        const int n3 = 3 * n;
        k_verlet_kick<<<std::max(1, std::min((n3 + 255) / 256, ctx->sm_count * 8)), 256, 0, ctx->stream>>>(
            force, n3, h, vel);
        if ((s = last_launch_status()) != LJ_OK) return s;
    }
    return LJ_OK;
}
