// generate.cu -- seeded particle generation on the device.
//
// Replaces InitRandStates + InitParticles / InitParticlesSphere
// (cudaLJ.cu:98-105, 174-220).  The reference draws with cuRAND XORWOW on the
// device and with drand48() on its OptiX host path
// (SDK/optixMultiSphere/optixSphere.cpp:132-155).  This file uses the POSIX
// drand48 linear congruential generator (X' = (a X + c) mod 2^48,
// a = 0x5DEECE66D, c = 0xB, srand48(seed): X0 = seed_lo32 << 16 | 0x330E) and
// evaluates it in parallel by jump-ahead: k steps of an affine map are again
// an affine map (A_k, C_k), composed from the precomputed powers 2^b.  Each
// particle consumes its draws in the host generator's order (x, y, z for the
// uniform box; theta then phi for the sphere), so the uniform output is bit
// for bit the sequence srand48(seed); drand48()... produces.
#include "ljcell_internal.cuh"

namespace ljc {

static constexpr unsigned long long kA = 0x5DEECE66DULL;
static constexpr unsigned long long kC = 0xBULL;
static constexpr unsigned long long kM = (1ULL << 48) - 1ULL;

struct JumpTable {
    unsigned long long a[48];
    unsigned long long c[48];
};

struct Affine {
    unsigned long long a, c;
};

// (first f, then g) as one map: x -> g.a (f.a x + f.c) + g.c
static inline Affine compose(Affine f, Affine g) {
    return Affine{(g.a * f.a) & kM, (g.a * f.c + g.c) & kM};
}

static Affine power(unsigned long long k) {
    Affine r{1, 0}, p{kA, kC};
    while (k) {
        if (k & 1) r = compose(r, p);
        p = compose(p, p);
        k >>= 1;
    }
    return r;
}

static JumpTable make_table() {
    JumpTable t;
    Affine p{kA, kC};
    for (int b = 0; b < 48; ++b) {
        t.a[b] = p.a;
        t.c[b] = p.c;
        p = compose(p, p);
    }
    return t;
}

__device__ __forceinline__ unsigned long long lcg_step(unsigned long long s) { return (kA * s + kC) & kM; }

__device__ __forceinline__ unsigned long long jump(unsigned long long s, unsigned long long k, const JumpTable& t) {
    for (int b = 0; k; ++b, k >>= 1)
        if (k & 1) s = (t.a[b] * s + t.c[b]) & kM;
    return s;
}

__device__ __forceinline__ double to_unit(unsigned long long s) { return (double)s * 0x1p-48; }

__global__ void __launch_bounds__(256) k_gen_uniform(unsigned long long x0, JumpTable jt, Affine skip, int n,
                                                     double l0, double l1, double l2, double e0, double e1,
                                                     double e2, float* __restrict__ x, float* __restrict__ y,
                                                     float* __restrict__ z, int* __restrict__ index,
                                                     float* __restrict__ v, float* __restrict__ xyz) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int stride = gridDim.x * blockDim.x;
    if (t >= n) return;
    unsigned long long s = jump(x0, 3ULL * (unsigned long long)t, jt);
    for (int i = t; i < n; i += stride) {
        s = lcg_step(s);
        const double ux = to_unit(s);
        s = lcg_step(s);
        const double uy = to_unit(s);
        s = lcg_step(s);
        const double uz = to_unit(s);
        // lo + (hi - lo) * u with two roundings, as the host computes it
        const float fx = __double2float_rn(__dadd_rn(l0, __dmul_rn(e0, ux)));
        const float fy = __double2float_rn(__dadd_rn(l1, __dmul_rn(e1, uy)));
        const float fz = __double2float_rn(__dadd_rn(l2, __dmul_rn(e2, uz)));
        if (x) x[i] = fx;
        if (y) y[i] = fy;
        if (z) z[i] = fz;
        if (index) index[i] = i;
        if (v) v[i] = -1.0f;
        if (xyz) {
            xyz[3 * (size_t)i + 0] = fx;
            xyz[3 * (size_t)i + 1] = fy;
            xyz[3 * (size_t)i + 2] = fz;
        }
        s = (skip.a * s + skip.c) & kM;
    }
}

__global__ void __launch_bounds__(256) k_gen_sphere(unsigned long long x0, JumpTable jt, Affine skip, int n,
                                                    double cx, double cy, double cz, double r,
                                                    float* __restrict__ x, float* __restrict__ y,
                                                    float* __restrict__ z, int* __restrict__ index,
                                                    float* __restrict__ v, float* __restrict__ xyz) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int stride = gridDim.x * blockDim.x;
    if (t >= n) return;
    unsigned long long s = jump(x0, 2ULL * (unsigned long long)t, jt);
    const double two_pi = 2.0 * 3.14159265358979323846;
    for (int i = t; i < n; i += stride) {
        s = lcg_step(s);
        const double theta = __dmul_rn(two_pi, to_unit(s));
        s = lcg_step(s);
        const double phi = acos(__dsub_rn(1.0, __dmul_rn(2.0, to_unit(s))));
        const double sp = sin(phi), cp = cos(phi), st = sin(theta), ct = cos(theta);
        const float fx = __double2float_rn(__dadd_rn(__dmul_rn(__dmul_rn(r, sp), ct), cx));
        const float fy = __double2float_rn(__dadd_rn(__dmul_rn(__dmul_rn(r, sp), st), cy));
        const float fz = __double2float_rn(__dadd_rn(__dmul_rn(r, cp), cz));
        if (x) x[i] = fx;
        if (y) y[i] = fy;
        if (z) z[i] = fz;
        if (index) index[i] = i;
        if (v) v[i] = -1.0f;
        if (xyz) {
            xyz[3 * (size_t)i + 0] = fx;
            xyz[3 * (size_t)i + 1] = fy;
            xyz[3 * (size_t)i + 2] = fz;
        }
        s = (skip.a * s + skip.c) & kM;
    }
}

static int gen_grid(const lj_ctx* ctx, int n) {
    const int want = (n + 255) / 256;
    const int cap = ctx->sm_count * 8;
    return want < cap ? (want > 0 ? want : 1) : cap;
}

}  // namespace ljc

using namespace ljc;

extern "C" lj_status lj_generate_uniform(lj_ctx* ctx, uint64_t seed, int n, const float lo[3], const float hi[3],
                                         lj_particles* out, float* xyz) {
    if (!ctx || n < 0 || !lo || !hi) return LJ_EINVAL;
    if (n == 0) return LJ_OK;
    lj_particles o{};
    if (out) o = *out;
    static const JumpTable jt = make_table();
    const int blocks = gen_grid(ctx, n);
    const unsigned long long stride = (unsigned long long)blocks * 256ULL;
    const Affine skip = power(3ULL * (stride - 1ULL));
    const unsigned long long x0 = ((unsigned long long)(uint32_t)seed << 16) | 0x330EULL;
    const double l0 = lo[0], l1 = lo[1], l2 = lo[2];
    k_gen_uniform<<<blocks, 256, 0, ctx->stream>>>(x0, jt, skip, n, l0, l1, l2, (double)hi[0] - l0,
                                                   (double)hi[1] - l1, (double)hi[2] - l2, o.x, o.y, o.z, o.index,
                                                   o.v, xyz);
    return last_launch_status();
}

extern "C" lj_status lj_generate_sphere(lj_ctx* ctx, uint64_t seed, int n, const float centre[3], float radius,
                                        lj_particles* out, float* xyz) {
    if (!ctx || n < 0 || !centre) return LJ_EINVAL;
    if (n == 0) return LJ_OK;
    lj_particles o{};
    if (out) o = *out;
    static const JumpTable jt = make_table();
    const int blocks = gen_grid(ctx, n);
    const unsigned long long stride = (unsigned long long)blocks * 256ULL;
    const Affine skip = power(2ULL * (stride - 1ULL));
    const unsigned long long x0 = ((unsigned long long)(uint32_t)seed << 16) | 0x330EULL;
    k_gen_sphere<<<blocks, 256, 0, ctx->stream>>>(x0, jt, skip, n, centre[0], centre[1], centre[2], radius, o.x,
                                                  o.y, o.z, o.index, o.v, xyz);
    return last_launch_status();
}
