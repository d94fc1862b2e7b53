// api.cu -- context, scratch memory, status and the end-to-end entry of the C ABI.
#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>

#include "ljcell_internal.cuh"

namespace ljc {

namespace {
// Test hook (lj_test_fail_alloc): the number of scratch growths until one is made to fail; 0 = off.
std::atomic<int> g_fail_alloc{0};
}  // namespace

// Grows a scratch buffer to at least `need` bytes.  On failure *p is null and *cap 0 (the old
// buffer is already freed), so the caller's next call grows it again.
lj_status grow(void** p, size_t* cap, size_t need) {
    if (need <= *cap && *p) return LJ_OK;
    if (*p) {
        cudaFree(*p);
        *p = nullptr;
        *cap = 0;
    }
    int left = g_fail_alloc.load();
    while (left > 0 && !g_fail_alloc.compare_exchange_weak(left, left - 1)) {
    }
    if (left == 1) return LJ_ENOMEM;  // the growth the test hook selected
    size_t want = need + need / 8 + 256;
    if (cudaMalloc(p, want) != cudaSuccess) {
        cudaGetLastError();
        *p = nullptr;
        return LJ_ENOMEM;
    }
    *cap = want;
    return LJ_OK;
}

lj_status last_launch_status() {
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? LJ_OK : LJ_ECUDA;
}

// Switches to the context's device for the duration of one API call.
struct DeviceScope {
    int prev = -1;
    bool ok = true;
    explicit DeviceScope(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) {
            ok = false;
            return;
        }
        if (prev != dev && cudaSetDevice(dev) != cudaSuccess) ok = false;
    }
    ~DeviceScope() {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

}  // namespace ljc

using namespace ljc;

extern "C" int lj_abi_version(void) { return LJCELL_ABI_VERSION; }

extern "C" lj_status lj_test_fail_alloc(int k) {
    if (k < 0) return LJ_EINVAL;
    g_fail_alloc.store(k);
    return LJ_OK;
}

extern "C" const char* lj_status_str(lj_status s) {
    switch (s) {
        case LJ_OK: return "ok";
        case LJ_EINVAL: return "invalid argument";
        case LJ_ENOMEM: return "device allocation failed";
        case LJ_ECUDA: return "CUDA runtime error";
        case LJ_ETIMEOUT: return "bounded device wait timed out";
        case LJ_ERANGE: return "non-finite coordinate or out-of-range index";
        case LJ_EUNSUPPORTED: return "unsupported size or mode";
        case LJ_ECHECK: return "consistency check failed (-DLJ_CHECKS build)";
    }
    return "unknown status";
}

extern "C" lj_status lj_create(lj_ctx** out, int device, void* stream) {
    if (!out) return LJ_EINVAL;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess) {
        cudaGetLastError();
        return LJ_ECUDA;
    }
    if (device < 0 || device >= ndev) return LJ_EINVAL;
    DeviceScope scope(device);
    if (!scope.ok) return LJ_ECUDA;
    lj_ctx* c = new (std::nothrow) lj_ctx();
    if (!c) return LJ_ENOMEM;
    std::memset(c, 0, sizeof(*c));
    c->device = device;
    c->stream = static_cast<cudaStream_t>(stream);
    if (cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) {
        delete c;
        return LJ_ECUDA;
    }
    if (cudaMalloc(&c->d_status, 256) != cudaSuccess || cudaMemset(c->d_status, 0, 256) != cudaSuccess) {
        cudaGetLastError();
        delete c;
        return LJ_ENOMEM;
    }
    c->d_cand = reinterpret_cast<unsigned long long*>(reinterpret_cast<char*>(c->d_status) + 64);
    *out = c;
    return LJ_OK;
}

extern "C" lj_status lj_destroy(lj_ctx* c) {
    if (!c) return LJ_EINVAL;
    DeviceScope scope(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    else cudaDeviceSynchronize();
    cudaFree(c->d_status);
    cudaFree(c->scan_state);
    cudaFree(c->cell_ticket);
    cudaFree(c->tmp4);
    cudaFree(c->large_cells);
    cudaFree(c->red);
    cudaFree(c->e2e);
    cudaFree(c->reorder);
    cudaFree(c->step);
    cudaFree(c->half);
    cudaFree(c->sel);
    cudaFree(c->check);
    cudaFree(c->cellpair);
    if (c->e2ea_ready) {
        cudaStreamSynchronize(c->up_stream);
        for (int i = 0; i < kE2EASlots + 7; ++i) cudaEventDestroy(c->e2ea_ev[i]);
        cudaStreamDestroy(c->up_stream);
    }
    if (c->e2ea_tot) {
        if (c->e2e_ready) cudaStreamSynchronize(c->copy_stream);
        cudaFreeHost(c->e2ea_tot);
    }
    if (c->e2e_ready) {
        cudaStreamSynchronize(c->copy_stream);
        for (int i = 0; i < 8; ++i) cudaEventDestroy(c->e2e_ev[i]);
        cudaStreamDestroy(c->copy_stream);
    }
    for (int i = 0; i < kE2EASlots; ++i) cudaFree(c->e2ea[i]);
    delete c;
    return LJ_OK;
}

extern "C" lj_status lj_set_stream(lj_ctx* c, void* stream) {
    if (!c) return LJ_EINVAL;
    c->stream = static_cast<cudaStream_t>(stream);
    return LJ_OK;
}

extern "C" lj_status lj_set_tuning(lj_ctx* c, const lj_tuning* t) {
    if (!c || !t || t->pair_kernel < 0 || t->pair_kernel > 12 || t->scatter_passes < 0 || t->scatter_passes > 8)
        return LJ_EINVAL;
    c->tuning = *t;
    return LJ_OK;
}

extern "C" lj_status lj_get_tuning(lj_ctx* c, lj_tuning* t) {
    if (!c || !t) return LJ_EINVAL;
    *t = c->tuning;
    return LJ_OK;
}

extern "C" lj_status lj_sync(lj_ctx* c) {
    if (!c) return LJ_EINVAL;
    DeviceScope scope(c->device);
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) return LJ_ECUDA;
    unsigned flags = 0;
    if (cudaMemcpy(&flags, c->d_status, sizeof(unsigned), cudaMemcpyDeviceToHost) != cudaSuccess) return LJ_ECUDA;
    if (flags) {
        if (cudaMemset(c->d_status, 0, sizeof(unsigned)) != cudaSuccess) return LJ_ECUDA;
        if (flags & kFlagTimeout) return LJ_ETIMEOUT;
        if (flags & kFlagCheck) return LJ_ECHECK;
        return LJ_ERANGE;
    }
    return LJ_OK;
}

extern "C" lj_status lj_grid_from_box(const float lo[3], const float hi[3], float cutoff, lj_grid* out) {
    if (!lo || !hi || !out || !(cutoff > 0.0f)) return LJ_EINVAL;
    lj_grid g;
    for (int d = 0; d < 3; ++d) {
        const float ext = hi[d] - lo[d];
        if (!(ext > 0.0f)) return LJ_EINVAL;
        const float q = ext / cutoff;
        if (!(q < 2147483647.0f)) return LJ_EUNSUPPORTED;
        const int G = static_cast<int>(q);
        g.dim[d] = G < 1 ? 1 : G;
        g.origin[d] = lo[d];
    }
    g.width = cutoff;
    if ((long long)g.dim[0] * g.dim[1] * g.dim[2] > 2147483646LL) return LJ_EUNSUPPORTED;
    *out = g;
    return LJ_OK;
}

extern "C" lj_status lj_grid_compat(float box_width, float cutoff, lj_grid* out) {
    const float lo[3] = {0.f, 0.f, 0.f};
    const float hi[3] = {box_width, box_width, box_width};
    return lj_grid_from_box(lo, hi, cutoff, out);
}

namespace ljc {

// The pair stage of lj_simulate_host runs in this many target chunks, so that each chunk's
// device-to-host copy of energy / force overlaps the next chunk's compute.
constexpr int kE2EChunks = 4;

// Totals of the chunks, summed in chunk order (deterministic).
__global__ void k_sum_totals(const lj_totals* __restrict__ part, int nparts, lj_totals* __restrict__ out) {
    double e = 0.0, w = 0.0;
    unsigned long long np = 0;
    for (int i = 0; i < nparts; ++i) {
        e += part[i].energy;
        w += part[i].virial;
        np += part[i].pairs;
    }
    *out = lj_totals{e, w, np, 0ULL};
}

lj_status e2e_setup(lj_ctx* c) {
    if (c->e2e_ready) return LJ_OK;
    if (cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking) != cudaSuccess) return LJ_ECUDA;
    for (int i = 0; i < 8; ++i)
        if (cudaEventCreateWithFlags(&c->e2e_ev[i], cudaEventDisableTiming) != cudaSuccess) {
            for (int j = 0; j < i; ++j) cudaEventDestroy(c->e2e_ev[j]);
            cudaStreamDestroy(c->copy_stream);
            c->copy_stream = nullptr;
            return LJ_ECUDA;
        }
    c->e2e_ready = true;
    return LJ_OK;
}

}  // namespace ljc

extern "C" lj_status lj_simulate_host(lj_ctx* c, const lj_grid* g, const lj_params* p, int n, const float* hx,
                                      const float* hy, const float* hz, float* h_energy, float* h_force,
                                      int* h_index, lj_totals* h_totals) {
    const NvtxRange nvtx_range("lj_simulate_host");
    if (!c || !g || !p || n < 0 || (n > 0 && (!hx || !hy || !hz))) return LJ_EINVAL;
    if (!(g->width > 0.0f) || g->dim[0] < 1 || g->dim[1] < 1 || g->dim[2] < 1) return LJ_EINVAL;
    if (!(p->cutoff > 0.0f) || !(p->cutoff <= g->width) || !(p->sigma > 0.0f)) return LJ_EINVAL;
    DeviceScope scope(c->device);
    if (!scope.ok) return LJ_ECUDA;
    const long long nc = (long long)g->dim[0] * g->dim[1] * g->dim[2];
    if (nc < 1 || nc > 2147483646LL) return LJ_EINVAL;
    lj_status s = e2e_setup(c);
    if (s != LJ_OK) return s;
    const size_t N = (size_t)(n > 0 ? n : 1);
    auto up = [](size_t b) { return (b + 255) & ~(size_t)255; };
    const size_t b_pos = up(3 * N * sizeof(float));
    const size_t b_cnt = up((size_t)nc * sizeof(int));
    const size_t b_off = up(((size_t)nc + 1) * sizeof(int));
    const size_t b_x4 = up(N * 16);
    const size_t b_cell = up(N * sizeof(int));
    const size_t b_e = up(N * sizeof(float));
    const size_t b_f = up(3 * N * sizeof(float));
    const size_t b_idx = up(N * sizeof(int));
    const size_t b_tot = up((kE2EChunks + 1) * sizeof(lj_totals));
    const size_t need = b_pos + b_cnt + b_off + b_x4 + b_cell + b_e + b_f + b_idx + b_tot;
    s = grow(&c->e2e, &c->e2e_bytes, need);
    if (s != LJ_OK) return s;
    char* base = static_cast<char*>(c->e2e);
    float* dpos = reinterpret_cast<float*>(base);
    base += b_pos;
    int* dcnt = reinterpret_cast<int*>(base);
    base += b_cnt;
    int* doff = reinterpret_cast<int*>(base);
    base += b_off;
    float* dx4 = reinterpret_cast<float*>(base);
    base += b_x4;
    int* dcell = reinterpret_cast<int*>(base);
    base += b_cell;
    float* de = reinterpret_cast<float*>(base);
    base += b_e;
    float* df = reinterpret_cast<float*>(base);
    base += b_f;
    int* didx = reinterpret_cast<int*>(base);
    base += b_idx;
    lj_totals* dtot = reinterpret_cast<lj_totals*>(base);
    cudaStream_t st = c->stream, cp = c->copy_stream;
    // every return leaves no copy in flight into the caller's host buffers
    struct Drain {
        cudaStream_t s;
        ~Drain() { cudaStreamSynchronize(s); }
    } drain{cp};
    const size_t pb = (size_t)n * sizeof(float);
    if (n > 0) {
        if (cudaMemcpyAsync(dpos, hx, pb, cudaMemcpyHostToDevice, st) != cudaSuccess ||
            cudaMemcpyAsync(dpos + N, hy, pb, cudaMemcpyHostToDevice, st) != cudaSuccess ||
            cudaMemcpyAsync(dpos + 2 * N, hz, pb, cudaMemcpyHostToDevice, st) != cudaSuccess)
            return LJ_ECUDA;
    }
    lj_particles sorted{};
    sorted.index = didx;
    s = lj_bin(c, g, n, dpos, dpos + N, dpos + 2 * N, 1, LJ_ORDER_X, dcnt, doff, nullptr, &sorted, dx4, dcell);
    if (s != LJ_OK) return s;
    // The index is final once binning is done: copy it back while the pair stage runs.
    if (cudaEventRecord(c->e2e_ev[0], st) != cudaSuccess || cudaStreamWaitEvent(cp, c->e2e_ev[0], 0) != cudaSuccess)
        return LJ_ECUDA;
    if (n > 0 && h_index &&
        cudaMemcpyAsync(h_index, didx, (size_t)n * sizeof(int), cudaMemcpyDeviceToHost, cp) != cudaSuccess)
        return LJ_ECUDA;
    // Pair stage in target chunks; chunk k's outputs go back on the copy stream during chunk k + 1.
    const int chunks = n < kE2EChunks * 4096 ? 1 : kE2EChunks;
    for (int k = 0; k < chunks; ++k) {
        const int kb = (int)((long long)n * k / chunks), ke = (int)((long long)n * (k + 1) / chunks);
        s = launch_pair_config(c, g, p, n, dx4, dcell, doff, LJ_ORDER_X, h_energy ? de : nullptr,
                               h_force ? df : nullptr, dtot + k, kb, ke);
        if (s != LJ_OK) return s;
        if (ke == kb) continue;
        if (cudaEventRecord(c->e2e_ev[1 + k], st) != cudaSuccess ||
            cudaStreamWaitEvent(cp, c->e2e_ev[1 + k], 0) != cudaSuccess)
            return LJ_ECUDA;
        const size_t cb = (size_t)(ke - kb) * sizeof(float);
        if (h_energy && cudaMemcpyAsync(h_energy + kb, de + kb, cb, cudaMemcpyDeviceToHost, cp) != cudaSuccess)
            return LJ_ECUDA;
        if (h_force &&
            cudaMemcpyAsync(h_force + 3 * (size_t)kb, df + 3 * (size_t)kb, 3 * cb, cudaMemcpyDeviceToHost, cp) !=
                cudaSuccess)
            return LJ_ECUDA;
    }
    k_sum_totals<<<1, 1, 0, st>>>(dtot, chunks, dtot + kE2EChunks);
    if ((s = last_launch_status()) != LJ_OK) return s;
    if (h_totals &&
        cudaMemcpyAsync(h_totals, dtot + kE2EChunks, sizeof(lj_totals), cudaMemcpyDeviceToHost, st) != cudaSuccess)
        return LJ_ECUDA;
    if (cudaStreamSynchronize(cp) != cudaSuccess) return LJ_ECUDA;
    return lj_sync(c);
}

namespace ljc {

constexpr int kE2EAPending = 64;  // queued lj_simulate_host_async calls whose totals await the wait call

// Copies the staged totals of the queued calls to their callers (after the copy stream is drained).
void e2ea_deliver(lj_ctx* c) {
    for (int i = 0; i < c->e2ea_pending; ++i)
        if (c->e2ea_dst[i]) *c->e2ea_dst[i] = c->e2ea_tot[i];
    c->e2ea_pending = 0;
}

lj_status e2ea_setup(lj_ctx* c) {
    if (c->e2ea_ready) return LJ_OK;
    if (cudaStreamCreateWithFlags(&c->up_stream, cudaStreamNonBlocking) != cudaSuccess) return LJ_ECUDA;
    for (int i = 0; i < kE2EASlots + 7; ++i)
        if (cudaEventCreateWithFlags(&c->e2ea_ev[i], cudaEventDisableTiming) != cudaSuccess) {
            for (int j = 0; j < i; ++j) cudaEventDestroy(c->e2ea_ev[j]);
            cudaStreamDestroy(c->up_stream);
            c->up_stream = nullptr;
            return LJ_ECUDA;
        }
    // every slot starts free
    for (int i = 0; i < kE2EASlots; ++i)
        if (cudaEventRecord(c->e2ea_ev[i], c->up_stream) != cudaSuccess) return LJ_ECUDA;
    // totals come back into pinned memory (a copy into pageable memory would make the call wait for
    // the whole step); lj_simulate_host_wait hands them to the caller
    if (cudaMallocHost(reinterpret_cast<void**>(&c->e2ea_tot), kE2EAPending * sizeof(lj_totals)) != cudaSuccess) {
        c->e2ea_tot = nullptr;
        return LJ_ENOMEM;
    }
    c->e2ea_pending = 0;
    c->e2ea_ready = true;
    return LJ_OK;
}

}  // namespace ljc

namespace ljc {

// One queued host-buffer step (lj_simulate_host_async and lj_simulate_host_inorder_async).
// inorder: the pair kernel writes energy and force at each particle's original index (the caller's
// order, no index array), and they come back after the whole pair stage; otherwise in sorted order,
// each target chunk's results during the next chunk.
lj_status simulate_async(lj_ctx* c, const lj_grid* g, const lj_params* p, int n, const float* hx, const float* hy,
                         const float* hz, float* h_energy, float* h_force, int* h_index, lj_totals* h_totals,
                         bool inorder) {
    if (!c || !g || !p || n < 0 || (n > 0 && (!hx || !hy || !hz))) return LJ_EINVAL;
    if (!(g->width > 0.0f) || g->dim[0] < 1 || g->dim[1] < 1 || g->dim[2] < 1) return LJ_EINVAL;
    if (!(p->cutoff > 0.0f) || !(p->cutoff <= g->width) || !(p->sigma > 0.0f)) return LJ_EINVAL;
    DeviceScope scope(c->device);
    if (!scope.ok) return LJ_ECUDA;
    const long long nc = (long long)g->dim[0] * g->dim[1] * g->dim[2];
    if (nc < 1 || nc > 2147483646LL) return LJ_EINVAL;
    lj_status s = e2e_setup(c);
    if (s != LJ_OK) return s;
    if ((s = e2ea_setup(c)) != LJ_OK) return s;
    if (c->e2ea_pending == kE2EAPending) {  // staging full: drain the queued calls first
        if (cudaStreamSynchronize(c->copy_stream) != cudaSuccess) return LJ_ECUDA;
        e2ea_deliver(c);
    }
    const int slot = c->e2ea_slot;
    cudaStream_t st = c->stream, cp = c->copy_stream, up = c->up_stream;
    cudaEvent_t* ev = c->e2ea_ev;
    // Nothing may touch this slot's buffers (grown or not) before its last download is done.
    if (cudaStreamWaitEvent(up, ev[slot], 0) != cudaSuccess || cudaStreamWaitEvent(st, ev[slot], 0) != cudaSuccess)
        return LJ_ECUDA;
    const size_t N = (size_t)(n > 0 ? n : 1);
    auto upb = [](size_t b) { return (b + 255) & ~(size_t)255; };
    const size_t b_pos = upb(3 * N * sizeof(float));
    const size_t b_cnt = upb((size_t)nc * sizeof(int));
    const size_t b_off = upb(((size_t)nc + 1) * sizeof(int));
    const size_t b_x4 = upb(N * 16);
    const size_t b_cell = upb(N * sizeof(int));
    const size_t b_e = upb(N * sizeof(float));
    const size_t b_f = upb(3 * N * sizeof(float));
    const size_t b_idx = upb(N * sizeof(int));
    const size_t b_tot = upb((kE2EChunks + 1) * sizeof(lj_totals));
    const size_t need = b_pos + b_cnt + b_off + b_x4 + b_cell + b_e + b_f + b_idx + b_tot;
    if (need > c->e2ea_bytes[slot]) {
        // a grown slot: wait for its previous download on the host before freeing it
        if (cudaEventSynchronize(ev[slot]) != cudaSuccess) return LJ_ECUDA;
        if ((s = grow(&c->e2ea[slot], &c->e2ea_bytes[slot], need)) != LJ_OK) return s;
    }
    char* base = static_cast<char*>(c->e2ea[slot]);
    float* dpos = reinterpret_cast<float*>(base);
    base += b_pos;
    int* dcnt = reinterpret_cast<int*>(base);
    base += b_cnt;
    int* doff = reinterpret_cast<int*>(base);
    base += b_off;
    float* dx4 = reinterpret_cast<float*>(base);
    base += b_x4;
    int* dcell = reinterpret_cast<int*>(base);
    base += b_cell;
    float* de = reinterpret_cast<float*>(base);
    base += b_e;
    float* df = reinterpret_cast<float*>(base);
    base += b_f;
    int* didx = reinterpret_cast<int*>(base);
    base += b_idx;
    lj_totals* dtot = reinterpret_cast<lj_totals*>(base);
    // upload on its own stream: it overlaps the previous call's compute and downloads
    const size_t pb = (size_t)n * sizeof(float);
    if (n > 0 && (cudaMemcpyAsync(dpos, hx, pb, cudaMemcpyHostToDevice, up) != cudaSuccess ||
                  cudaMemcpyAsync(dpos + N, hy, pb, cudaMemcpyHostToDevice, up) != cudaSuccess ||
                  cudaMemcpyAsync(dpos + 2 * N, hz, pb, cudaMemcpyHostToDevice, up) != cudaSuccess))
        return LJ_ECUDA;
    if (cudaEventRecord(ev[kE2EASlots], up) != cudaSuccess ||
        cudaStreamWaitEvent(st, ev[kE2EASlots], 0) != cudaSuccess)
        return LJ_ECUDA;
    lj_particles sorted{};
    sorted.index = didx;
    s = lj_bin(c, g, n, dpos, dpos + N, dpos + 2 * N, 1, LJ_ORDER_X, dcnt, doff, nullptr, &sorted, dx4, dcell);
    if (s != LJ_OK) return s;
    if (cudaEventRecord(ev[kE2EASlots + 1], st) != cudaSuccess ||
        cudaStreamWaitEvent(cp, ev[kE2EASlots + 1], 0) != cudaSuccess)
        return LJ_ECUDA;
    if (n > 0 && h_index && !inorder &&
        cudaMemcpyAsync(h_index, didx, (size_t)n * sizeof(int), cudaMemcpyDeviceToHost, cp) != cudaSuccess)
        return LJ_ECUDA;
    const int chunks = inorder || n < kE2EChunks * 4096 ? 1 : kE2EChunks;
    for (int k = 0; k < chunks; ++k) {
        const int kb = (int)((long long)n * k / chunks), ke = (int)((long long)n * (k + 1) / chunks);
        s = launch_pair_config(c, g, p, n, dx4, dcell, doff, LJ_ORDER_X, h_energy ? de : nullptr,
                               h_force ? df : nullptr, dtot + k, kb, ke, inorder);
        if (s != LJ_OK) return s;
        if (ke == kb || inorder) continue;
        if (cudaEventRecord(ev[kE2EASlots + 2 + k], st) != cudaSuccess ||
            cudaStreamWaitEvent(cp, ev[kE2EASlots + 2 + k], 0) != cudaSuccess)
            return LJ_ECUDA;
        const size_t cb = (size_t)(ke - kb) * sizeof(float);
        if (h_energy && cudaMemcpyAsync(h_energy + kb, de + kb, cb, cudaMemcpyDeviceToHost, cp) != cudaSuccess)
            return LJ_ECUDA;
        if (h_force &&
            cudaMemcpyAsync(h_force + 3 * (size_t)kb, df + 3 * (size_t)kb, 3 * cb, cudaMemcpyDeviceToHost, cp) !=
                cudaSuccess)
            return LJ_ECUDA;
    }
    k_sum_totals<<<1, 1, 0, st>>>(dtot, chunks, dtot + kE2EChunks);
    if ((s = last_launch_status()) != LJ_OK) return s;
    if (cudaEventRecord(ev[kE2EASlots + 6], st) != cudaSuccess ||
        cudaStreamWaitEvent(cp, ev[kE2EASlots + 6], 0) != cudaSuccess)
        return LJ_ECUDA;
    if (inorder && n > 0) {
        const size_t eb = (size_t)n * sizeof(float);
        if (h_energy && cudaMemcpyAsync(h_energy, de, eb, cudaMemcpyDeviceToHost, cp) != cudaSuccess)
            return LJ_ECUDA;
        if (h_force && cudaMemcpyAsync(h_force, df, 3 * eb, cudaMemcpyDeviceToHost, cp) != cudaSuccess)
            return LJ_ECUDA;
    }
    const int q = c->e2ea_pending;
    if (cudaMemcpyAsync(c->e2ea_tot + q, dtot + kE2EChunks, sizeof(lj_totals), cudaMemcpyDeviceToHost, cp) !=
        cudaSuccess)
        return LJ_ECUDA;
    c->e2ea_dst[q] = h_totals;
    c->e2ea_pending = q + 1;
    // the slot is free again once its downloads are done
    if (cudaEventRecord(ev[slot], cp) != cudaSuccess) return LJ_ECUDA;
    c->e2ea_slot = (slot + 1) % kE2EASlots;
    return LJ_OK;
}

}  // namespace ljc

extern "C" lj_status lj_simulate_host_async(lj_ctx* c, const lj_grid* g, const lj_params* p, int n, const float* hx,
                                            const float* hy, const float* hz, float* h_energy, float* h_force,
                                            int* h_index, lj_totals* h_totals) {
    const NvtxRange nvtx_range("lj_simulate_host_async");
    return simulate_async(c, g, p, n, hx, hy, hz, h_energy, h_force, h_index, h_totals, false);
}

extern "C" lj_status lj_simulate_host_inorder_async(lj_ctx* c, const lj_grid* g, const lj_params* p, int n,
                                                    const float* hx, const float* hy, const float* hz,
                                                    float* h_energy, float* h_force, lj_totals* h_totals) {
    const NvtxRange nvtx_range("lj_simulate_host_inorder_async");
    return simulate_async(c, g, p, n, hx, hy, hz, h_energy, h_force, nullptr, h_totals, true);
}

extern "C" lj_status lj_simulate_host_inorder(lj_ctx* c, const lj_grid* g, const lj_params* p, int n,
                                              const float* hx, const float* hy, const float* hz, float* h_energy,
                                              float* h_force, lj_totals* h_totals) {
    const NvtxRange nvtx_range("lj_simulate_host_inorder");
    const lj_status s = simulate_async(c, g, p, n, hx, hy, hz, h_energy, h_force, nullptr, h_totals, true);
    const lj_status w = c ? lj_simulate_host_wait(c) : LJ_EINVAL;
    return s != LJ_OK ? s : w;
}

extern "C" lj_status lj_simulate_host_wait(lj_ctx* c) {
    if (!c) return LJ_EINVAL;
    DeviceScope scope(c->device);
    if (!scope.ok) return LJ_ECUDA;
    if (c->e2ea_ready && cudaStreamSynchronize(c->up_stream) != cudaSuccess) return LJ_ECUDA;
    if (c->e2e_ready && cudaStreamSynchronize(c->copy_stream) != cudaSuccess) return LJ_ECUDA;
    if (c->e2ea_ready) e2ea_deliver(c);
    return lj_sync(c);
}
