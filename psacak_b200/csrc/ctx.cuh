// ctx.cuh -- builder context: device, stream, stream-ordered allocations,
// scratch for the primitives, the per-level trace.
#pragma once

#include <mutex>
#include <vector>

#include "prims.cuh"

struct psacak_ctx;

namespace psk {

struct Ctx {
    Device dev;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;  // stream of the current call
    cudaMemPool_t pool = nullptr;
    uint32_t *h_pinned = nullptr;   // small pinned buffer for scalar read-backs
    uint32_t *d_partial = nullptr;  // MAX_CHUNKS * 4 uint32 scan partials
    uint32_t *d_hist = nullptr;     // 256 * RADIX_MAX_CTAS radix histograms
    uint32_t *d_scalars = nullptr;  // 64 device scalars
    uint32_t *d_err = nullptr;      // device error word
    uint32_t scan_ctas = 0;         // CTAs of the chunked scans
    uint32_t radix_ctas = 0;        // CTAs of the radix passes
    psacak_schedule sched{};
    // When set, level 0 stops after building its reduced string and copies
    // it here (used by psacak_debug_reduced8).
    uint32_t *debug_red = nullptr;
    uint64_t debug_cap = 0, debug_n1 = 0, debug_k = 0;
    std::vector<psacak_level_info> trace;
    bool profiling = false;
    Profiler prof;
    unsigned long long *d_induced = nullptr;  // entries scattered by the bucket scans
    std::mutex mu;

    template <class T>
    status_t alloc(T **p, size_t count) {
        size_t bytes = count * sizeof(T);
        if (bytes == 0) bytes = 16;
        void *q = nullptr;
        cudaError_t e = cudaMallocFromPoolAsync(&q, bytes, pool, stream);
        if (e != cudaSuccess) {
            *p = nullptr;
            return set_error(PSACAK_ENOMEM, "device allocation of %zu bytes failed: %s", bytes,
                             cudaGetErrorString(e));
        }
        *p = (T *)q;
        return PSACAK_OK;
    }
    void release(void *p) {
        if (p) cudaFreeAsync(p, stream);
    }
    // Copies `count` uint32 from device to host and waits for the stream.
    status_t read_u32(const uint32_t *d, uint32_t *h, size_t count = 1) {
        PSK_CUDA(cudaMemcpyAsync(h_pinned, d, count * sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
        PSK_CUDA(cudaStreamSynchronize(stream));
        for (size_t i = 0; i < count; i++) h[i] = h_pinned[i];
        return PSACAK_OK;
    }
    status_t sync() {
        PSK_CUDA(cudaStreamSynchronize(stream));
        return PSACAK_OK;
    }
    status_t check_device_error() {
        uint32_t e = 0;
        PSK_TRY(read_u32(d_err, &e));
        if (e) {
            PSK_CUDA(cudaMemsetAsync(d_err, 0, sizeof(uint32_t), stream));
            if (e & DEVERR_TIMEOUT) return set_error(PSACAK_ETIMEOUT, "a bounded device wait ran out (0x%x)", e);
            return set_error(PSACAK_EINTERNAL, "device-side consistency check failed (0x%x)", e);
        }
        return PSACAK_OK;
    }
};

// RAII holder of a stream-ordered device allocation.
template <class T> struct DBuf {
    Ctx *ctx = nullptr;
    T *p = nullptr;
    DBuf() = default;
    DBuf(const DBuf &) = delete;
    DBuf &operator=(const DBuf &) = delete;
    ~DBuf() { reset(); }
    status_t init(Ctx &c, size_t count) {
        reset();
        ctx = &c;
        return c.alloc(&p, count);
    }
    void reset() {
        if (ctx && p) ctx->release(p);
        p = nullptr;
    }
    T *get() const { return p; }
    operator T *() const { return p; }
};

}  // namespace psk

struct psacak_ctx {
    psk::Ctx c;
};
