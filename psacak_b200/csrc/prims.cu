// prims.cu -- non-template pieces of the device primitives and the
// library-wide error reporting.
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include "prims.cuh"

namespace psk {

std::atomic<uint64_t> g_kernel_launches{0};
thread_local Profiler *t_prof = nullptr;

static thread_local char t_last_error[512] = "";

status_t set_error(status_t code, const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(t_last_error, sizeof(t_last_error), fmt, ap);
    va_end(ap);
    return code;
}

status_t cuda_status(cudaError_t e, const char *what, const char *file, int line) {
    const char *base = strrchr(file, '/');
    base = base ? base + 1 : file;
    status_t code = (e == cudaErrorMemoryAllocation) ? PSACAK_ENOMEM : PSACAK_ECUDA;
    return set_error(code, "%s failed: %s (%s:%d)", what, cudaGetErrorString(e), base, line);
}

const char *last_error() { return t_last_error; }
void clear_error() { t_last_error[0] = 0; }

__global__ void __launch_bounds__(1024) k_radix_scan(uint32_t *hist, uint32_t total) {
    __shared__ uint32_t smem[33];
    uint32_t per = (total + 1023) / 1024;
    uint32_t b = threadIdx.x * per;
    uint32_t e = b + per < total ? b + per : total;
    uint32_t s = 0;
    for (uint32_t i = b; i < e; i++) s += hist[i];
    uint32_t ex;
    block_scan<uint32_t, OpSum<uint32_t>, 1024>(s, OpSum<uint32_t>(), smem, &ex, (uint32_t *)nullptr);
    for (uint32_t i = b; i < e; i++) {
        uint32_t v = hist[i];
        hist[i] = ex;
        ex += v;
    }
}

}  // namespace psk
