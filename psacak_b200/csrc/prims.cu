// prims.cu -- non-template pieces of the device primitives and the
// library-wide error reporting.
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include "radix.cuh"

namespace psk {

std::atomic<uint64_t> g_kernel_launches{0};
std::atomic<uint64_t> g_round_trips{0};
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

__global__ void k_copy_words(const uint32_t *__restrict__ src, uint32_t *dst, uint32_t count) {
    for (uint32_t i = threadIdx.x; i < count; i += blockDim.x) dst[i] = src[i];
}

status_t read_back(const uint32_t *d, uint32_t *mapped, uint32_t count, cudaStream_t s) {
    if (count == 0) return PSACAK_OK;
    PSK_ROUND_TRIP();
    k_copy_words<<<1, 256, 0, s>>>(d, mapped, count);
    PSK_KCOUNT();
    PSK_CUDA(cudaGetLastError());
    PSK_CUDA(cudaStreamSynchronize(s));
    return PSACAK_OK;
}

__global__ void k_radix_bases(const uint32_t *hist, uint32_t *bases) {
    __shared__ uint32_t smem[33];
    const uint32_t p = blockIdx.x;
    uint32_t v = hist[p * 256 + threadIdx.x];
    uint32_t ex;
    block_scan<uint32_t, OpSum<uint32_t>, 256>(v, OpSum<uint32_t>(), smem, &ex, (uint32_t *)nullptr);
    bases[p * 256 + threadIdx.x] = ex;
}

}  // namespace psk
