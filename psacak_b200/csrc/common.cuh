// common.cuh -- shared definitions for the psacak_b200 CUDA library.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stddef.h>

#include "../../include/psacak_b200.h"

namespace psk {

constexpr uint32_t FULL_MASK = 0xFFFFFFFFu;

// Error returned by internal host helpers: 0 = ok, else a PSACAK_E* code.
typedef int status_t;

status_t set_error(status_t code, const char *fmt, ...);
status_t cuda_status(cudaError_t e, const char *what, const char *file, int line);

#define PSK_CUDA(call)                                                      \
    do {                                                                    \
        cudaError_t _e = (call);                                            \
        if (_e != cudaSuccess) return ::psk::cuda_status(_e, #call, __FILE__, __LINE__); \
    } while (0)

#define PSK_TRY(expr)                 \
    do {                              \
        ::psk::status_t _s = (expr);  \
        if (_s != PSACAK_OK) return _s; \
    } while (0)

#define PSK_LAUNCH_CHECK() PSK_CUDA(cudaGetLastError())

__host__ __device__ inline uint64_t ceil_div(uint64_t a, uint64_t b) { return (a + b - 1) / b; }

inline int bitlen(uint64_t x) {
    int b = 0;
    while (x) { b++; x >>= 1; }
    return b;
}

// ---------------------------------------------------------------------------
// Device-side error word.  Kernels that detect an inconsistency (a count that
// does not add up, a wait that ran out) OR a code into it instead of trapping;
// the host reads it after each build and turns it into a PSACAK_E* status.
// ---------------------------------------------------------------------------
enum : uint32_t {
    DEVERR_COUNT = 1u << 0,     // a bucket or level count did not add up
    DEVERR_RANGE = 1u << 1,     // an index fell outside its buffer
    DEVERR_TIMEOUT = 1u << 2,   // a bounded wait ran out
};

__device__ __forceinline__ void dev_fail(uint32_t *err, uint32_t code) {
    if (err) atomicOr(err, code);
}

// The error word is err[0] of a two-word array; err[1], when non-zero,
// replaces the compiled poll limit of every bounded wait (a test sets it
// through psacak_debug_set_limits to make a wait run out quickly).
// spin_spend keeps a wait's remaining budget in `left`: 0 means "not loaded
// yet", so the override is read once, at the first poll that finds nothing
// ready, and costs no register beyond the counter it replaces.  Returns true
// when the budget is spent.
__device__ __forceinline__ bool spin_spend(uint32_t &left, const uint32_t *err, uint32_t dflt) {
    if (left == 0) {
        uint32_t lim = dflt;
        if (err) {
            const uint32_t o = *(const volatile uint32_t *)(err + 1);
            if (o) lim = o;
        }
        left = lim + 1;
    }
    return --left == 0;
}

__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm volatile("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31; }

template <class T>
__device__ __forceinline__ T warp_inclusive_sum(T v) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        T t = __shfl_up_sync(FULL_MASK, v, o);
        if ((int)lane_id() >= o) v += t;
    }
    return v;
}

template <class T>
__device__ __forceinline__ T warp_inclusive_max(T v) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        T t = __shfl_up_sync(FULL_MASK, v, o);
        if ((int)lane_id() >= o) v = v > t ? v : t;
    }
    return v;
}

// Block-wide exclusive sum over one value per thread; returns the exclusive
// prefix and writes the block total to *total.  `smem` holds >= 33 T.
template <class T, int BLOCK>
__device__ __forceinline__ T block_exclusive_sum(T v, T *smem, T *total) {
    constexpr int NW = BLOCK / 32;
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    T inc = warp_inclusive_sum(v);
    if (l == 31) smem[w] = inc;
    __syncthreads();
    if (w == 0) {
        T x = l < NW ? smem[l] : T(0);
        T xi = warp_inclusive_sum(x);
        if (l < NW) smem[l] = xi - x;
        if (l == NW - 1) smem[32] = xi;
    }
    __syncthreads();
    T r = smem[w] + inc - v;
    if (total) *total = smem[32];
    __syncthreads();
    return r;
}

// Block-wide inclusive max.
template <class T, int BLOCK>
__device__ __forceinline__ T block_inclusive_max(T v, T *smem) {
    constexpr int NW = BLOCK / 32;
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    T inc = warp_inclusive_max(v);
    if (l == 31) smem[w] = inc;
    __syncthreads();
    if (w == 0) {
        T x = l < NW ? smem[l] : T(0);
        T xi = warp_inclusive_max(x);
        if (l < NW) smem[l] = xi;
    }
    __syncthreads();
    T pre = w > 0 ? smem[w - 1] : T(0);
    T r = inc > pre ? inc : pre;
    __syncthreads();
    return r;
}

// Bit access on a packed bitmap (bit i of word i/32).
__device__ __forceinline__ bool bm_get(const uint32_t *bm, uint64_t i) {
    return (bm[i >> 5] >> (i & 31)) & 1u;
}

struct Device {
    int id = 0;
    int num_sms = 148;
    size_t smem_optin = 227 * 1024;
};

}  // namespace psk
