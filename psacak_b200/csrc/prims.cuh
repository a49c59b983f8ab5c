// prims.cuh -- shared device building blocks: launch counting, scan
// operators, warp and block scans.  The device-wide primitives built on them
// are the single-pass scatter (onesweep.cuh), radix passes (radix.cuh) and
// the single-pass scan (lbscan.cuh).
#pragma once

#include <atomic>

#include "common.cuh"

namespace psk {

extern std::atomic<uint64_t> g_kernel_launches;
#define PSK_KCOUNT() (::psk::g_kernel_launches.fetch_add(1, std::memory_order_relaxed))
// Host round trips inside a build: the host waits for values the device
// computed (counts, histograms) before it can decide what to launch next.
extern std::atomic<uint64_t> g_round_trips;
#define PSK_ROUND_TRIP() (::psk::g_round_trips.fetch_add(1, std::memory_order_relaxed))
}  // namespace psk
#include "prof.cuh"
namespace psk {

constexpr uint32_t MAX_CHUNKS = 1024;  // cap on the CTAs of grid-stride helper kernels

// Scan operators.  kFields / field(f, a, b): the value as 32-bit fields and
// the combination of field f (the single-pass scan publishes each field on
// its own).
template <class T> struct OpSum {
    static constexpr int kFields = 1;
    __device__ __forceinline__ T operator()(T a, T b) const { return a + b; }
    __device__ __forceinline__ static T identity() { return T(0); }
    __device__ __forceinline__ static uint32_t field(int, uint32_t a, uint32_t b) { return a + b; }
};
template <class T> struct OpMax {
    static constexpr int kFields = 1;
    __device__ __forceinline__ T operator()(T a, T b) const { return a > b ? a : b; }
    __device__ __forceinline__ static T identity() { return T(0); }
    __device__ __forceinline__ static uint32_t field(int, uint32_t a, uint32_t b) { return a > b ? a : b; }
};

// Shuffle-up of any scan value; aggregate value types provide an overload
// in their own namespace (found by argument-dependent lookup).
template <class T>
__device__ __forceinline__ T shfl_up_t(T v, int o) { return __shfl_up_sync(FULL_MASK, v, o); }

template <class T, class Op>
__device__ __forceinline__ T warp_scan_inclusive(T v, Op op) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        T t = shfl_up_t(v, o);
        if ((int)(threadIdx.x & 31) >= o) v = op(t, v);
    }
    return v;
}

// Block-wide scan with a generic associative op.  Returns the inclusive
// value; *excl receives the exclusive one (identity for thread 0) and
// *total the block aggregate.  smem must hold 33 T.
template <class T, class Op, int BLOCK>
__device__ __forceinline__ T block_scan(T v, Op op, T *smem, T *excl, T *total) {
    constexpr int NW = BLOCK / 32;
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    T inc = warp_scan_inclusive(v, op);
    if (l == 31) smem[w] = inc;
    __syncthreads();
    if (w == 0) {
        T x = l < NW ? smem[l] : Op::identity();
        T xi = warp_scan_inclusive(x, op);
        if (l < NW) smem[l] = xi;
    }
    __syncthreads();
    T pre = w > 0 ? smem[w - 1] : Op::identity();
    T res = w > 0 ? op(pre, inc) : inc;
    // exclusive = pre (+) inclusive-within-warp-exclusive
    T wex = shfl_up_t(inc, 1);
    T ex;
    if (l == 0) ex = pre;
    else ex = w > 0 ? op(pre, wex) : wex;
    if (excl) *excl = ex;
    if (total) *total = smem[NW - 1];
    __syncthreads();
    return res;
}

// LSD radix sort of (key, value) pairs: see radix.cuh (single-pass scatter).
// ---------------------------------------------------------------------------
constexpr uint32_t RADIX_MAX_CTAS = 1024;

}  // namespace psk
