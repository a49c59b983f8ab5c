// prims.cuh -- device-wide building blocks: chunked scans, stream compaction
// and LSD radix-sort passes.  All are "reduce-then-scan" designs: a first
// kernel reduces each CTA's contiguous chunk, a single-CTA kernel scans the
// per-chunk partials, a last kernel rescans each chunk with its carry.  No
// kernel waits on another CTA, so nothing here can spin.
#pragma once

#include <atomic>

#include "common.cuh"

namespace psk {

extern std::atomic<uint64_t> g_kernel_launches;
#define PSK_KCOUNT() (::psk::g_kernel_launches.fetch_add(1, std::memory_order_relaxed))
}  // namespace psk
#include "prof.cuh"
namespace psk {

constexpr int SCAN_BLOCK = 256;
constexpr int SCAN_IPT = 8;
constexpr int SCAN_TILE = SCAN_BLOCK * SCAN_IPT;
constexpr uint32_t MAX_CHUNKS = 1024;

struct Chunking {
    uint32_t G;      // number of chunks (= CTAs)
    uint64_t chunk;  // items per chunk (multiple of tile)
};

inline Chunking make_chunking(uint64_t n, uint64_t tile, uint32_t max_ctas) {
    Chunking c;
    uint64_t tiles = ceil_div(n ? n : 1, tile);
    uint32_t G = (uint32_t)(tiles < max_ctas ? tiles : max_ctas);
    if (G == 0) G = 1;
    c.G = G;
    c.chunk = ceil_div(tiles, G) * tile;
    return c;
}

template <class T> struct OpSum {
    __device__ __forceinline__ T operator()(T a, T b) const { return a + b; }
    __device__ __forceinline__ static T identity() { return T(0); }
};
template <class T> struct OpMax {
    __device__ __forceinline__ T operator()(T a, T b) const { return a > b ? a : b; }
    __device__ __forceinline__ static T identity() { return T(0); }
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

// ---------------------------------------------------------------------------
// Chunked scan.  `ld(i)` yields the value of item i; `st(i, excl, v)` is
// called for each item with its exclusive prefix (across the whole range).
// ---------------------------------------------------------------------------
template <class T, class Op, class Load>
__global__ void __launch_bounds__(SCAN_BLOCK) k_chunk_reduce(Load ld, uint64_t n, uint64_t chunk,
                                                             T *partial, Op op) {
    __shared__ T smem[33];
    uint64_t start = (uint64_t)blockIdx.x * chunk;
    uint64_t end = start + chunk < n ? start + chunk : n;
    T acc = Op::identity();
    for (uint64_t i = start + threadIdx.x; i < end; i += SCAN_BLOCK) acc = op(acc, ld(i));
    T total;
    block_scan<T, Op, SCAN_BLOCK>(acc, op, smem, (T *)nullptr, &total);
    if (threadIdx.x == 0) partial[blockIdx.x] = total;
}

// Exclusive scan of the G partials in place (G <= 1024), one CTA of 1024.
template <class T, class Op>
__global__ void __launch_bounds__(1024) k_scan_partials(T *partial, uint32_t G, T *total_out, Op op) {
    __shared__ T smem[33];
    T v = threadIdx.x < G ? partial[threadIdx.x] : Op::identity();
    T ex, tot;
    block_scan<T, Op, 1024>(v, op, smem, &ex, &tot);
    if (threadIdx.x < G) partial[threadIdx.x] = ex;
    if (threadIdx.x == 0 && total_out) *total_out = tot;
}

template <class T, class Op, class Load, class Store>
__global__ void __launch_bounds__(SCAN_BLOCK) k_chunk_scan(Load ld, Store st, uint64_t n, uint64_t chunk,
                                                           const T *partial, Op op) {
    __shared__ T smem[33];
    uint64_t start = (uint64_t)blockIdx.x * chunk;
    uint64_t end = start + chunk < n ? start + chunk : n;
    T carry = partial[blockIdx.x];
    for (uint64_t base = start; base < end; base += SCAN_TILE) {
        T v[SCAN_IPT];
        T acc = Op::identity();
#pragma unroll
        for (int k = 0; k < SCAN_IPT; k++) {
            uint64_t i = base + (uint64_t)threadIdx.x * SCAN_IPT + k;
            v[k] = i < end ? ld(i) : Op::identity();
            acc = op(acc, v[k]);
        }
        T ex, tot;
        block_scan<T, Op, SCAN_BLOCK>(acc, op, smem, &ex, &tot);
        T run = op(carry, ex);
        if (threadIdx.x == 0) run = carry;
#pragma unroll
        for (int k = 0; k < SCAN_IPT; k++) {
            uint64_t i = base + (uint64_t)threadIdx.x * SCAN_IPT + k;
            if (i < end) st(i, run, v[k]);
            run = op(run, v[k]);
        }
        carry = op(carry, tot);
    }
}

// Runs the three kernels.  `partial` must hold MAX_CHUNKS T; `total_out`
// (device, nullable) receives the op-aggregate of all items.
template <class T, class Op, class Load, class Store>
status_t chunk_scan(Load ld, Store st, uint64_t n, T *partial, T *total_out, Op op,
                    uint32_t max_ctas, cudaStream_t s) {
    Chunking c = make_chunking(n, SCAN_TILE, max_ctas < MAX_CHUNKS ? max_ctas : MAX_CHUNKS);
    if (n > 0) {
        PSK_PROF_LAUNCH(s, "scan_reduce", n, 0,
                        (k_chunk_reduce<T, Op, Load><<<c.G, SCAN_BLOCK, 0, s>>>(ld, n, c.chunk, partial, op)));
    }
    PSK_PROF_LAUNCH(s, "scan_partials", c.G, 0,
                    (k_scan_partials<T, Op><<<1, 1024, 0, s>>>(partial, n > 0 ? c.G : 0, total_out, op)));
    if (n > 0) {
        PSK_PROF_LAUNCH(s, "scan_apply", n, 0,
                        (k_chunk_scan<T, Op, Load, Store><<<c.G, SCAN_BLOCK, 0, s>>>(ld, st, n, c.chunk, partial, op)));
    }
    PSK_LAUNCH_CHECK();
    return PSACAK_OK;
}

// ---------------------------------------------------------------------------
// Stable stream compaction: items with pred(i) are passed to emit(i, slot)
// in index order with consecutive slots; *count_out (device) = number kept.
// ---------------------------------------------------------------------------
template <class Pred> struct FlagLoad {
    Pred p;
    __device__ __forceinline__ uint32_t operator()(uint64_t i) const { return p(i) ? 1u : 0u; }
};
template <class Pred, class Emit> struct FlagStore {
    Pred p;
    Emit e;
    __device__ __forceinline__ void operator()(uint64_t i, uint32_t excl, uint32_t v) const {
        if (v) e(i, excl);
    }
};

template <class Pred, class Emit>
status_t compact(Pred pred, Emit emit, uint64_t n, uint32_t *partial, uint32_t *count_out,
                 uint32_t max_ctas, cudaStream_t s) {
    return chunk_scan<uint32_t, OpSum<uint32_t>>(FlagLoad<Pred>{pred}, FlagStore<Pred, Emit>{pred, emit},
                                                 n, partial, count_out, OpSum<uint32_t>(), max_ctas, s);
}

// LSD radix sort of (key, value) pairs: see radix.cuh (single-pass scatter).
// ---------------------------------------------------------------------------
constexpr uint32_t RADIX_MAX_CTAS = 1024;

}  // namespace psk
