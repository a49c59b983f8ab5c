// onesweep.cuh -- single-pass stable scatter by an 8-bit digit with
// decoupled look-back.
//
// One kernel moves every item to its digit's output range, stable in input
// order: each CTA claims the next tile (atomic ticket, so tiles are claimed
// in order), ranks its items per digit in shared memory, publishes its
// per-digit counts, and adds the counts of the tiles before it by walking
// back until it meets a tile that already published an inclusive prefix.
// The items are staged through shared memory in digit order so that the
// writes leave in runs.
//
// Status words are 64-bit: [epoch:30 | flag:2 | count:32].  The epoch of a
// launch is part of every word it writes, so words left by earlier launches
// read as "not ready" and the array never needs clearing.  Every wait is
// bounded: after SPIN_LIMIT polls the CTA records DEVERR_TIMEOUT and
// proceeds (the build then fails with PSACAK_ETIMEOUT).  A predecessor tile
// has always been claimed by a running or finished CTA, so the wait ends in
// normal operation.
//
// A Policy supplies, per item index i < n:
//   load(i, item, digit)            -> digit in [0, 256) or >= 256 to drop it
//   out0(digit), kOutSign (+1 / -1) -> the rank-th item of a digit (rank
//                                      counting from 0 over all tiles of this
//                                      launch) goes to out0(digit) + kOutSign * rank
//   store(index, item, digit)
//   finish(digit, total)            -> called once per digit by the last tile
//   kMinBlocks                      -> CTAs per SM the register budget must allow
//                                      at 12 items per thread (raised by
//                                      12 / IPT for smaller tiles)
#pragma once

#include <type_traits>
#include <utility>

#include "prims.cuh"

namespace psk {

constexpr int OS_BLOCK = 256;
constexpr int OS_WARPS = OS_BLOCK / 32;
constexpr uint32_t OS_SPIN_LIMIT = 1u << 24;
// Predecessor status words read per look-back step: 4 for the scatters (a
// measured ~4% gain on the bucket scans), 1 for the radix passes, whose
// 64-register budget the window's loads would strain (measured 2% slower).
constexpr int OS_LB_WINDOW = 4;

constexpr uint64_t OS_FLAG_AGG = 1ull;
constexpr uint64_t OS_FLAG_PREFIX = 2ull;

__device__ __forceinline__ uint64_t os_word(uint32_t epoch, uint64_t flag, uint32_t count) {
    return ((uint64_t)epoch << 34) | (flag << 32) | count;
}

__device__ __forceinline__ uint64_t os_load(const uint64_t *p) {
    uint64_t v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void os_store(uint64_t *p, uint64_t v) {
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Publishes this tile's count of digit d and returns the digit's exclusive
// prefix over all earlier tiles: walks back over aggregates until a tile
// with an inclusive prefix, then publishes its own inclusive prefix.  Each
// poll of a not-yet-ready word counts against OS_SPIN_LIMIT.  PUBLISHED:
// the caller has already published the count (an aggregate, or for tile 0
// its prefix), so only the walk and the final prefix remain.
template <int WINDOW = OS_LB_WINDOW, bool PUBLISHED = false>
__device__ __forceinline__ uint32_t os_lookback(uint64_t *status, uint32_t tile, uint32_t d, uint32_t count,
                                                uint32_t epoch, uint32_t *err) {
    uint64_t *my = status + (uint64_t)tile * 256 + d;
    if (tile == 0) {
        if (!PUBLISHED) os_store(my, os_word(epoch, OS_FLAG_PREFIX, count));
        return 0;
    }
    if (!PUBLISHED) os_store(my, os_word(epoch, OS_FLAG_AGG, count));
    uint32_t excl = 0;
    int64_t t = (int64_t)tile - 1;
    uint32_t left = 0;  // poll budget (spin_spend)
    while (t >= 0) {
        // WINDOW predecessors per step, their loads in flight together (a
        // walk over tiles that have only published their counts costs one
        // latency per window, not per tile)
        uint64_t v[WINDOW];
#pragma unroll
        for (int k = 0; k < WINDOW; k++)
            v[k] = t - k >= 0 ? os_load(status + (uint64_t)(t - k) * 256 + d) : 0ull;
        int k = 0;
        bool found = false;
        for (; k < WINDOW && t - k >= 0; k++) {
            const uint32_t ep = (uint32_t)(v[k] >> 34);
            const uint64_t fl = (v[k] >> 32) & 3ull;
            if (ep != epoch || fl == 0) break;  // not ready: poll again from this tile
            excl += (uint32_t)v[k];
            if (fl == OS_FLAG_PREFIX) {
                found = true;
                break;
            }
        }
        if (found) break;
        if (k == 0 && spin_spend(left, err, OS_SPIN_LIMIT)) {
            dev_fail(err, DEVERR_TIMEOUT);
            break;
        }
        t -= k;
    }
    os_store(my, os_word(epoch, OS_FLAG_PREFIX, excl + count));
    return excl;
}

// A policy with `using Pre = ...` loads in two phases: pre(i, Pre&) for
// every item of the thread, then load(i, const Pre&, item, digit).
template <class P, class = void> struct os_two_phase : std::false_type {};
template <class P> struct os_two_phase<P, std::void_t<typename P::Pre>> : std::true_type {};

// A policy with `bool active(d)` names the digits its items can take (the
// same for every tile of a launch); the others skip the look-back -- their
// counts are 0 in every tile -- so a tile polls only for digits that can
// move.  An item whose digit is not active is recorded as DEVERR_RANGE.
template <class P, class = void> struct os_has_active : std::false_type {};
template <class P>
struct os_has_active<P, std::void_t<decltype(std::declval<const P &>().active(0u))>> : std::true_type {};
template <class P> __device__ __forceinline__ bool os_active(const P &pol, uint32_t d) {
    if constexpr (os_has_active<P>::value) return pol.active(d);
    else return true;
}

constexpr int os_min_blocks(int at12, int ipt) { return ipt < 12 ? at12 * 12 / ipt : at12; }

template <class Policy, int IPT>
__global__ void __launch_bounds__(OS_BLOCK, os_min_blocks(Policy::kMinBlocks, IPT)) k_onesweep(Policy pol, uint64_t n, uint64_t *status, uint32_t *ticket,
                                                       uint32_t epoch, uint32_t ntiles, uint32_t *err) {
    using Item = typename Policy::Item;
    constexpr int TILE = OS_BLOCK * IPT;
    extern __shared__ __align__(16) unsigned char os_smem[];
    Item *s_item = (Item *)os_smem;
    uint8_t *s_dig = (uint8_t *)(s_item + TILE);
    __shared__ uint32_t s_tstart[256];
    __shared__ uint64_t s_obase[256];  // output index of tile position i = s_obase[digit] + kOutSign * i
    __shared__ uint16_t s_wcnt[OS_WARPS][256];
    __shared__ uint32_t s_scan[33];
    __shared__ uint32_t s_tile;

    const int w = threadIdx.x >> 5;
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t lt = lanemask_lt();

    if (threadIdx.x == 0) s_tile = atomicAdd(ticket, 1u);
    for (int i = threadIdx.x; i < OS_WARPS * 256; i += OS_BLOCK) (&s_wcnt[0][0])[i] = 0;
    __syncthreads();
    const uint32_t tile = s_tile;
    const uint64_t base = (uint64_t)tile * TILE;
    const uint32_t cnt = n - base < (uint64_t)TILE ? (uint32_t)(n - base) : (uint32_t)TILE;  // items of this tile

    // load every item of the thread first (independent loads in flight);
    // two-phase policies read their direct operands for every item before
    // any dependent gather
    Item it[IPT];
    uint32_t dg[IPT];
    if constexpr (os_two_phase<Policy>::value) {
        typename Policy::Pre pre[IPT];
#pragma unroll
        for (int r = 0; r < IPT; r++) {
            const uint32_t li = (uint32_t)w * 32 * IPT + (uint32_t)r * 32 + lane;
            if (li < cnt) pol.pre(base + li, pre[r]);
        }
#pragma unroll
        for (int r = 0; r < IPT; r++) {
            const uint32_t li = (uint32_t)w * 32 * IPT + (uint32_t)r * 32 + lane;
            dg[r] = 256;
            if (li < cnt) pol.load(base + li, pre[r], it[r], dg[r]);
        }
    } else {
#pragma unroll
        for (int r = 0; r < IPT; r++) {
            const uint32_t li = (uint32_t)w * 32 * IPT + (uint32_t)r * 32 + lane;
            dg[r] = 256;
            if (li < cnt) pol.load(base + li, it[r], dg[r]);
        }
    }
    // stable ranks within the warp's sub-tile
    uint16_t rk[IPT];
#pragma unroll
    for (int r = 0; r < IPT; r++) {
        uint32_t d = dg[r] < 256 ? dg[r] : 256u;
        uint32_t peers = __match_any_sync(FULL_MASK, d);
        uint32_t prior = d < 256 ? s_wcnt[w][d] : 0u;
        rk[r] = (uint16_t)(prior + __popc(peers & lt));
        __syncwarp();
        if (d < 256 && (int)lane == __ffs(peers) - 1) s_wcnt[w][d] = (uint16_t)(prior + __popc(peers));
        __syncwarp();
        dg[r] = d;
    }
    __syncthreads();
    const uint32_t d = threadIdx.x;  // this thread's digit from here on
    uint32_t count = 0;
#pragma unroll
    for (int ww = 0; ww < OS_WARPS; ww++) {
        uint32_t c = s_wcnt[ww][d];
        s_wcnt[ww][d] = (uint16_t)count;
        count += c;
    }
    uint32_t excl = 0;
    if (os_active(pol, d)) excl = os_lookback(status, tile, d, count, epoch, err);
    else if (count) dev_fail(err, DEVERR_RANGE);
    uint32_t ex, tot;
    block_scan<uint32_t, OpSum<uint32_t>, OS_BLOCK>(count, OpSum<uint32_t>(), s_scan, &ex, &tot);
    s_tstart[d] = ex;
    // the digit's item at tile position i has launch rank excl + i - ex
    // (modular arithmetic: the true index is in range)
    s_obase[d] = Policy::kOutSign > 0 ? pol.out0(d) + excl - ex : pol.out0(d) - excl + ex;
    if (tile == ntiles - 1) pol.finish(d, excl + count);
    __syncthreads();
    // stage in digit order
#pragma unroll
    for (int r = 0; r < IPT; r++) {
        if (dg[r] < 256) {
            uint32_t pos = s_tstart[dg[r]] + s_wcnt[w][dg[r]] + rk[r];
            s_item[pos] = it[r];
            s_dig[pos] = (uint8_t)dg[r];
        }
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < tot; i += OS_BLOCK) {
        const uint32_t dd = s_dig[i];
        const uint64_t idx = Policy::kOutSign > 0 ? s_obase[dd] + i : s_obase[dd] - i;
        pol.store(idx, s_item[i], dd);
    }
}

// Scratch of one onesweep launch sequence: status words for `max_tiles`
// tiles, a ticket per launch, and the launch epoch.
struct OnesweepScratch {
    uint64_t *status = nullptr;
    uint32_t *tickets = nullptr;  // 64 tickets, reused round robin
    uint64_t max_tiles = 0;
    uint32_t epoch = 0;
};

template <class Policy, int IPT>
status_t onesweep(Policy pol, uint64_t n, OnesweepScratch &sc, uint32_t *err, cudaStream_t s, const char *pname,
                  uint64_t pbytes) {
    if (n == 0) return PSACAK_OK;
    constexpr int TILE = OS_BLOCK * IPT;
    const uint64_t ntiles = ceil_div(n, TILE);
    if (ntiles > sc.max_tiles) return set_error(PSACAK_EINTERNAL, "onesweep: %llu tiles exceed scratch", (unsigned long long)ntiles);
    sc.epoch = (sc.epoch + 1) & ((1u << 30) - 1);
    if (sc.epoch == 0) sc.epoch = 1;
    uint32_t *ticket = sc.tickets + (sc.epoch & 63);
    PSK_CUDA(cudaMemsetAsync(ticket, 0, sizeof(uint32_t), s));
    const size_t smem = (size_t)TILE * (sizeof(typename Policy::Item) + 1);
    PSK_CUDA(cudaFuncSetAttribute(k_onesweep<Policy, IPT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    PSK_PROF_LAUNCH(s, pname, n, pbytes,
                    (k_onesweep<Policy, IPT><<<(uint32_t)ntiles, OS_BLOCK, smem, s>>>(pol, n, sc.status, ticket,
                                                                                      sc.epoch, (uint32_t)ntiles,
                                                                                      err)));
    PSK_LAUNCH_CHECK();
    return PSACAK_OK;
}

}  // namespace psk

namespace psk {

// Runtime choice of the tile (items per thread: 8, 12 or 16).
template <class Policy>
status_t onesweep_ipt(Policy pol, uint64_t n, int ipt, OnesweepScratch &sc, uint32_t *err, cudaStream_t s,
                      const char *pname, uint64_t pbytes) {
    if (ipt == 8) return onesweep<Policy, 8>(pol, n, sc, err, s, pname, pbytes);
    if (ipt == 16) return onesweep<Policy, 16>(pol, n, sc, err, s, pname, pbytes);
    return onesweep<Policy, 12>(pol, n, sc, err, s, pname, pbytes);
}

// Stable compaction through the same kernel: kept items carry digit 0.
template <class Pred, class Emit> struct CompactPolicy {
    using Item = uint32_t;
    static constexpr int kMinBlocks = 4;
    Pred pred;
    Emit emit;
    uint32_t *count;
    __device__ __forceinline__ void load(uint64_t i, Item &it, uint32_t &d) const {
        if (pred(i)) {
            d = 0;
            it = (uint32_t)i;
        }
    }
    static constexpr int kOutSign = 1;
    __device__ __forceinline__ bool active(uint32_t d) const { return d == 0; }
    __device__ __forceinline__ uint64_t out0(uint32_t) const { return 0; }
    __device__ __forceinline__ void store(uint64_t idx, const Item &it, uint32_t) const { emit((uint64_t)it, (uint32_t)idx); }
    __device__ __forceinline__ void finish(uint32_t d, uint32_t total) const {
        if (d == 0 && count) *count = total;
    }
};

// Single-pass stable compaction: emit(i, slot) for every i < n with pred(i),
// slots consecutive in index order; *count_out (device, nullable) = kept.
template <class Pred, class Emit>
status_t compact1(Pred pred, Emit emit, uint64_t n, uint32_t *count_out, OnesweepScratch &sc, uint32_t *err,
                  cudaStream_t s, const char *pname, int ipt = 12) {
    if (n == 0) {
        if (count_out) PSK_CUDA(cudaMemsetAsync(count_out, 0, sizeof(uint32_t), s));
        return PSACAK_OK;
    }
    return onesweep_ipt(CompactPolicy<Pred, Emit>{pred, emit, count_out}, n, ipt, sc, err, s, pname, 0);
}

}  // namespace psk
