// lbscan.cuh -- single-pass scan with decoupled look-back.
//
// `ld(i)` yields the value of item i; `st(i, excl, v)` is called once per
// item with its exclusive prefix over the whole range and its own value.
// Each CTA claims the next tile of LS_BLOCK * ls_ipt<T>() items (atomic
// ticket, so tiles are claimed in order), loads its items once, scans them, publishes the tile
// aggregate and walks back over earlier tiles -- 32 at a time, one per lane
// of warp 0 -- until it meets one that has published its inclusive prefix.
// The items' values stay in registers between the load and the store, so
// every item is loaded exactly once (the chunked reduce-then-scan reads it
// twice) and any number of tiles are in flight at once.
//
// Publication: a 32-bit value travels inside its flag word
// [epoch:30 | flag:2 | value:32] (one relaxed 64-bit store / load, as in the
// onesweep status words).  Wider values are stored first (st.cg) and the
// flag word [epoch | flag | 0] follows with release semantics; readers poll
// with acquire loads and then read the value (ld.cg).  Flags carry the
// launch epoch, so the flag array never needs clearing and stale words read
// as "not ready".  The flags and values live in their own arrays
// (ScanScratch), apart from the onesweep status words.  Every wait is
// bounded by LS_SPIN_LIMIT polls, after which DEVERR_TIMEOUT is recorded and
// the CTA goes on.  A tile's
// predecessors have all been claimed by running CTAs, so the walk ends in
// normal operation.
//
// Op must be associative and commutative (sum, max and the per-field
// sums/maxima used here) with an identity.
#pragma once

#include "onesweep.cuh"

namespace psk {

constexpr int LS_BLOCK = 256;
constexpr int LS_IPT_MIN = 8;  // items per thread of 16-byte values; 32-bit values take 16
constexpr int LS_TILE_MIN = LS_BLOCK * LS_IPT_MIN;
template <class T> constexpr int ls_ipt() { return sizeof(T) == 4 ? 16 : LS_IPT_MIN; }
constexpr uint32_t LS_SPIN_LIMIT = 1u << 24;
constexpr uint32_t LS_MAX_VALUE_BYTES = 16;

struct ScanScratch {
    uint64_t *flags = nullptr;      // one word per tile
    unsigned char *vals = nullptr;  // aggregates then inclusive prefixes, max_tiles values each
    uint64_t max_tiles = 0;
};

template <class T> __device__ __forceinline__ void st_cg_words(T *p, const T &v);
template <class T> __device__ __forceinline__ T ld_cg_words(const T *p);

__device__ __forceinline__ uint64_t ld_acquire_u64(const uint64_t *p) {
    uint64_t v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_u64(uint64_t *p, uint64_t v) {
    asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
template <class T> __device__ __forceinline__ uint32_t as_u32(const T &v) {
    return *reinterpret_cast<const uint32_t *>(&v);
}
template <class T> __device__ __forceinline__ T from_u32(uint32_t w) {
    T v;
    *reinterpret_cast<uint32_t *>(&v) = w;
    return v;
}

// Publishes (flag, value) for tile t.
template <class T>
__device__ __forceinline__ void ls_publish(uint64_t *flags, T *vals, uint32_t t, uint32_t epoch, uint64_t flag,
                                           const T &v) {
    if constexpr (sizeof(T) == 4) {
        os_store(flags + t, os_word(epoch, flag, as_u32(v)));
    } else {
        st_cg_words(vals + t, v);
        st_release_u64(flags + t, os_word(epoch, flag, 0));
    }
}

template <class T> __device__ __forceinline__ void st_cg_words(T *p, const T &v) {
    static_assert(sizeof(T) % 4 == 0, "scan values are whole 32-bit words");
    const uint32_t *s = reinterpret_cast<const uint32_t *>(&v);
    uint32_t *d = reinterpret_cast<uint32_t *>(p);
#pragma unroll
    for (int i = 0; i < (int)(sizeof(T) / 4); i++) __stcg(d + i, s[i]);
}
template <class T> __device__ __forceinline__ T ld_cg_words(const T *p) {
    T v;
    uint32_t *d = reinterpret_cast<uint32_t *>(&v);
    const uint32_t *s = reinterpret_cast<const uint32_t *>(p);
#pragma unroll
    for (int i = 0; i < (int)(sizeof(T) / 4); i++) d[i] = __ldcg(s + i);
    return v;
}
template <class T> __device__ __forceinline__ T shfl_words(const T &v, int src) {
    T r;
    const uint32_t *s = reinterpret_cast<const uint32_t *>(&v);
    uint32_t *d = reinterpret_cast<uint32_t *>(&r);
#pragma unroll
    for (int i = 0; i < (int)(sizeof(T) / 4); i++) d[i] = __shfl_sync(FULL_MASK, s[i], src);
    return r;
}

template <class T, class Op, class Load, class Store>
__global__ void __launch_bounds__(LS_BLOCK) k_lbscan(Load ld, Store st, uint64_t n, Op op, uint64_t *flags, T *aggs,
                                                     T *prefs, uint32_t *ticket, uint32_t epoch, uint32_t ntiles,
                                                     T *total_out, uint32_t *err) {
    constexpr int IPT = ls_ipt<T>();
    constexpr int TILE = LS_BLOCK * IPT;
    constexpr bool PACKED = sizeof(T) == 4;
    __shared__ T smem[33];
    __shared__ T s_excl;
    __shared__ uint32_t s_tile;
    if (threadIdx.x == 0) s_tile = atomicAdd(ticket, 1u);
    __syncthreads();
    const uint32_t tile = s_tile;
    const uint64_t base = (uint64_t)tile * TILE;
    T v[IPT];
    T acc = Op::identity();
#pragma unroll
    for (int k = 0; k < IPT; k++) {
        const uint64_t i = base + (uint64_t)threadIdx.x * IPT + k;
        v[k] = i < n ? ld(i) : Op::identity();
        acc = op(acc, v[k]);
    }
    T ex, tot;
    block_scan<T, Op, LS_BLOCK>(acc, op, smem, &ex, &tot);
    if (threadIdx.x < 32) {
        const uint32_t lane = threadIdx.x;
        T excl = Op::identity();
        if (tile == 0) {
            if (lane == 0) ls_publish(flags, prefs, 0, epoch, OS_FLAG_PREFIX, tot);
        } else {
            if (lane == 0) ls_publish(flags, aggs, tile, epoch, OS_FLAG_AGG, tot);
            int64_t top = (int64_t)tile - 1;  // nearest tile not yet accounted for
            uint32_t spins = 0;
            while (true) {
                const int64_t t = top - (int64_t)lane;
                bool ready = true;
                uint32_t fl = (uint32_t)OS_FLAG_PREFIX;  // below tile 0: an empty prefix
                uint64_t f = 0;
                if (t >= 0) {
                    f = PACKED ? os_load(flags + t) : ld_acquire_u64(flags + t);
                    fl = (uint32_t)((f >> 32) & 3ull);
                    ready = (uint32_t)(f >> 34) == epoch && fl != 0;
                }
                const uint32_t pmask = __ballot_sync(FULL_MASK, ready && fl == (uint32_t)OS_FLAG_PREFIX);
                const uint32_t nready = __ballot_sync(FULL_MASK, !ready);
                const int last = pmask ? __ffs(pmask) - 1 : 31;  // lanes 0..last are needed
                const uint32_t need = last == 31 ? FULL_MASK : ((1u << (last + 1)) - 1u);
                if (nready & need) {
                    if (++spins > LS_SPIN_LIMIT) {
                        dev_fail(err, DEVERR_TIMEOUT);
                        break;
                    }
                    continue;
                }
                T val = Op::identity();
                if ((int)lane <= last && t >= 0) {
                    if constexpr (PACKED) val = from_u32<T>((uint32_t)f);
                    else val = fl == (uint32_t)OS_FLAG_PREFIX ? ld_cg_words(prefs + t) : ld_cg_words(aggs + t);
                }
                val = shfl_words(warp_scan_inclusive(val, op), 31);
                excl = op(excl, val);
                if (pmask) break;
                top -= 32;
            }
            if (lane == 0) ls_publish(flags, prefs, tile, epoch, OS_FLAG_PREFIX, op(excl, tot));
        }
        if (lane == 0) {
            s_excl = excl;
            if (tile == ntiles - 1 && total_out) *total_out = op(excl, tot);
        }
    }
    __syncthreads();
    T run = threadIdx.x == 0 ? s_excl : op(s_excl, ex);
#pragma unroll
    for (int k = 0; k < IPT; k++) {
        const uint64_t i = base + (uint64_t)threadIdx.x * IPT + k;
        if (i < n) st(i, run, v[k]);
        run = op(run, v[k]);
    }
}

// Runs the scan; `total_out` (device, nullable) receives the aggregate of
// all items (the identity when n == 0).
template <class T, class Op, class Load, class Store>
status_t lb_scan(Load ld, Store st, uint64_t n, T *total_out, Op op, ScanScratch &ss, OnesweepScratch &os,
                 uint32_t *err, cudaStream_t s, const char *pname = "scan") {
    static_assert(sizeof(T) <= LS_MAX_VALUE_BYTES, "scan value too large for the scratch");
    if (n == 0) {
        if (total_out) PSK_CUDA(cudaMemsetAsync(total_out, 0, sizeof(T), s));
        return PSACAK_OK;
    }
    const uint64_t ntiles = ceil_div(n, (uint64_t)LS_BLOCK * ls_ipt<T>());
    if (ntiles > ss.max_tiles)
        return set_error(PSACAK_EINTERNAL, "scan: %llu tiles exceed scratch", (unsigned long long)ntiles);
    os.epoch = (os.epoch + 1) & ((1u << 30) - 1);
    if (os.epoch == 0) os.epoch = 1;
    uint32_t *ticket = os.tickets + (os.epoch & 63);
    PSK_CUDA(cudaMemsetAsync(ticket, 0, sizeof(uint32_t), s));
    T *aggs = reinterpret_cast<T *>(ss.vals);
    T *prefs = aggs + ss.max_tiles;
    PSK_PROF_LAUNCH(s, pname, n, 0,
                    (k_lbscan<T, Op, Load, Store><<<(uint32_t)ntiles, LS_BLOCK, 0, s>>>(
                        ld, st, n, op, ss.flags, aggs, prefs, ticket, os.epoch, (uint32_t)ntiles, total_out, err)));
    PSK_LAUNCH_CHECK();
    return PSACAK_OK;
}

}  // namespace psk
