// lbscan.cuh -- single-pass scan with decoupled look-back.
//
// `ld(i)` yields the value of item i; `st(i, excl, v)` is called once per
// item with its exclusive prefix over the whole range and its own value.
// Each CTA claims the next tile of LS_BLOCK * IPT items (atomic ticket, so
// tiles are claimed in order), loads its items once, scans them, publishes
// the tile aggregate and walks back over earlier tiles -- 32 at a time, one
// per lane -- until it meets one that has published its inclusive prefix.
// The items' values stay in registers between the load and the store, so
// every item is loaded exactly once and any number of tiles are in flight
// at once.
//
// Scan values are tuples of 32-bit fields combined field by field (sums and
// maxima); the Op says how (Op::kFields, Op::field(f, a, b)).  Every field
// is published in its own status word [epoch:30 | flag:2 | value:32] (one
// relaxed 64-bit store or load, as in the onesweep status words), and warp
// f of the CTA walks back for field f, so a wide value costs no more
// round trips than a 32-bit one.  Flags carry the launch epoch, so the
// status array never needs clearing and stale words read as "not ready".
// Every wait is bounded by LS_SPIN_LIMIT polls, after which DEVERR_TIMEOUT
// is recorded and the CTA goes on.  A tile's predecessors have all been
// claimed by running CTAs, so the walk ends in normal operation.
//
// A Load may declare `using Payload = P;` and provide `T operator()(i, P&)`:
// whatever the store needs besides the prefix (gathered values, ranks) is
// then read in the load phase, where its latency overlaps the scan and the
// look-back, and handed to `st(i, excl, v, payload)`.  A Load may also set
// `static constexpr int kIPT` (items per thread) when its payload is large.
#pragma once

#include <type_traits>

#include "onesweep.cuh"

namespace psk {

constexpr int LS_BLOCK = 256;
constexpr int LS_IPT_MIN = 4;  // smallest tile: 1024 items (sizes the scratch)
constexpr int LS_TILE_MIN = LS_BLOCK * LS_IPT_MIN;
constexpr int LS_MAX_FIELDS = 4;
constexpr uint32_t LS_SPIN_LIMIT = 1u << 24;

// Payload plumbing: loads without a Payload type carry an empty one.
struct NoPayload {};
template <class L, class = void> struct scan_payload {
    using type = NoPayload;
    static constexpr bool has = false;
};
template <class L> struct scan_payload<L, std::void_t<typename L::Payload>> {
    using type = typename L::Payload;
    static constexpr bool has = true;
};
template <class L, class = void> struct scan_ipt_of {
    static constexpr int value = 0;
};
template <class L> struct scan_ipt_of<L, std::void_t<decltype(L::kIPT)>> {
    static constexpr int value = L::kIPT;
};
// A Load with `using Pre = Q;`, `void pre(i, Q&)` and `T operator()(i, const
// Q&, P&)` loads in two phases: pre() for every item of the thread (its
// direct operands, all in flight together), then the value and payload,
// whose dependent gathers are again issued together.
template <class L, class = void> struct scan_two_phase : std::false_type {};
template <class L> struct scan_two_phase<L, std::void_t<typename L::Pre>> : std::true_type {};
// Items per thread: the Load's choice, else 16 for 32-bit values and 8 for
// wider ones.
template <class T, class Load> constexpr int scan_ipt() {
    return scan_ipt_of<Load>::value ? scan_ipt_of<Load>::value : (sizeof(T) == 4 ? 16 : 8);
}

struct ScanScratch {
    uint64_t *flags = nullptr;  // LS_MAX_FIELDS status words per tile
    uint64_t max_tiles = 0;
};

template <class T> __device__ __forceinline__ uint32_t word_of(const T &v, int f) {
    return reinterpret_cast<const uint32_t *>(&v)[f];
}
template <class T> __device__ __forceinline__ void set_word(T &v, int f, uint32_t w) {
    reinterpret_cast<uint32_t *>(&v)[f] = w;
}

// `dn` (nullable): the item count lives on the device (written by an earlier
// kernel); the launch covers n_max items and the tiles past the count exit
// at once (with no items at all, tile 0 writes the identity as the total).
// At least 4 CTAs per SM (64 registers a thread): the scans wait on memory,
// and a fourth CTA's loads in flight are worth more than the registers it
// takes (the round scans of the 1 GiB build: 36.2 ms, against 36.8 ms at 3
// CTAs and 76 registers).
constexpr int LS_MIN_BLOCKS = 4;
template <class T, class Op, class Load, class Store>
__global__ void __launch_bounds__(LS_BLOCK, LS_MIN_BLOCKS) k_lbscan(Load ld, Store st, uint64_t n_max, Op op, uint64_t *flags,
                                                     uint32_t *ticket, uint32_t epoch, uint32_t ntiles_max,
                                                     T *total_out, uint32_t *err, const uint32_t *dn) {
    constexpr int IPT = scan_ipt<T, Load>();
    constexpr int TILE = LS_BLOCK * IPT;
    constexpr int NF = Op::kFields;
    static_assert(NF * 4 == (int)sizeof(T) && NF <= LS_MAX_FIELDS, "scan value = Op::kFields 32-bit fields");
    static_assert(IPT >= LS_IPT_MIN, "tile below the scratch's sizing");
    using PL = scan_payload<Load>;
    __shared__ T smem[33];
    __shared__ uint32_t s_excl[NF];
    __shared__ uint32_t s_tile;
    if (threadIdx.x == 0) s_tile = atomicAdd(ticket, 1u);
    __syncthreads();
    const uint32_t tile = s_tile;
    uint64_t n = n_max;
    uint32_t ntiles = ntiles_max;
    if (dn) {
        const uint64_t d = *dn;
        if (d > n_max && tile == 0 && threadIdx.x == 0) dev_fail(err, DEVERR_RANGE);
        n = d < n_max ? d : n_max;
        ntiles = (uint32_t)((n + TILE - 1) / TILE);
        if (tile >= ntiles) {
            if (tile == 0 && threadIdx.x == 0 && total_out) *total_out = Op::identity();
            return;
        }
    }
    const uint64_t base = (uint64_t)tile * TILE;
    T v[IPT];
    typename PL::type pl[IPT];
    T acc = Op::identity();
    if constexpr (scan_two_phase<Load>::value) {
        typename Load::Pre pre[IPT];
#pragma unroll
        for (int k = 0; k < IPT; k++) {
            const uint64_t i = base + (uint64_t)threadIdx.x * IPT + k;
            if (i < n) ld.pre(i, pre[k]);
        }
#pragma unroll
        for (int k = 0; k < IPT; k++) {
            const uint64_t i = base + (uint64_t)threadIdx.x * IPT + k;
            v[k] = i < n ? ld(i, pre[k], pl[k]) : Op::identity();
            acc = op(acc, v[k]);
        }
    } else {
#pragma unroll
        for (int k = 0; k < IPT; k++) {
            const uint64_t i = base + (uint64_t)threadIdx.x * IPT + k;
            if constexpr (PL::has) v[k] = i < n ? ld(i, pl[k]) : Op::identity();
            else v[k] = i < n ? ld(i) : Op::identity();
            acc = op(acc, v[k]);
        }
    }
    T ex, tot;
    block_scan<T, Op, LS_BLOCK>(acc, op, smem, &ex, &tot);
    const int w = threadIdx.x >> 5;
    if (w < NF) {
        const int f = w;
        const uint32_t lane = threadIdx.x & 31;
        const uint32_t tot_f = word_of(tot, f);
        const uint32_t id_f = word_of(Op::identity(), f);
        uint32_t excl = id_f;
        if (tile == 0) {
            if (lane == 0) os_store(flags + f, os_word(epoch, OS_FLAG_PREFIX, tot_f));
        } else {
            if (lane == 0) os_store(flags + (uint64_t)tile * NF + f, os_word(epoch, OS_FLAG_AGG, tot_f));
            int64_t top = (int64_t)tile - 1;  // nearest tile not yet accounted for
            uint32_t left = 0;  // poll budget (spin_spend)
            while (true) {
                const int64_t t = top - (int64_t)lane;
                bool ready = true;
                uint32_t fl = (uint32_t)OS_FLAG_PREFIX;  // below tile 0: an empty prefix
                uint32_t val = id_f;
                if (t >= 0) {
                    const uint64_t word = os_load(flags + (uint64_t)t * NF + f);
                    fl = (uint32_t)((word >> 32) & 3ull);
                    ready = (uint32_t)(word >> 34) == epoch && fl != 0;
                    val = (uint32_t)word;
                }
                const uint32_t pmask = __ballot_sync(FULL_MASK, ready && fl == (uint32_t)OS_FLAG_PREFIX);
                const uint32_t nready = __ballot_sync(FULL_MASK, !ready);
                const int last = pmask ? __ffs(pmask) - 1 : 31;  // lanes 0..last are needed
                const uint32_t need = last == 31 ? FULL_MASK : ((1u << (last + 1)) - 1u);
                if (nready & need) {
                    if (spin_spend(left, err, LS_SPIN_LIMIT)) {
                        dev_fail(err, DEVERR_TIMEOUT);
                        break;
                    }
                    continue;
                }
                if ((int)lane > last) val = id_f;
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) val = Op::field(f, val, __shfl_xor_sync(FULL_MASK, val, o));
                excl = Op::field(f, excl, val);
                if (pmask) break;
                top -= 32;
            }
            if (lane == 0)
                os_store(flags + (uint64_t)tile * NF + f, os_word(epoch, OS_FLAG_PREFIX, Op::field(f, excl, tot_f)));
        }
        if (lane == 0) s_excl[f] = excl;
    }
    __syncthreads();
    T tex;
#pragma unroll
    for (int f = 0; f < NF; f++) set_word(tex, f, s_excl[f]);
    if (threadIdx.x == 0 && tile == ntiles - 1 && total_out) *total_out = op(tex, tot);
    T run = threadIdx.x == 0 ? tex : op(tex, ex);
#pragma unroll
    for (int k = 0; k < IPT; k++) {
        const uint64_t i = base + (uint64_t)threadIdx.x * IPT + k;
        if constexpr (PL::has) {
            if (i < n) st(i, run, v[k], pl[k]);
        } else {
            if (i < n) st(i, run, v[k]);
        }
        run = op(run, v[k]);
    }
}

// Runs the scan; `total_out` (device, nullable) receives the aggregate of
// all items (the identity when n == 0).
// `dn` (nullable): the item count is read on the device (at most n).
// `bytes`: the launch's algorithmic bytes for the profiler (0: no model).
template <class T, class Op, class Load, class Store>
status_t lb_scan(Load ld, Store st, uint64_t n, T *total_out, Op op, ScanScratch &ss, OnesweepScratch &os,
                 uint32_t *err, cudaStream_t s, const char *pname = "scan", const uint32_t *dn = nullptr,
                 uint64_t bytes = 0) {
    if (n == 0) {
        if (total_out) PSK_CUDA(cudaMemsetAsync(total_out, 0, sizeof(T), s));
        return PSACAK_OK;
    }
    const uint64_t ntiles = ceil_div(n, (uint64_t)LS_BLOCK * scan_ipt<T, Load>());
    if (ntiles > ss.max_tiles)
        return set_error(PSACAK_EINTERNAL, "scan: %llu tiles exceed scratch", (unsigned long long)ntiles);
    os.epoch = (os.epoch + 1) & ((1u << 30) - 1);
    if (os.epoch == 0) os.epoch = 1;
    uint32_t *ticket = os.tickets + (os.epoch & 63);
    PSK_CUDA(cudaMemsetAsync(ticket, 0, sizeof(uint32_t), s));
    PSK_PROF_LAUNCH(s, pname, n, bytes,
                    (k_lbscan<T, Op, Load, Store><<<(uint32_t)ntiles, LS_BLOCK, 0, s>>>(
                        ld, st, n, op, ss.flags, ticket, os.epoch, (uint32_t)ntiles, total_out, err, dn)));
    PSK_LAUNCH_CHECK();
    return PSACAK_OK;
}

}  // namespace psk
