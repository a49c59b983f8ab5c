// radix.cuh -- LSD radix sort of (key, value) pairs on 8-bit digits.
//
// One histogram kernel reads the keys once and counts the digits of every
// pass; for sorts of RADIX_PROBE_MIN keys or more the host reads those
// counts (one sync per sort) and skips passes in which a single digit holds
// every key.  Shorter sorts run every pass without that round trip (a pass
// over fewer keys costs less than the read-back).  Each pass is one
// onesweep kernel (single-pass stable scatter with decoupled look-back).
#pragma once

#include "onesweep.cuh"
#include "tma.cuh"

namespace psk {

constexpr int RADIX_MAX_PASSES = 8;
constexpr uint64_t RADIX_PROBE_MIN = 1ull << 20;
constexpr int RADIX_HIST_BLOCK = 256;

// One radix pass as a TMA-fed onesweep tile.  A full tile's keys and values
// arrive in shared memory by two bulk copies on an mbarrier (the ragged last
// tile, or unaligned arrays, use plain loads), so no item is held in a
// register while its load is in flight.  Items are ranked from shared
// memory exactly as in k_onesweep (stable per-warp ranks, decoupled
// look-back per digit), and the staging permutes 16-bit tile indices instead
// of whole items: the scatter reads s_perm[i] and copies that item to
// digit base + i, so consecutive threads write consecutive slots of a digit.
// Shared memory: TILE * (sizeof(K) + sizeof(V) + 2) + 6.3 KB.
// Stable ranks of the warp's IPT x 32 items of the tile (item idx = warp *
// 32 * IPT + r * 32 + lane) by the digit (key >> shift) & dmask: rd[r] =
// rank within the warp << 9 | digit (256 = no item); wcnt = the warp's digit
// counters.  FULL: all TILE items are present (no validity tests).
template <class K, int IPT, bool FULL>
__device__ __forceinline__ void radix_rank(const K *s_k, uint32_t cnt, int shift, uint32_t dmask, uint16_t *wcnt,
                                           uint32_t (&rd)[IPT]) {
    const int w = threadIdx.x >> 5;
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t lt = lanemask_lt();
#pragma unroll
    for (int r = 0; r < IPT; r++) {
        const uint32_t idx = (uint32_t)w * 32 * IPT + (uint32_t)r * 32 + lane;
        const bool valid = FULL || idx < cnt;
        // the digit lies in one 32-bit half of the key (shift is a multiple of 8)
        const uint32_t half = sizeof(K) == 8 ? reinterpret_cast<const uint32_t *>(s_k)[2 * idx + (shift >> 5)]
                                             : (uint32_t)s_k[idx];
        const uint32_t d = valid ? (half >> (shift & 31)) & dmask : 256u;
        // lanes with the same digit: the intersection of eight bit ballots
        // (ALU votes instead of one match.any through the MIO pipe)
        uint32_t peers = FULL_MASK;
        if (!FULL) {
            peers = __ballot_sync(FULL_MASK, valid);
            if (!valid) peers = ~peers;
        }
#pragma unroll
        for (int b = 0; b < 8; b++) {
            const uint32_t bit = (d >> b) & 1u;
            const uint32_t bb = __ballot_sync(FULL_MASK, bit);
            peers &= bit ? bb : ~bb;
        }
        const uint32_t prior = (FULL || d < 256) ? wcnt[d] : 0u;
        rd[r] = ((prior + __popc(peers & lt)) << 9) | d;
        __syncwarp();
        if ((FULL || d < 256) && (int)lane == __ffs(peers) - 1) wcnt[d] = (uint16_t)(prior + __popc(peers));
        __syncwarp();
    }
}

constexpr int RS_MIN_BLOCKS = 4;
constexpr int RADIX_IPT = 12;  // items per thread of the radix passes (3072-item tiles)

// `dn` (nullable): the key count is read on the device (at most n_max, the
// count the grid was sized for); tiles past it exit at once.
template <class K, class V, int IPT>
__global__ void __launch_bounds__(OS_BLOCK, RS_MIN_BLOCKS)
    k_radix_pass(const K *__restrict__ kin, const V *__restrict__ vin, K *__restrict__ kout, V *__restrict__ vout,
                 int shift, uint32_t dmask, const uint32_t *__restrict__ dbase, uint64_t n_max, int bulk_ok,
                 uint64_t *status, uint32_t *ticket, uint32_t epoch, uint32_t *err, const uint32_t *dn) {
    constexpr int TILE = OS_BLOCK * IPT;
    extern __shared__ __align__(128) unsigned char rs_smem[];
    K *s_k = (K *)rs_smem;
    V *s_v = (V *)(s_k + TILE);
    uint16_t *s_perm = (uint16_t *)(s_v + TILE);
    __shared__ __align__(8) uint64_t s_bar;
    __shared__ uint32_t s_gbase[256];
    __shared__ uint32_t s_tstart[256];
    __shared__ uint16_t s_wcnt[OS_WARPS][256];
    __shared__ uint32_t s_scan[33];
    __shared__ uint32_t s_tile;
    __shared__ uint32_t s_hist[256];

    const int w = threadIdx.x >> 5;
    const uint32_t lane = threadIdx.x & 31;

    if (threadIdx.x == 0) {
        s_tile = atomicAdd(ticket, 1u);
        mbar_init(&s_bar, 1);
    }
    for (int i = threadIdx.x; i < OS_WARPS * 256; i += OS_BLOCK) (&s_wcnt[0][0])[i] = 0;
    s_hist[threadIdx.x] = 0;
    __syncthreads();
    const uint32_t tile = s_tile;
    const uint64_t base = (uint64_t)tile * TILE;
    uint64_t n = n_max;
    if (dn) {
        const uint64_t d = *dn;
        n = d < n_max ? d : n_max;
        if (base >= n) return;  // the whole CTA: no copy was issued
    }
    const uint32_t cnt = (uint32_t)(n - base < (uint64_t)TILE ? n - base : (uint64_t)TILE);
    const bool bulk = bulk_ok && cnt == (uint32_t)TILE;
    if (bulk) {
        if (threadIdx.x == 0) {
            mbar_arrive_expect_tx(&s_bar, TILE * (uint32_t)(sizeof(K) + sizeof(V)));
            bulk_g2s(s_k, kin + base, TILE * (uint32_t)sizeof(K), &s_bar);
            bulk_g2s(s_v, vin + base, TILE * (uint32_t)sizeof(V), &s_bar);
        }
        // one outcome for the whole CTA: the ranking below uses
        // __syncthreads and full-warp ballots
        if (!mbar_wait_cta(&s_bar, 0, err)) return;
    } else {
        for (uint32_t i = threadIdx.x; i < cnt; i += OS_BLOCK) {
            s_k[i] = kin[base + i];
            s_v[i] = vin[base + i];
        }
        __syncthreads();
    }

    // early counts: the tile's digit counts by shared-memory atomics, published
    // before the ranking so that later tiles' look-backs find them sooner (a
    // measured 3.5% off the pass time; the ranking's own counts equal them)
    {
#pragma unroll
        for (int r = 0; r < IPT; r++) {
            const uint32_t idx = (uint32_t)w * 32 * IPT + (uint32_t)r * 32 + lane;
            if (idx < cnt) {
                const uint32_t half = sizeof(K) == 8 ? reinterpret_cast<const uint32_t *>(s_k)[2 * idx + (shift >> 5)]
                                                     : (uint32_t)s_k[idx];
                atomicAdd(&s_hist[(half >> (shift & 31)) & dmask], 1u);
            }
        }
        __syncthreads();
        uint64_t *my = status + (uint64_t)tile * 256 + threadIdx.x;
        os_store(my, os_word(epoch, tile == 0 ? OS_FLAG_PREFIX : OS_FLAG_AGG, s_hist[threadIdx.x]));
    }
    // stable ranks within the warp's sub-tile; packed (rank << 9 | digit)
    uint32_t rd[IPT];
    if (cnt == (uint32_t)TILE) radix_rank<K, IPT, true>(s_k, cnt, shift, dmask, s_wcnt[w], rd);
    else radix_rank<K, IPT, false>(s_k, cnt, shift, dmask, s_wcnt[w], rd);
    __syncthreads();
    const uint32_t d = threadIdx.x;  // this thread's digit from here on
    uint32_t count = 0;
#pragma unroll
    for (int ww = 0; ww < OS_WARPS; ww++) {
        uint32_t c = s_wcnt[ww][d];
        s_wcnt[ww][d] = (uint16_t)count;
        count += c;
    }
    const uint32_t excl = os_lookback<1, true>(status, tile, d, count, epoch, err);
    uint32_t ex, tot;
    block_scan<uint32_t, OpSum<uint32_t>, OS_BLOCK>(count, OpSum<uint32_t>(), s_scan, &ex, &tot);
    s_tstart[d] = ex;
    s_gbase[d] = dbase[d] + excl - ex;  // global slot of tile position i = s_gbase[digit] + i
    __syncthreads();
#pragma unroll
    for (int r = 0; r < IPT; r++) {
        const uint32_t dd = rd[r] & 511u;
        if (dd < 256) {
            const uint32_t idx = (uint32_t)w * 32 * IPT + (uint32_t)r * 32 + lane;
            s_perm[s_tstart[dd] + s_wcnt[w][dd] + (rd[r] >> 9)] = (uint16_t)idx;
        }
    }
    __syncthreads();
    // n < 2^32 items: 32-bit output slots
    const uint32_t n32 = (uint32_t)n;
    for (uint32_t i = threadIdx.x; i < cnt; i += OS_BLOCK) {
        const uint32_t li = s_perm[i];
        const K k = s_k[li];
        const uint32_t half = sizeof(K) == 8 ? (uint32_t)(shift >= 32 ? (uint64_t)k >> 32 : (uint64_t)k) : (uint32_t)k;
        const uint32_t o = s_gbase[(half >> (shift & 31)) & dmask] + i;
        if (o < n32) {
            kout[o] = k;
            vout[o] = s_v[li];
        } else {
            dev_fail(err, DEVERR_RANGE);
        }
    }
}

template <class K, class V, int IPT>
status_t radix_pass(const K *kin, const V *vin, K *kout, V *vout, int shift, uint32_t dmask, const uint32_t *dbase,
                    uint64_t n, OnesweepScratch &sc, uint32_t *err, cudaStream_t s, const uint32_t *dn = nullptr) {
    constexpr int TILE = OS_BLOCK * IPT;
    const uint64_t ntiles = ceil_div(n, TILE);
    if (ntiles > sc.max_tiles) return set_error(PSACAK_EINTERNAL, "radix pass: %llu tiles exceed scratch", (unsigned long long)ntiles);
    if (TILE > 65536) return set_error(PSACAK_EINTERNAL, "radix pass: tile too large");
    sc.epoch = (sc.epoch + 1) & ((1u << 30) - 1);
    if (sc.epoch == 0) sc.epoch = 1;
    uint32_t *ticket = sc.tickets + (sc.epoch & 63);
    PSK_CUDA(cudaMemsetAsync(ticket, 0, sizeof(uint32_t), s));
    const int bulk_ok = ((((uintptr_t)kin) | ((uintptr_t)vin)) & 15u) == 0;
    const size_t smem = (size_t)TILE * (sizeof(K) + sizeof(V) + 2);
    PSK_CUDA(cudaFuncSetAttribute(k_radix_pass<K, V, IPT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    PSK_PROF_LAUNCH(s, "radix_pass", n, 2 * n * (sizeof(K) + sizeof(V)),
                    (k_radix_pass<K, V, IPT><<<(uint32_t)ntiles, OS_BLOCK, smem, s>>>(
                        kin, vin, kout, vout, shift, dmask, dbase, n, bulk_ok, sc.status, ticket, sc.epoch, err, dn)));
    PSK_LAUNCH_CHECK();
    return PSACAK_OK;
}

// Digit counts of every pass: hist[p * 256 + d].
template <class K>
__global__ void __launch_bounds__(RADIX_HIST_BLOCK) k_radix_hist(const K *__restrict__ keys, uint64_t n, int begin_bit,
                                                                 int npasses, int end_bit, uint32_t *hist) {
    __shared__ uint32_t sh[RADIX_MAX_PASSES * 256];
    for (int i = threadIdx.x; i < RADIX_MAX_PASSES * 256; i += RADIX_HIST_BLOCK) sh[i] = 0;
    __syncthreads();
    const uint32_t lane = threadIdx.x & 31;
    for (uint64_t base = (uint64_t)blockIdx.x * RADIX_HIST_BLOCK; base < n; base += (uint64_t)gridDim.x * RADIX_HIST_BLOCK) {
        uint64_t i = base + threadIdx.x;
        bool valid = i < n;
        K k = valid ? keys[i] : K(0);
        for (int p = 0; p < npasses; p++) {
            int shift = begin_bit + 8 * p;
            int bits = end_bit - shift < 8 ? end_bit - shift : 8;
            uint32_t d = (uint32_t)(k >> shift) & ((1u << bits) - 1);
            // warp fast path: every lane has the same digit
            uint32_t d0 = __shfl_sync(FULL_MASK, d, 0);
            uint32_t vmask = __ballot_sync(FULL_MASK, valid);
            if (__all_sync(FULL_MASK, !valid || d == d0)) {
                if (lane == 0) atomicAdd(&sh[p * 256 + d0], __popc(vmask));
            } else if (valid) {
                atomicAdd(&sh[p * 256 + d], 1u);
            }
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < npasses * 256; i += RADIX_HIST_BLOCK)
        if (sh[i]) atomicAdd(&hist[i], sh[i]);
}

// Digit counting for kernels that produce radix keys: each thread of a
// block adds its key (valid or not: every lane of the warp must call it) to
// the block's shared histograms sh[p * 256 + d]; radix_flush_digits adds
// them to the device histograms at the end of the block.
template <class K>
__device__ __forceinline__ void radix_count_digits(uint32_t *sh, K k, bool valid, int begin_bit, int npasses,
                                                   int end_bit) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t vmask = __ballot_sync(FULL_MASK, valid);
    for (int p = 0; p < npasses; p++) {
        int shift = begin_bit + 8 * p;
        int bits = end_bit - shift < 8 ? end_bit - shift : 8;
        uint32_t d = (uint32_t)(k >> shift) & ((1u << bits) - 1);
        uint32_t d0 = __shfl_sync(FULL_MASK, d, 0);
        if (__all_sync(FULL_MASK, !valid || d == d0)) {
            if (lane == 0 && vmask) atomicAdd(&sh[p * 256 + d0], __popc(vmask));
        } else if (valid) {
            atomicAdd(&sh[p * 256 + d], 1u);
        }
    }
}
__device__ __forceinline__ void radix_flush_digits(const uint32_t *sh, int npasses, uint32_t *hist) {
    for (int i = threadIdx.x; i < npasses * 256; i += blockDim.x)
        if (sh[i]) atomicAdd(&hist[i], sh[i]);
}

// Exclusive digit bases per pass (one block of 256 threads per pass).
__global__ void k_radix_bases(const uint32_t *hist, uint32_t *bases);

// dst[i] = src[i] for i < count, by one block (small copies that must not
// wait for a copy engine).
__global__ void k_copy_words(const uint32_t *__restrict__ src, uint32_t *dst, uint32_t count);

// Reads `count` words back to the host: a one-block kernel stores them into
// `mapped` (the device view of pinned, mapped host memory) and the stream is
// synchronised.  Unlike a device-to-host memcpy this does not queue behind
// bulk copies that a copy engine is working through on another stream.
status_t read_back(const uint32_t *d, uint32_t *mapped, uint32_t count, cudaStream_t s);

// When `hist_ready` is set, the producer of the keys has already counted
// the digits of every pass into d_hist (see radix_count_digits), and the
// histogram kernel is skipped.  `dn` (nullable): the key count is on the
// device, n is its bound; every pass runs (nothing to probe on the host).
template <class K, class V>
status_t radix_sort_pairs(K *k0, V *v0, K *k1, V *v1, uint64_t n, int begin_bit, int end_bit, uint32_t *d_hist,
                          uint32_t *h_hist, uint32_t *h_hist_mapped, OnesweepScratch &sc, uint32_t *err, int *result_in_1, cudaStream_t s,
                          int ipt = 12, bool hist_ready = false, const uint32_t *dn = nullptr) {
    *result_in_1 = 0;
    if (n <= 1 || end_bit <= begin_bit) return PSACAK_OK;
    const int npasses = (end_bit - begin_bit + 7) / 8;
    if (npasses > RADIX_MAX_PASSES) return set_error(PSACAK_EINTERNAL, "radix sort: too many passes");
    uint32_t *bases = d_hist + RADIX_MAX_PASSES * 256;
    if (!hist_ready) {
        PSK_CUDA(cudaMemsetAsync(d_hist, 0, RADIX_MAX_PASSES * 256 * sizeof(uint32_t), s));
        uint64_t g = ceil_div(n, RADIX_HIST_BLOCK * 16);
        PSK_PROF_LAUNCH(s, "radix_hist", n, n * sizeof(K),
                        (k_radix_hist<K><<<(uint32_t)(g < 1184 ? g : 1184), RADIX_HIST_BLOCK, 0, s>>>(
                            k0, n, begin_bit, npasses, end_bit, d_hist)));
    }
    PSK_PROF_LAUNCH(s, "radix_bases", npasses * 256, 0, (k_radix_bases<<<npasses, 256, 0, s>>>(d_hist, bases)));
    if (dn && !hist_ready) return set_error(PSACAK_EINTERNAL, "radix sort: a device count needs counted digits");
    const bool probe = !dn && n >= RADIX_PROBE_MIN;
    if (probe) PSK_TRY(read_back(d_hist, h_hist_mapped, npasses * 256, s));
    K *ki = k0, *ko = k1;
    V *vi = v0, *vo = v1;
    int flip = 0;
    for (int p = 0; p < npasses; p++) {
        bool trivial = false;
        if (probe)
            for (int d = 0; d < 256; d++)
                if (h_hist[p * 256 + d] == n) trivial = true;
        if (trivial) continue;
        int shift = begin_bit + 8 * p;
        int bits = end_bit - shift < 8 ? end_bit - shift : 8;
        const uint32_t dmask = (1u << bits) - 1;
        if (ipt == 8) {
            PSK_TRY((radix_pass<K, V, 8>(ki, vi, ko, vo, shift, dmask, bases + p * 256, n, sc, err, s, dn)));
        } else if (ipt == 16) {
            PSK_TRY((radix_pass<K, V, 16>(ki, vi, ko, vo, shift, dmask, bases + p * 256, n, sc, err, s, dn)));
        } else {
            PSK_TRY((radix_pass<K, V, 12>(ki, vi, ko, vo, shift, dmask, bases + p * 256, n, sc, err, s, dn)));
        }
        K *tk = ki; ki = ko; ko = tk;
        V *tv = vi; vi = vo; vo = tv;
        flip ^= 1;
    }
    *result_in_1 = flip;
    return PSACAK_OK;
}

}  // namespace psk
