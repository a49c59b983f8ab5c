// radix.cuh -- LSD radix sort of (key, value) pairs on 8-bit digits.
//
// One histogram kernel reads the keys once and counts the digits of every
// pass; the host reads those counts (one sync per sort) and skips passes in
// which a single digit holds every key.  Each remaining pass is one
// onesweep kernel (single-pass stable scatter with decoupled look-back).
#pragma once

#include "onesweep.cuh"

namespace psk {

constexpr int RADIX_MAX_PASSES = 8;
constexpr int RADIX_HIST_BLOCK = 256;

template <class K, class V> struct RadixItem {
    K k;
    V v;
};

template <class K, class V> struct RadixPolicy {
    using Item = RadixItem<K, V>;
    static constexpr int kMinBlocks = sizeof(K) == 8 ? 3 : 4;
    const K *kin;
    const V *vin;
    K *kout;
    V *vout;
    int shift;
    uint32_t dmask;
    const uint32_t *base;  // 256 digit bases of this pass
    __device__ __forceinline__ void load(uint64_t i, Item &it, uint32_t &d) const {
        it.k = kin[i];
        it.v = vin[i];
        d = (uint32_t)(it.k >> shift) & dmask;
    }
    __device__ __forceinline__ uint64_t out(uint32_t d, uint64_t r) const { return (uint64_t)base[d] + r; }
    __device__ __forceinline__ void store(uint64_t idx, const Item &it, uint32_t) const {
        kout[idx] = it.k;
        vout[idx] = it.v;
    }
    __device__ __forceinline__ void finish(uint32_t, uint32_t) const {}
};

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

// Exclusive digit bases per pass (one block of 256 threads per pass).
__global__ void k_radix_bases(const uint32_t *hist, uint32_t *bases);

template <class K, class V>
status_t radix_sort_pairs(K *k0, V *v0, K *k1, V *v1, uint64_t n, int begin_bit, int end_bit, uint32_t *d_hist,
                          uint32_t *h_hist, OnesweepScratch &sc, uint32_t *err, int *result_in_1, cudaStream_t s,
                          int ipt = 12) {
    *result_in_1 = 0;
    if (n <= 1 || end_bit <= begin_bit) return PSACAK_OK;
    const int npasses = (end_bit - begin_bit + 7) / 8;
    if (npasses > RADIX_MAX_PASSES) return set_error(PSACAK_EINTERNAL, "radix sort: too many passes");
    uint32_t *bases = d_hist + RADIX_MAX_PASSES * 256;
    PSK_CUDA(cudaMemsetAsync(d_hist, 0, RADIX_MAX_PASSES * 256 * sizeof(uint32_t), s));
    uint64_t g = ceil_div(n, RADIX_HIST_BLOCK * 16);
    PSK_PROF_LAUNCH(s, "radix_hist", n, n * sizeof(K),
                    (k_radix_hist<K><<<(uint32_t)(g < 1184 ? g : 1184), RADIX_HIST_BLOCK, 0, s>>>(
                        k0, n, begin_bit, npasses, end_bit, d_hist)));
    PSK_PROF_LAUNCH(s, "radix_bases", npasses * 256, 0, (k_radix_bases<<<npasses, 256, 0, s>>>(d_hist, bases)));
    PSK_CUDA(cudaMemcpyAsync(h_hist, d_hist, npasses * 256 * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    PSK_CUDA(cudaStreamSynchronize(s));
    K *ki = k0, *ko = k1;
    V *vi = v0, *vo = v1;
    int flip = 0;
    for (int p = 0; p < npasses; p++) {
        bool trivial = false;
        for (int d = 0; d < 256; d++)
            if (h_hist[p * 256 + d] == n) trivial = true;
        if (trivial) continue;
        int shift = begin_bit + 8 * p;
        int bits = end_bit - shift < 8 ? end_bit - shift : 8;
        RadixPolicy<K, V> pol{ki, vi, ko, vo, shift, (1u << bits) - 1, bases + p * 256};
        PSK_TRY((onesweep_ipt<RadixPolicy<K, V>>(pol, n, ipt, sc, err, s, "radix_pass",
                                                 2 * n * (sizeof(K) + sizeof(V)))));
        K *tk = ki; ki = ko; ko = tk;
        V *tv = vi; vi = vo; vo = tv;
        flip ^= 1;
    }
    *result_in_1 = flip;
    return PSACAK_OK;
}

}  // namespace psk
