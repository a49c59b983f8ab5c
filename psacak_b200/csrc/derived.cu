// derived.cu -- arrays derived from a suffix array on the device: the
// inverse suffix array, the Burrows-Wheeler transform and the LCP array.
// None of them is in hucsmn/psacak; they are the usual consumers of its
// output.  The suffix array excludes the sentinel (the reference's
// convention, src/lib.rs:30-43).
//
// LCP uses the permuted-LCP method (Kaerkkaeinen, Manzini, Puglisi,
// "Permuted longest-common-prefix array", CPM 2009):
//   phi[SA[i]] = SA[i-1], the suffix just before SA[i] in suffix order;
//   PLCP[j] = lcp(j, phi[j]), and LCP[i] = PLCP[SA[i]];
//   j is reducible when text[j-1] == text[phi[j]-1]: then phi[j-1] =
//   phi[j] - 1 and PLCP[j] = PLCP[j-1] - 1.
// Only irreducible positions compare characters (their PLCP values sum to
// O(n log n) for any text), the others take PLCP[r] - (j - r) from the last
// irreducible position r <= j, found by a max-scan.
#include "ctx.cuh"
#include "../../include/psacak_b200.h"

namespace psk {

void clear_error();

constexpr uint32_t PHI_NONE = 0xFFFFFFFFu;

__global__ void k_isa(const uint32_t *__restrict__ sa, uint64_t n, uint32_t *isa, uint32_t *err) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t v = sa[i];
        if (v < n) isa[v] = (uint32_t)i;
        else dev_fail(err, DEVERR_RANGE);
    }
}

__global__ void k_phi(const uint32_t *__restrict__ sa, uint64_t n, uint32_t *phi, uint32_t *err) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t v = sa[i];
        if (v < n) phi[v] = i > 0 ? sa[i - 1] : PHI_NONE;
        else dev_fail(err, DEVERR_RANGE);
    }
}

// Symbols one thread compares for an irreducible position before handing
// it to a whole CTA (k_plcp_long): a long run of one character has a single
// irreducible position whose PLCP is about the run's length, which one
// thread would walk alone.  Set high enough that the many irreducible
// positions of moderately long repeats (a genome's copies) stay with their
// threads, which run side by side.
constexpr uint32_t LCP_THREAD_MAX = 16384;
constexpr int LCP_LONG_BLOCK = 256;
constexpr int LCP_LONG_SYMS = 16;  // per thread and step: 4096 symbols per CTA step

// PLCP of the irreducible positions (by comparison) and their bitmap.
// Comparisons that reach LCP_THREAD_MAX symbols are listed in `longs` (up to
// `long_cap`; beyond it the thread goes on alone) with their PLCP so far.
template <class C>
__global__ void k_plcp_irreducible(const C *__restrict__ text, uint64_t n, const uint32_t *__restrict__ phi,
                                   uint32_t *plcp, uint32_t *irr, uint32_t *longs, uint32_t *nlong,
                                   uint32_t long_cap) {
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;  // a multiple of 32
    for (uint64_t jb = (uint64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31u); jb < n; jb += stride) {
        const uint64_t j = jb + lane;
        bool ir = false;
        if (j < n) {
            const uint32_t p = phi[j];
            ir = j == 0 || p == PHI_NONE || p == 0 || text[j - 1] != text[p - 1];
            if (ir) {
                uint64_t h = 0;
                if (p != PHI_NONE) {
                    while (h < LCP_THREAD_MAX && j + h < n && p + h < n && text[j + h] == text[p + h]) h++;
                    if (h == LCP_THREAD_MAX && j + h < n && p + h < n) {
                        const uint32_t slot = atomicAdd(nlong, 1u);
                        if (slot < long_cap) longs[slot] = (uint32_t)j;
                        else
                            while (j + h < n && p + h < n && text[j + h] == text[p + h]) h++;
                    }
                }
                plcp[j] = (uint32_t)h;
            }
        }
        const uint32_t word = __ballot_sync(FULL_MASK, ir);
        if (lane == 0 && jb < n) irr[jb >> 5] = word;
    }
}

// The listed long comparisons, one CTA each: every step compares the next
// LCP_LONG_BLOCK x LCP_LONG_SYMS symbols of both suffixes, each thread a
// stretch of LCP_LONG_SYMS, and the CTA takes the first mismatch.
template <class C>
__global__ void __launch_bounds__(LCP_LONG_BLOCK) k_plcp_long(const C *__restrict__ text, uint64_t n,
                                                             const uint32_t *__restrict__ phi, uint32_t *plcp,
                                                             const uint32_t *__restrict__ longs,
                                                             const uint32_t *nlong, uint32_t long_cap) {
    __shared__ uint32_t s_min[LCP_LONG_BLOCK / 32];
    const uint32_t count = *nlong < long_cap ? *nlong : long_cap;
    constexpr uint32_t STEP = LCP_LONG_BLOCK * LCP_LONG_SYMS;
    for (uint32_t it = blockIdx.x; it < count; it += gridDim.x) {
        const uint64_t j = longs[it];
        const uint64_t p = phi[j];
        uint64_t h = plcp[j];
        const uint64_t lim = n - (j > p ? j : p);  // both suffixes end at n
        while (true) {
            uint32_t first = 0xFFFFFFFFu;  // this thread's first mismatch in the step
            const uint64_t o = h + (uint64_t)threadIdx.x * LCP_LONG_SYMS;
            for (uint32_t k = 0; k < LCP_LONG_SYMS; k++) {
                const uint64_t q = o + k;
                if (q >= lim || text[j + q] != text[p + q]) {
                    first = (uint32_t)(q - h);
                    break;
                }
            }
            for (int d = 16; d > 0; d >>= 1) {
                const uint32_t other = __shfl_xor_sync(FULL_MASK, first, d);
                first = other < first ? other : first;
            }
            if ((threadIdx.x & 31) == 0) s_min[threadIdx.x >> 5] = first;
            __syncthreads();
            uint32_t m = 0xFFFFFFFFu;
            for (int w = 0; w < LCP_LONG_BLOCK / 32; w++) m = s_min[w] < m ? s_min[w] : m;
            __syncthreads();
            if (m != 0xFFFFFFFFu) {
                h += m;
                break;
            }
            h += STEP;
        }
        if (threadIdx.x == 0) plcp[j] = (uint32_t)h;
    }
}

// Reducible positions: PLCP[j] = PLCP[r] - (j - r), r = last irreducible <= j.
struct AnchorLoad {
    const uint32_t *irr;
    __device__ __forceinline__ uint32_t operator()(uint64_t j) const {
        return bm_get(irr, j) ? (uint32_t)(j + 1) : 0u;
    }
};
struct AnchorStore {
    uint32_t *plcp;
    uint32_t *err;
    __device__ __forceinline__ void operator()(uint64_t j, uint32_t excl, uint32_t v) const {
        if (v) return;  // irreducible: compared already
        if (excl == 0) {  // position 0 is irreducible, so every position has an anchor
            dev_fail(err, DEVERR_RANGE);
            return;
        }
        const uint64_t r = excl - 1;
        plcp[j] = plcp[r] - (uint32_t)(j - r);
    }
};

__global__ void k_lcp_gather(const uint32_t *__restrict__ sa, uint64_t n, const uint32_t *__restrict__ plcp,
                             uint32_t *lcp) {
    constexpr int U = 4;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i0 = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i0 < n; i0 += stride * U) {
        uint32_t s[U], v[U];
#pragma unroll
        for (int u = 0; u < U; u++) s[u] = i0 + u * stride < n ? sa[i0 + u * stride] : 0u;
#pragma unroll
        for (int u = 0; u < U; u++) v[u] = i0 + u * stride < n && s[u] < n ? plcp[s[u]] : 0u;
#pragma unroll
        for (int u = 0; u < U; u++)
            if (i0 + u * stride < n) lcp[i0 + u * stride] = v[u];
    }
}

// BWT rows in the divbwt convention: row 0 is the sentinel's rotation
// (character text[n-1]); row i+1 is SA[i], whose character is text[SA[i]-1],
// except the row of SA[i] = 0 (the primary index), which is left out.
__global__ void k_find_primary(const uint32_t *__restrict__ sa, uint64_t n, uint32_t *row) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        if (sa[i] == 0) *row = (uint32_t)i;
}
__global__ void k_bwt(const uint8_t *__restrict__ text, const uint32_t *__restrict__ sa, uint64_t n, uint32_t zrow,
                      uint8_t *bwt, uint32_t *err) {
    constexpr int U = 4;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    if (blockIdx.x == 0 && threadIdx.x == 0) bwt[0] = text[n - 1];
    for (uint64_t i0 = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i0 < n; i0 += stride * U) {
        uint32_t s[U];
        uint8_t c[U];
#pragma unroll
        for (int u = 0; u < U; u++) s[u] = i0 + u * stride < n ? sa[i0 + u * stride] : 0u;
#pragma unroll
        for (int u = 0; u < U; u++) c[u] = s[u] > 0 && s[u] <= n ? text[s[u] - 1] : 0;
#pragma unroll
        for (int u = 0; u < U; u++) {
            const uint64_t i = i0 + u * stride;
            if (i >= n || i == zrow) continue;
            if (s[u] > n) dev_fail(err, DEVERR_RANGE);
            bwt[i < zrow ? i + 1 : i] = c[u];
        }
    }
}

static inline uint32_t grid_for_n(uint64_t n, uint32_t cap = 16384) {
    uint64_t g = ceil_div(n ? n : 1, 256);
    return (uint32_t)(g < cap ? g : cap);
}

template <class C>
static int lcp_dev(psacak_ctx *ctx, const C *d_text, uint64_t n, const uint32_t *d_sa, uint32_t *d_lcp, void *stream) {
    clear_error();
    if (!ctx) return set_error(PSACAK_EINVAL, "null context");
    if (n >= 0xFFFFFFFFull) return set_error(PSACAK_EINVAL, "n = %llu is not below 2^32 - 1", (unsigned long long)n);
    if (n > 0 && (!d_text || !d_sa || !d_lcp)) return set_error(PSACAK_EINVAL, "null text, suffix-array or LCP pointer");
    std::lock_guard<std::mutex> g(ctx->c.mu);
    Ctx &c = ctx->c;
    PSK_CUDA(cudaSetDevice(c.dev.id));
    c.stream = stream ? (cudaStream_t)stream : c.own_stream;
    if (n == 0) return PSACAK_OK;
    cudaStream_t s = c.stream;
    DBuf<uint32_t> plcp, irr, longs;
    PSK_TRY(plcp.init(c, n));
    PSK_TRY(irr.init(c, ceil_div(n, 32) + 1));
    const uint32_t long_cap = (uint32_t)(n / 64 + 1024);
    PSK_TRY(longs.init(c, long_cap));
    uint32_t *nlong = c.d_scalars + 42;
    PSK_CUDA(cudaMemsetAsync(nlong, 0, sizeof(uint32_t), s));
    uint32_t *phi = d_lcp;  // the output holds phi until the final gather
    PSK_PROF_LAUNCH(s, "lcp_phi", n, 12ull * n, (k_phi<<<grid_for_n(n), 256, 0, s>>>(d_sa, n, phi, c.d_err)));
    PSK_PROF_LAUNCH(s, "lcp_irreducible", n, 0,
                    (k_plcp_irreducible<C><<<grid_for_n(n), 256, 0, s>>>(d_text, n, phi, plcp, irr, longs, nlong,
                                                                          long_cap)));
    PSK_PROF_LAUNCH(s, "lcp_long", n, 0,
                    (k_plcp_long<C><<<2 * (uint32_t)c.dev.num_sms, LCP_LONG_BLOCK, 0, s>>>(d_text, n, phi, plcp, longs,
                                                                                           nlong, long_cap)));
    PSK_TRY((c.scan<uint32_t, OpMax<uint32_t>>(AnchorLoad{irr}, AnchorStore{plcp, c.d_err}, n, (uint32_t *)nullptr,
                                               OpMax<uint32_t>(), "lcp_reducible")));
    PSK_PROF_LAUNCH(s, "lcp_gather", n, 12ull * n, (k_lcp_gather<<<grid_for_n(n), 256, 0, s>>>(d_sa, n, plcp, d_lcp)));
    PSK_LAUNCH_CHECK();
    PSK_TRY(c.sync());
    return c.check_device_error();
}

}  // namespace psk

using namespace psk;

extern "C" {

int psacak_isa_dev(psacak_ctx *ctx, const uint32_t *d_sa, uint64_t n, uint32_t *d_isa, void *stream) {
    clear_error();
    if (!ctx) return set_error(PSACAK_EINVAL, "null context");
    if (n >= 0xFFFFFFFFull) return set_error(PSACAK_EINVAL, "n = %llu is not below 2^32 - 1", (unsigned long long)n);
    if (n > 0 && (!d_sa || !d_isa)) return set_error(PSACAK_EINVAL, "null suffix-array or output pointer");
    std::lock_guard<std::mutex> g(ctx->c.mu);
    Ctx &c = ctx->c;
    PSK_CUDA(cudaSetDevice(c.dev.id));
    c.stream = stream ? (cudaStream_t)stream : c.own_stream;
    if (n == 0) return PSACAK_OK;
    PSK_PROF_LAUNCH(c.stream, "isa", n, 8ull * n, (k_isa<<<grid_for_n(n), 256, 0, c.stream>>>(d_sa, n, d_isa, c.d_err)));
    PSK_LAUNCH_CHECK();
    PSK_TRY(c.sync());
    return c.check_device_error();
}

int psacak_bwt8_dev(psacak_ctx *ctx, const uint8_t *d_text, uint64_t n, const uint32_t *d_sa, uint8_t *d_bwt,
                    uint64_t *primary, void *stream) {
    clear_error();
    if (!ctx || !primary) return set_error(PSACAK_EINVAL, "null context or primary-index pointer");
    if (n >= 0xFFFFFFFFull) return set_error(PSACAK_EINVAL, "n = %llu is not below 2^32 - 1", (unsigned long long)n);
    if (n > 0 && (!d_text || !d_sa || !d_bwt)) return set_error(PSACAK_EINVAL, "null text, suffix-array or BWT pointer");
    std::lock_guard<std::mutex> g(ctx->c.mu);
    Ctx &c = ctx->c;
    PSK_CUDA(cudaSetDevice(c.dev.id));
    c.stream = stream ? (cudaStream_t)stream : c.own_stream;
    *primary = 0;
    if (n == 0) return PSACAK_OK;
    cudaStream_t s = c.stream;
    uint32_t *d_row = c.d_scalars + 41;
    PSK_CUDA(cudaMemsetAsync(d_row, 0xFF, sizeof(uint32_t), s));
    PSK_PROF_LAUNCH(s, "bwt_primary", n, 4ull * n, (k_find_primary<<<grid_for_n(n), 256, 0, s>>>(d_sa, n, d_row)));
    uint32_t zrow = 0;
    PSK_TRY(c.read_u32(d_row, &zrow));
    if (zrow >= n) return set_error(PSACAK_EINVAL, "the suffix array has no entry 0");
    PSK_PROF_LAUNCH(s, "bwt", n, 6ull * n, (k_bwt<<<grid_for_n(n), 256, 0, s>>>(d_text, d_sa, n, zrow, d_bwt, c.d_err)));
    PSK_LAUNCH_CHECK();
    PSK_TRY(c.sync());
    *primary = (uint64_t)zrow + 1;
    return c.check_device_error();
}

int psacak_lcp8_dev(psacak_ctx *ctx, const uint8_t *d_text, uint64_t n, const uint32_t *d_sa, uint32_t *d_lcp,
                    void *stream) {
    return lcp_dev<uint8_t>(ctx, d_text, n, d_sa, d_lcp, stream);
}

int psacak_lcp32_dev(psacak_ctx *ctx, const uint32_t *d_text, uint64_t n, const uint32_t *d_sa, uint32_t *d_lcp,
                     void *stream) {
    return lcp_dev<uint32_t>(ctx, d_text, n, d_sa, d_lcp, stream);
}

}  // extern "C"
