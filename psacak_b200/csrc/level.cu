// level.cu -- per-level kernels (typing, naming, translation, permutation).
#include "level.cuh"

namespace psk {

// ---------------------------------------------------------------------------
// L/S typing (the reference's foreach_typedchars, src/common.rs:43-68).
//
// Position i is S iff text[i] < text[i+1], L iff text[i] > text[i+1], and
// takes the type of i+1 when the two are equal; n-1 is L.  So the type of i
// is the type of the first "change point" q >= i (q = n-1 or text[q] !=
// text[q+1]).  Each warp builds 32-position words with ballots, a block-wide
// max-scan finds for every word the nearest change point to its right inside
// the 8192-position tile, and a per-tile carry (computed by a chunked
// max-scan over tiles) covers equal runs that cross tiles.
// ---------------------------------------------------------------------------

// Code of the first change point of each tile: 0 none, 1 L, 2 S.
template <class C>
__global__ void __launch_bounds__(TYPE_BLOCK) k_tile_first(const C *__restrict__ text, uint64_t n,
                                                           uint64_t ntiles, uint32_t *code_out) {
    __shared__ unsigned long long s_first;
    for (uint64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        uint64_t start = tile * TYPE_TILE;
        uint64_t end = start + TYPE_TILE < n ? start + TYPE_TILE : n;
        if (threadIdx.x == 0) s_first = ~0ull;
        __syncthreads();
        uint32_t code = 0;
        for (uint64_t base = start; base < end; base += TYPE_BLOCK) {
            uint64_t p = base + threadIdx.x;
            bool c = p < end && (p == n - 1 || text[p] != text[p + 1]);
            if (c) atomicMin(&s_first, (unsigned long long)p);
            if (__syncthreads_or(c)) {
                uint64_t q = s_first;
                uint32_t t = (q == n - 1) ? 0u : (text[q] < text[q + 1] ? 1u : 0u);
                code = 1 + t;
                break;
            }
        }
        if (threadIdx.x == 0) code_out[tile] = code;
        __syncthreads();
    }
}

struct TileCarryLoad {
    const uint32_t *code;
    uint64_t T;
    __device__ __forceinline__ uint32_t operator()(uint64_t r) const {
        uint32_t c = code[T - 1 - r];
        return c ? (uint32_t)(((r + 1) << 1) | (c - 1)) : 0u;
    }
};
struct TileCarryStore {
    uint32_t *carry;
    uint64_t T;
    __device__ __forceinline__ void operator()(uint64_t r, uint32_t excl, uint32_t) const {
        carry[T - 1 - r] = excl ? (excl & 1u) : 0u;
    }
};

template <class C, bool HIST>
__global__ void __launch_bounds__(TYPE_BLOCK) k_type_main(const C *__restrict__ text, uint64_t n, uint64_t ntiles,
                                                          const uint32_t *__restrict__ tile_carry,
                                                          uint32_t *__restrict__ types, uint32_t *__restrict__ lms,
                                                          uint32_t *__restrict__ lms_wcnt, ByteHist *ghist) {
    __shared__ uint32_t s_scan[33];
    __shared__ uint32_t s_hi[TYPE_BLOCK];
    __shared__ uint32_t s_hist[HIST ? (TYPE_BLOCK / 32) * 3 * 256 : 1];
    const int w = threadIdx.x >> 5;
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t nwords = ceil_div(n, 32);
    if (HIST)
        for (int i = threadIdx.x; i < (TYPE_BLOCK / 32) * 3 * 256; i += TYPE_BLOCK) s_hist[i] = 0;

    for (uint64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const uint64_t tstart = tile * TYPE_TILE;
        uint32_t myC = 0, myD = 0;
        uint32_t pk[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
        for (int it = 0; it < 32; it++) {
            uint64_t p = tstart + (uint64_t)(w * 32 + it) * 32 + lane;
            bool valid = p < n;
            C a = valid ? text[p] : C(0);
            C b = (p + 1 < n) ? text[p + 1] : C(0);
            bool last = (p == n - 1);
            bool c = valid && (last || a != b);
            bool sd = valid && !last && a < b;
            uint32_t cw = __ballot_sync(FULL_MASK, c);
            uint32_t dw = __ballot_sync(FULL_MASK, sd);
            if ((int)lane == it) {
                myC = cw;
                myD = dw;
            }
            if (HIST) pk[it >> 2] |= ((uint32_t)(uint8_t)a) << ((it & 3) * 8);
        }
        // Nearest change point to the right of this word within the tile: an
        // exclusive max-scan run in reversed word order (scan slot u holds
        // word 255-u), each value tagged with its slot so the max picks the
        // nearest word.
        const uint32_t u = TYPE_BLOCK - 1 - threadIdx.x;
        uint32_t enc = 0;
        if (myC) {
            int lb = __ffs(myC) - 1;
            enc = ((u + 1) << 1) | ((myD >> lb) & 1u);
        }
        s_hi[u] = enc;
        __syncthreads();
        uint32_t rv = s_hi[threadIdx.x];
        uint32_t rex;
        block_scan<uint32_t, OpMax<uint32_t>, TYPE_BLOCK>(rv, OpMax<uint32_t>(), s_scan, &rex, (uint32_t *)nullptr);
        s_hi[TYPE_BLOCK - 1 - threadIdx.x] = rex;
        __syncthreads();
        uint32_t excl = s_hi[threadIdx.x];
        __syncthreads();
        uint32_t cur = excl ? (excl & 1u) : tile_carry[tile];
        uint32_t T = 0;
#pragma unroll
        for (int k = 31; k >= 0; k--) {
            if ((myC >> k) & 1u) cur = (myD >> k) & 1u;
            T |= cur << k;
        }
        const uint64_t wg = tile * TYPE_BLOCK + threadIdx.x;
        const uint64_t p0 = wg * 32;
        uint32_t vmask = 0;
        if (p0 < n) vmask = (n - p0 >= 32) ? FULL_MASK : (uint32_t)((1ull << (n - p0)) - 1);
        T &= vmask;
        s_hi[threadIdx.x] = T >> 31;
        __syncthreads();
        uint32_t prevS;
        if (threadIdx.x > 0) {
            prevS = s_hi[threadIdx.x - 1];
        } else if (p0 == 0 || p0 >= n) {
            prevS = 1;  // position 0 is never LMS
        } else {
            C x = text[p0 - 1], y = text[p0];
            prevS = (x != y) ? (x < y ? 1u : 0u) : (T & 1u);
        }
        uint32_t Lm = T & ~((T << 1) | prevS) & vmask;
        if (wg < nwords) {
            types[wg] = T;
            lms[wg] = Lm;
            lms_wcnt[wg] = __popc(Lm);
        }
        if (HIST) {
            // per-warp private histograms: lanes add their own position
            // (conflicts only among the lanes of one warp)
            uint32_t *wh = s_hist + w * 3 * 256;
#pragma unroll
            for (int it = 0; it < 32; it++) {
                const uint32_t Tw = __shfl_sync(FULL_MASK, T, it);
                const uint32_t Lw = __shfl_sync(FULL_MASK, Lm, it);
                const uint64_t p = tstart + (uint64_t)(w * 32 + it) * 32 + lane;
                if (p < n) {
                    const uint32_t a = (pk[it >> 2] >> ((it & 3) * 8)) & 0xFFu;
                    atomicAdd(&wh[a], 1u);
                    if (!((Tw >> lane) & 1u)) atomicAdd(&wh[256 + a], 1u);
                    if ((Lw >> lane) & 1u) atomicAdd(&wh[512 + a], 1u);
                }
            }
        }
        __syncthreads();
    }
    if (HIST) {
        __syncthreads();
        for (int i = threadIdx.x; i < 256; i += TYPE_BLOCK) {
            uint32_t a = 0, b = 0, m = 0;
            for (int ww = 0; ww < TYPE_BLOCK / 32; ww++) {
                a += s_hist[ww * 768 + i];
                b += s_hist[ww * 768 + 256 + i];
                m += s_hist[ww * 768 + 512 + i];
            }
            if (a) atomicAdd(&ghist->count[i], a);
            if (b) atomicAdd(&ghist->lcount[i], b);
            if (m) atomicAdd(&ghist->lmscount[i], m);
        }
    }
}

template <class C>
status_t type_text(const C *text, uint64_t n, uint32_t *types, uint32_t *lms, uint32_t *lms_wcnt,
                   ByteHist *hist, uint32_t *scratch, const ScanEnv &env, uint32_t max_ctas, cudaStream_t s) {
    if (n == 0) return PSACAK_OK;
    uint64_t ntiles = ceil_div(n, TYPE_TILE);
    uint32_t *code = scratch;
    uint32_t *carry = scratch + ntiles;
    uint32_t grid = (uint32_t)(ntiles < max_ctas ? ntiles : max_ctas);
    PSK_PROF_LAUNCH(s, "type_tile_first", ntiles, 0, (k_tile_first<C><<<grid, TYPE_BLOCK, 0, s>>>(text, n, ntiles, code)));
    PSK_TRY((lb_scan<uint32_t, OpMax<uint32_t>>(TileCarryLoad{code, ntiles}, TileCarryStore{carry, ntiles}, ntiles,
                                                (uint32_t *)nullptr, OpMax<uint32_t>(), *env.ss, *env.os, env.err, s,
                                                "scan_tile_carry")));
    // algorithmic bytes: the text once, two bitmaps and the word counts
    const uint64_t tbytes = n * sizeof(C) + 3 * ceil_div(n, 32) * 4;
    if (hist) {
        PSK_CUDA(cudaMemsetAsync(hist, 0, sizeof(ByteHist), s));
        PSK_PROF_LAUNCH(s, "type_main", n, tbytes,
                        (k_type_main<C, true><<<grid, TYPE_BLOCK, 0, s>>>(text, n, ntiles, carry, types, lms, lms_wcnt,
                                                                         hist)));
    } else {
        PSK_PROF_LAUNCH(s, "type_main", n, tbytes,
                        (k_type_main<C, false><<<grid, TYPE_BLOCK, 0, s>>>(text, n, ntiles, carry, types, lms,
                                                                          lms_wcnt, nullptr)));
    }
    PSK_LAUNCH_CHECK();
    return PSACAK_OK;
}

template status_t type_text<uint8_t>(const uint8_t *, uint64_t, uint32_t *, uint32_t *, uint32_t *, ByteHist *,
                                     uint32_t *, const ScanEnv &, uint32_t, cudaStream_t);
template status_t type_text<uint32_t>(const uint32_t *, uint64_t, uint32_t *, uint32_t *, uint32_t *, ByteHist *,
                                      uint32_t *, const ScanEnv &, uint32_t, cudaStream_t);

struct PrefLoad {
    const uint32_t *w;
    __device__ __forceinline__ uint32_t operator()(uint64_t i) const { return w[i]; }
};
struct PrefStore {
    uint32_t *pref;
    __device__ __forceinline__ void operator()(uint64_t i, uint32_t excl, uint32_t) const { pref[i] = excl; }
};

__global__ void k_copy_total(const uint32_t *total, uint32_t *dst) { *dst = *total; }

status_t lms_prefix(const uint32_t *lms_wcnt, uint64_t nwords, uint32_t *pref, uint32_t *total,
                    const ScanEnv &env, cudaStream_t s) {
    PSK_TRY((lb_scan<uint32_t, OpSum<uint32_t>>(PrefLoad{lms_wcnt}, PrefStore{pref}, nwords, total, OpSum<uint32_t>(),
                                                *env.ss, *env.os, env.err, s, "scan_lms_prefix")));
    k_copy_total<<<1, 1, 0, s>>>(total, pref + nwords);
    PSK_KCOUNT();
    PSK_LAUNCH_CHECK();
    return PSACAK_OK;
}

// ---------------------------------------------------------------------------
// Naming (the reference's name_lmssubstrings, src/naming.rs:20-93, with the
// equality of UintFingerprint::equals, src/naming.rs:388-408): two LMS
// substrings are equal iff they have the same length up to and including the
// next LMS position and the same characters; a substring that reaches the
// end of the text contains the sentinel and equals nothing else.
// ---------------------------------------------------------------------------
// lmsx[w] = lms[w] | pref[w] << 32: a word of the LMS bitmap beside the
// number of LMS positions before it, so that one 8-byte read gives both the
// next LMS position after p and the rank of p.
__global__ void k_lms_pack(const uint32_t *__restrict__ lms, const uint32_t *__restrict__ pref, uint64_t nwords,
                           uint64_t *lmsx) {
    for (uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; w < nwords; w += (uint64_t)gridDim.x * blockDim.x)
        lmsx[w] = lms[w] | (uint64_t)pref[w] << 32;
}

// First LMS position after p (n if none); x0 = lmsx[p >> 5].
__device__ __forceinline__ uint64_t next_lms(const uint64_t *lmsx, uint64_t n, uint64_t p, uint64_t x0) {
    uint64_t w = p >> 5;
    uint32_t sh = (uint32_t)(p & 31);
    uint32_t word = sh == 31 ? 0u : ((uint32_t)x0 & (FULL_MASK << (sh + 1)));
    const uint64_t nwords = ceil_div(n, 32);
    while (!word) {
        w++;
        if (w >= nwords) return n;
        word = (uint32_t)lmsx[w];
    }
    return (w << 5) + (uint64_t)(__ffs(word) - 1);
}

// Fingerprint of the LMS substring at p: its length up to the next LMS
// position (or "reaches the end", which equals nothing) and its first 16
// bytes packed, zero-padded -- the GPU form of UintFingerprint::get
// (src/naming.rs:339-385).  Equal fingerprints decide equality outright
// when the substring fits in them; longer ones compare their remaining
// characters.
template <class C> struct LmsFp {
    static constexpr uint32_t W = 16 / sizeof(C);  // characters held
    static constexpr uint32_t END = 0xFFFFFFFFu;
    uint32_t len;   // next LMS - p, or END
    uint32_t w[4];  // first min(len + 1, W) characters
};
template <class C>
__device__ __forceinline__ LmsFp<C> lms_fp(const C *text, uint64_t n, const uint64_t *lmsx, uint64_t p, uint64_t x0) {
    LmsFp<C> f;
    const uint64_t e = next_lms(lmsx, n, p, x0);
    f.len = e >= n ? LmsFp<C>::END : (uint32_t)(e - p);
#pragma unroll
    for (int i = 0; i < 4; i++) f.w[i] = 0;
    const uint32_t take = f.len == LmsFp<C>::END ? 0u : (f.len + 1 < LmsFp<C>::W ? f.len + 1 : LmsFp<C>::W);
    for (uint32_t k = 0; k < take; k++) {
        const uint32_t c = (uint32_t)text[p + k];
        if (sizeof(C) == 1) f.w[k >> 2] |= c << ((k & 3) * 8);
        else f.w[k] = c;
    }
    return f;
}
template <class C>
__device__ __forceinline__ bool lms_fp_equal(const C *text, const LmsFp<C> &fa, uint64_t a, const LmsFp<C> &fb,
                                             uint64_t b) {
    if (fa.len == LmsFp<C>::END || fa.len != fb.len) return false;
    if (fa.w[0] != fb.w[0] || fa.w[1] != fb.w[1] || fa.w[2] != fb.w[2] || fa.w[3] != fb.w[3]) return false;
    for (uint64_t k = LmsFp<C>::W; k <= fa.len; k++)
        if (text[a + k] != text[b + k]) return false;
    return true;
}

// flags[i] = (1 iff sorted LMS substring i differs from i - 1) << 31 | the
// text-order rank of its LMS position (< n1 <= 2^31).  Each thread
// fingerprints its own substring once and takes its neighbour's from the
// lane below (lane 0 fingerprints its neighbour itself).
template <class C>
__global__ void k_name_flags(const C *__restrict__ text, uint64_t n, const uint64_t *__restrict__ lmsx,
                             const uint32_t *__restrict__ sorted, uint64_t n1, uint32_t *flags) {
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;  // a multiple of 32
    for (uint64_t ib = (uint64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31u); ib < n1; ib += stride) {
        const uint64_t i = ib + lane;
        const bool valid = i < n1;
        const uint64_t p = valid ? sorted[i] : 0;
        const uint64_t x = valid ? lmsx[p >> 5] : 0ull;
        LmsFp<C> f;
        if (valid) f = lms_fp(text, n, lmsx, p, x);
        else f.len = LmsFp<C>::END;
        uint64_t q = __shfl_up_sync(FULL_MASK, p, 1);
        LmsFp<C> g;
        g.len = __shfl_up_sync(FULL_MASK, f.len, 1);
#pragma unroll
        for (int k = 0; k < 4; k++) g.w[k] = __shfl_up_sync(FULL_MASK, f.w[k], 1);
        if (valid) {
            uint32_t flag = 1;
            if (i > 0) {
                if (lane == 0) {
                    q = sorted[i - 1];
                    g = lms_fp(text, n, lmsx, q, lmsx[q >> 5]);
                }
                flag = lms_fp_equal(text, g, q, f, p) ? 0u : 1u;
            }
            const uint32_t rank = (uint32_t)(x >> 32) + __popc((uint32_t)x & (uint32_t)((1ull << (p & 31)) - 1));
            flags[i] = flag << 31 | rank;
        }
    }
}

// The load takes the flag and the text-order rank of the LMS position that
// k_name_flags packed together, so the scan reads one sequential word per
// item and the store only writes.
struct NameLoad {
    using Payload = uint32_t;  // rank of sorted[i] among the LMS positions
    static constexpr int kIPT = 8;
    const uint32_t *flags;
    __device__ __forceinline__ uint32_t operator()(uint64_t i, uint32_t &rank) const {
        const uint32_t v = flags[i];
        rank = v & 0x7FFFFFFFu;
        return v >> 31;
    }
};
struct NameStore {
    uint32_t *red;
    uint32_t *heads;
    uint64_t n1;
    __device__ __forceinline__ void operator()(uint64_t i, uint32_t excl, uint32_t v, uint32_t rank) const {
        uint32_t name = excl + v - 1;
        red[rank] = name;
        if (v) heads[name] = (uint32_t)i;
        if (i == n1 - 1) heads[name + 1] = (uint32_t)n1;
    }
};

template <class C>
status_t name_lms(const C *text, uint64_t n, const uint32_t *lms, const uint32_t *lms_pref,
                  const uint32_t *sorted, uint64_t n1, uint32_t *red, uint32_t *heads, uint32_t *flags,
                  uint64_t *lmsx, uint32_t *k_out, const ScanEnv &env, uint32_t max_ctas, cudaStream_t s) {
    if (n1 == 0) {
        PSK_CUDA(cudaMemsetAsync(k_out, 0, sizeof(uint32_t), s));
        return PSACAK_OK;
    }
    const uint64_t nwords = ceil_div(n, 32);
    const uint64_t gw = ceil_div(nwords, 256);
    PSK_PROF_LAUNCH(s, "name_flags", nwords, 16 * nwords,
                    (k_lms_pack<<<(uint32_t)(gw < 4096 ? gw : 4096), 256, 0, s>>>(lms, lms_pref, nwords, lmsx)));
    uint32_t grid = (uint32_t)(ceil_div(n1, 256) < (uint64_t)max_ctas * 4 ? ceil_div(n1, 256) : (uint64_t)max_ctas * 4);
    PSK_PROF_LAUNCH(s, "name_flags", n1, 0, (k_name_flags<C><<<grid, 256, 0, s>>>(text, n, lmsx, sorted, n1, flags)));
    PSK_LAUNCH_CHECK();
    return lb_scan<uint32_t, OpSum<uint32_t>>(NameLoad{flags}, NameStore{red, heads, n1}, n1, k_out,
                                              OpSum<uint32_t>(), *env.ss, *env.os, env.err, s, "scan_names");
}

template status_t name_lms<uint8_t>(const uint8_t *, uint64_t, const uint32_t *, const uint32_t *, const uint32_t *,
                                    uint64_t, uint32_t *, uint32_t *, uint32_t *, uint64_t *, uint32_t *,
                                    const ScanEnv &, uint32_t, cudaStream_t);
template status_t name_lms<uint32_t>(const uint32_t *, uint64_t, const uint32_t *, const uint32_t *,
                                     const uint32_t *, uint64_t, uint32_t *, uint32_t *, uint32_t *, uint64_t *,
                                     uint32_t *, const ScanEnv &, uint32_t, cudaStream_t);

__global__ void k_translate(uint32_t *red, uint64_t n1, const uint32_t *__restrict__ types,
                            const uint32_t *__restrict__ heads, uint32_t *err) {
    constexpr int U = 4;  // symbols per thread step: their gathers overlap
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t p0 = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; p0 < n1; p0 += stride * U) {
        uint32_t c[U], v[U];
#pragma unroll
        for (int u = 0; u < U; u++) c[u] = p0 + u * stride < n1 ? red[p0 + u * stride] : 0u;
#pragma unroll
        for (int u = 0; u < U; u++) {
            const uint64_t p = p0 + u * stride;
            v[u] = 0;
            if (p < n1 && c[u] < n1) v[u] = bm_get(types, p) ? heads[c[u] + 1] - 1 : heads[c[u]];
        }
#pragma unroll
        for (int u = 0; u < U; u++) {
            const uint64_t p = p0 + u * stride;
            if (p >= n1) continue;
            if (c[u] >= n1) dev_fail(err, DEVERR_RANGE);
            red[p] = v[u];
        }
    }
}

status_t translate_names(uint32_t *red, uint64_t n1, const uint32_t *types, const uint32_t *heads, uint32_t *err,
                         cudaStream_t s) {
    if (n1 == 0) return PSACAK_OK;
    uint64_t g = ceil_div(n1, 256);
    k_translate<<<(uint32_t)(g < 8192 ? g : 8192), 256, 0, s>>>(red, n1, types, heads, err);
    PSK_KCOUNT();
    PSK_LAUNCH_CHECK();
    return PSACAK_OK;
}

// Byte levels: the permuted list carries each LMS position's predecessor
// window, p | win_fill(text, p) << 32, so that the final placement needs no
// gather from the text.
__global__ void k_lms_list8(const uint8_t *__restrict__ text, const uint32_t *__restrict__ lms,
                            const uint32_t *__restrict__ pref, uint64_t nwords, uint64_t *plist) {
    for (uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; w < nwords; w += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t word = lms[w];
        uint32_t o = pref[w];
        while (word) {
            int b = __ffs(word) - 1;
            const uint64_t p = (w << 5) + b;  // LMS positions are > 0
            plist[o++] = p | (uint64_t)win_fill(text, (uint32_t)p) << 32;
            word &= word - 1;
        }
    }
}

// Any level, doubling engine: the permuted list carries each LMS position's
// symbol, p | text[p] << 32, so that the final placement (which compares the
// symbols of neighbouring list entries) reads the list in order only.
template <class C>
__global__ void k_lms_list_sym(const C *__restrict__ text, const uint32_t *__restrict__ lms,
                               const uint32_t *__restrict__ pref, uint64_t nwords, uint64_t *plist) {
    for (uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; w < nwords; w += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t word = lms[w];
        uint32_t o = pref[w];
        while (word) {
            int b = __ffs(word) - 1;
            const uint64_t p = (w << 5) + b;
            plist[o++] = p | (uint64_t)(uint32_t)text[p] << 32;
            word &= word - 1;
        }
    }
}

// out[i] = plist[sa1[i]] for 64-bit list entries.
__global__ void k_permute_pairs(const uint32_t *__restrict__ sa1, uint64_t n1, const uint64_t *__restrict__ plist,
                                uint64_t *out, uint32_t *err) {
    constexpr int U = 4;  // entries per thread step: their gathers overlap
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i0 = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i0 < n1; i0 += stride * U) {
        uint32_t r[U];
        uint64_t v[U];
#pragma unroll
        for (int u = 0; u < U; u++) r[u] = i0 + u * stride < n1 ? sa1[i0 + u * stride] : 0u;
#pragma unroll
        for (int u = 0; u < U; u++) v[u] = r[u] < n1 ? plist[r[u]] : 1ull;
#pragma unroll
        for (int u = 0; u < U; u++) {
            const uint64_t i = i0 + u * stride;
            if (i >= n1) continue;
            if (r[u] >= n1) dev_fail(err, DEVERR_RANGE);
            out[i] = v[u];
        }
    }
}

status_t permute_lms8(const uint32_t *sa1, uint64_t n1, const uint8_t *text, const uint32_t *lms,
                      const uint32_t *lms_pref, uint64_t n, uint64_t *plist, uint64_t *out, uint32_t *err,
                      cudaStream_t s) {
    if (n1 == 0) return PSACAK_OK;
    uint64_t nwords = ceil_div(n, 32);
    uint64_t g = ceil_div(nwords, 256);
    k_lms_list8<<<(uint32_t)(g < 8192 ? g : 8192), 256, 0, s>>>(text, lms, lms_pref, nwords, plist);
    PSK_KCOUNT();
    g = ceil_div(n1, 256);
    k_permute_pairs<<<(uint32_t)(g < 8192 ? g : 8192), 256, 0, s>>>(sa1, n1, plist, out, err);
    PSK_KCOUNT();
    PSK_LAUNCH_CHECK();
    return PSACAK_OK;
}

template <class C>
status_t permute_lms_sym(const uint32_t *sa1, uint64_t n1, const C *text, const uint32_t *lms, const uint32_t *lms_pref,
                         uint64_t n, uint64_t *plist, uint64_t *out, uint32_t *err, cudaStream_t s) {
    if (n1 == 0) return PSACAK_OK;
    uint64_t nwords = ceil_div(n, 32);
    uint64_t g = ceil_div(nwords, 256);
    k_lms_list_sym<C><<<(uint32_t)(g < 8192 ? g : 8192), 256, 0, s>>>(text, lms, lms_pref, nwords, plist);
    PSK_KCOUNT();
    g = ceil_div(n1, 256);
    k_permute_pairs<<<(uint32_t)(g < 8192 ? g : 8192), 256, 0, s>>>(sa1, n1, plist, out, err);
    PSK_KCOUNT();
    PSK_LAUNCH_CHECK();
    return PSACAK_OK;
}
template status_t permute_lms_sym<uint8_t>(const uint32_t *, uint64_t, const uint8_t *, const uint32_t *,
                                           const uint32_t *, uint64_t, uint64_t *, uint64_t *, uint32_t *, cudaStream_t);
template status_t permute_lms_sym<uint32_t>(const uint32_t *, uint64_t, const uint32_t *, const uint32_t *,
                                            const uint32_t *, uint64_t, uint64_t *, uint64_t *, uint32_t *,
                                            cudaStream_t);

__global__ void k_direct_inverse(const uint32_t *__restrict__ red, uint64_t n1, uint32_t *sa1, uint32_t *err) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n1; i += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t c = red[i];
        if (c < n1) sa1[c] = (uint32_t)i;
        else dev_fail(err, DEVERR_RANGE);
    }
}

status_t direct_inverse(const uint32_t *red, uint64_t n1, uint32_t *sa1, uint32_t *err, cudaStream_t s) {
    if (n1 == 0) return PSACAK_OK;
    uint64_t g = ceil_div(n1, 256);
    k_direct_inverse<<<(uint32_t)(g < 8192 ? g : 8192), 256, 0, s>>>(red, n1, sa1, err);
    PSK_KCOUNT();
    PSK_LAUNCH_CHECK();
    return PSACAK_OK;
}

// saca_tiny for n <= 3 (src/common.rs:13-25): insertion sort by suffix order.
template <class C>
__global__ void k_tiny_sa(const C *text, uint32_t n, uint32_t *sa) {
    if (threadIdx.x || blockIdx.x) return;
    uint32_t v[4];
    for (uint32_t i = 0; i < n; i++) v[i] = i;
    for (uint32_t i = 1; i < n; i++) {
        for (uint32_t j = i; j > 0; j--) {
            uint32_t a = v[j - 1], b = v[j];
            // is suffix b < suffix a ?
            uint32_t la = n - a, lb = n - b, k = 0;
            bool less = false;
            for (;; k++) {
                if (k == lb) { less = (lb < la); break; }
                if (k == la) { less = false; break; }
                if (text[b + k] != text[a + k]) { less = text[b + k] < text[a + k]; break; }
            }
            if (!less) break;
            v[j - 1] = b;
            v[j] = a;
        }
    }
    for (uint32_t i = 0; i < n; i++) sa[i] = v[i];
}

template <class C>
status_t tiny_sa(const C *text, uint64_t n, uint32_t *sa, cudaStream_t s) {
    if (n == 0) return PSACAK_OK;
    if (n > 4) return set_error(PSACAK_EINTERNAL, "tiny_sa called with n=%llu", (unsigned long long)n);
    k_tiny_sa<C><<<1, 32, 0, s>>>(text, (uint32_t)n, sa);
    PSK_KCOUNT();
    PSK_LAUNCH_CHECK();
    return PSACAK_OK;
}
template status_t tiny_sa<uint8_t>(const uint8_t *, uint64_t, uint32_t *, cudaStream_t);
template status_t tiny_sa<uint32_t>(const uint32_t *, uint64_t, uint32_t *, cudaStream_t);

// ---------------------------------------------------------------------------
// Burkhardt-Kaerkkaeinen suffix-array check.
// ---------------------------------------------------------------------------
__global__ void k_check_isa(const uint32_t *__restrict__ sa, uint64_t n, uint32_t *isa, uint32_t *bad) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t x = sa[i];
        if (x >= n) {
            atomicOr(bad, 1u);
            continue;
        }
        uint32_t old = atomicExch(&isa[x], (uint32_t)i);
        if (old != 0xFFFFFFFFu) atomicOr(bad, 2u);
    }
}

template <class C>
__global__ void k_check_order(const C *__restrict__ text, uint64_t n, const uint32_t *__restrict__ sa,
                              const uint32_t *__restrict__ isa, uint32_t *bad) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x + 1; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t a = sa[i - 1], b = sa[i];
        if (a >= n || b >= n) continue;
        C ca = text[a], cb = text[b];
        if (ca > cb) {
            atomicOr(bad, 4u);
        } else if (ca == cb) {
            int64_t ra = (a + 1 < n) ? (int64_t)isa[a + 1] : -1;
            int64_t rb = (b + 1 < n) ? (int64_t)isa[b + 1] : -1;
            if (ra >= rb) atomicOr(bad, 8u);
        }
    }
}

template <class C>
status_t check_sa(const C *text, uint64_t n, const uint32_t *sa, uint32_t *isa, uint32_t *bad, cudaStream_t s) {
    PSK_CUDA(cudaMemsetAsync(bad, 0, sizeof(uint32_t), s));
    if (n == 0) return PSACAK_OK;
    PSK_CUDA(cudaMemsetAsync(isa, 0xFF, n * sizeof(uint32_t), s));
    uint64_t g = ceil_div(n, 256);
    uint32_t grid = (uint32_t)(g < 16384 ? g : 16384);
    k_check_isa<<<grid, 256, 0, s>>>(sa, n, isa, bad);
    PSK_KCOUNT();
    k_check_order<C><<<grid, 256, 0, s>>>(text, n, sa, isa, bad);
    PSK_KCOUNT();
    PSK_LAUNCH_CHECK();
    return PSACAK_OK;
}
template status_t check_sa<uint8_t>(const uint8_t *, uint64_t, const uint32_t *, uint32_t *, uint32_t *, cudaStream_t);
template status_t check_sa<uint32_t>(const uint32_t *, uint64_t, const uint32_t *, uint32_t *, uint32_t *,
                                     cudaStream_t);

}  // namespace psk
