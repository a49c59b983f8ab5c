// level.cuh -- per-level kernels shared by every recursion level: L/S typing,
// LMS bitmaps, naming of sorted LMS substrings, translation of names into
// bucket pointers, permutation of the reduced suffix array, tiny levels.
#pragma once

#include "lbscan.cuh"

namespace psk {

// Positions per typing tile: 256 words of 32 positions.
constexpr int TYPE_BLOCK = 256;
constexpr uint64_t TYPE_TILE = 32ull * TYPE_BLOCK;

struct Workspace;  // fwd

// What a single-pass scan needs: its flag/value scratch, the tickets and
// launch epoch it shares with the onesweep kernels, and the error word.
struct ScanEnv {
    ScanScratch *ss;
    OnesweepScratch *os;
    uint32_t *err;
};

// Histograms of a byte level: per character its count, its L-type count and
// its LMS count (the reference's Buckets::new, src/psacak8.rs:355-374).
struct ByteHist {
    uint32_t count[256];
    uint32_t lcount[256];
    uint32_t lmscount[256];
};

// L/S typing of `text` into packed bitmaps: bit i of `types` is 1 iff
// position i is S-type; bit i of `lms` is 1 iff position i is LMS.  Also
// writes per-word LMS popcounts into `lms_wcnt` (nwords entries) and, for
// bytes, accumulates `hist`.  `scratch` holds >= 2 * ntiles uint32.
template <class C>
status_t type_text(const C *text, uint64_t n, uint32_t *types, uint32_t *lms, uint32_t *lms_wcnt,
                   ByteHist *hist, uint32_t *scratch, const ScanEnv &env, uint32_t max_ctas, cudaStream_t s);

// Exclusive prefix of LMS popcounts: pref[w] = LMS positions before word w;
// pref[nwords] = total, also copied to *total (device).
status_t lms_prefix(const uint32_t *lms_wcnt, uint64_t nwords, uint32_t *pref, uint32_t *total,
                    const ScanEnv &env, cudaStream_t s);

// Names the n1 sorted LMS substrings `sorted` (positions in `text`) and
// builds the reduced string: red[rank(p)] = name.  `flags` is scratch of n1
// words, `lmsx` of ceil(n / 32) 64-bit words.  heads[c] = index in `sorted`
// where name c starts (k entries, then n1).  *k_out (device) = number of
// names.
template <class C>
status_t name_lms(const C *text, uint64_t n, const uint32_t *lms, const uint32_t *lms_pref,
                  const uint32_t *sorted, uint64_t n1, uint32_t *red, uint32_t *heads, uint32_t *flags,
                  uint64_t *lmsx, uint32_t *k_out, const ScanEnv &env, uint32_t max_ctas, cudaStream_t s);

// Translates names in `red` (types in `types`) into bucket pointers in place:
// L -> heads[c], S -> heads[c+1] - 1 (the reference's translate,
// src/naming.rs:263-274).  heads has k+1 entries (heads[k] = n1).
status_t translate_names(uint32_t *red, uint64_t n1, const uint32_t *types, const uint32_t *heads,
                         uint32_t *err, cudaStream_t s);

// Predecessor window of a byte-level SA entry x > 0, kept beside the entry
// by the bucket scans: byte 0 = text[x-1] (the character that decides
// whether x induces x-1 and into which bucket), bytes 1 and 2 = text[x-2]
// and text[x-3], bits 24..25 = how many of those two look-ahead bytes are
// valid.  The window of x-1 is this one shifted by a byte while a
// look-ahead byte is left, so only every third step of an induction chain
// reads the text (three adjacent bytes, one sector).  Bytes of positions
// below 0 are 0 and never used: entry 0 induces nothing.
constexpr uint32_t WIN_FULL = 2u << 24;
__device__ __forceinline__ uint32_t win_fill(const uint8_t *text, uint32_t x) {
    const uint32_t a = text[x - 1];
    const uint32_t b = x >= 2 ? text[x - 2] : 0u;
    const uint32_t c = x >= 3 ? text[x - 3] : 0u;
    return a | b << 8 | c << 16 | WIN_FULL;
}
// Window of x - 1 from the window w of x (x >= 1).
__device__ __forceinline__ uint32_t win_next(uint32_t w, const uint8_t *text, uint32_t x) {
    const uint32_t k = w >> 24;
    if (k) return ((w >> 8) & 0xFFFFu) | ((k - 1) << 24);
    return x >= 2 ? win_fill(text, x - 1) : 0u;
}
// Window of the suffix d characters into a run (1 <= d <= r) in front of a
// suffix x: text[x-1 .. x-r] are c and text[x-r-1] is e.
__device__ __forceinline__ uint32_t run_win(uint32_t d, uint32_t r, uint32_t c, uint32_t e) {
    const uint32_t left = r - d;
    const uint32_t b0 = left > 0 ? c : e, b1 = left > 1 ? c : e, b2 = left > 2 ? c : e;
    return b0 | b1 << 8 | b2 << 16 | (left < 2 ? left : 2u) << 24;
}

// Byte levels: out[i] = P[sa1[i]] | win_fill(text, P[sa1[i]]) << 32, the
// permuted LMS positions with their predecessor windows.  `plist` is
// scratch of n1 entries.
status_t permute_lms8(const uint32_t *sa1, uint64_t n1, const uint8_t *text, const uint32_t *lms,
                      const uint32_t *lms_pref, uint64_t n, uint64_t *plist, uint64_t *out, uint32_t *err,
                      cudaStream_t s);

// Any level: out[i] = P[sa1[i]] | text[P[sa1[i]]] << 32 where P lists the
// LMS positions of `lms` in text order (the reference's
// permutate_lmssuffixes, src/naming.rs:413-430), with the positions'
// symbols.  `plist` is scratch of n1 entries.
template <class C>
status_t permute_lms_sym(const uint32_t *sa1, uint64_t n1, const C *text, const uint32_t *lms, const uint32_t *lms_pref,
                         uint64_t n, uint64_t *plist, uint64_t *out, uint32_t *err, cudaStream_t s);

// Direct inverse when all names are unique: sa1[red[i]] = i.
status_t direct_inverse(const uint32_t *red, uint64_t n1, uint32_t *sa1, uint32_t *err, cudaStream_t s);

// SA of a text of length <= 3 (saca_tiny for the reference's small cases).
template <class C>
status_t tiny_sa(const C *text, uint64_t n, uint32_t *sa, cudaStream_t s);

// Burkhardt-Kaerkkaeinen check; *bad (device) receives 0 iff correct.
template <class C>
status_t check_sa(const C *text, uint64_t n, const uint32_t *sa, uint32_t *isa, uint32_t *bad,
                  cudaStream_t s);

}  // namespace psk
