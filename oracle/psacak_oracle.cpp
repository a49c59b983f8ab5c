/*
 * psacak_oracle.cpp -- CPU restatement of hucsmn/psacak's serial pSACAK.
 *
 * TEST INFRASTRUCTURE ONLY (see psacak_oracle.h).  It is the checker the GPU
 * builder is compared against, never part of the product path.
 *
 * The restatement follows the reference crate's serial code paths, written
 * here as C++ templates over the character type (uint8_t or uint32_t) and
 * a uint32_t index type, which is the only pair the reference instantiates
 * on its public path.  Every function names the reference item (path:line
 * inside the crate) whose behaviour it reproduces.  The reference's
 * parallel/pipelined variants produce identical results by the reference's
 * own property tests, so the serial path is the one restated.
 *
 * Parity is pinned by: the reference's golden vectors (src/lib.rs:12-15,
 * :37-42; src/psacak8.rs:508-524; src/psacak32.rs:826-842), agreement with
 * saca_tiny on random texts (src/psacak8.rs:531-534, src/psacak32.rs:849-852)
 * and the O(n) Burkhardt-Kaerkkaeinen check; all live in tests/.
 */
#include "psacak_oracle.h"

#include <algorithm>
#include <cstring>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <functional>
#include <map>
#include <vector>

/* The pipelined scans of the reference's par_induce_sort (psacak_oracle_par.cpp). */
namespace oracle_par {
void induce_sort32_par(const uint32_t *text, uint32_t *suf, size_t len, bool left_most, unsigned threads);
size_t name_chunks_par(uint32_t *lmssubs, size_t n, uint32_t *work, size_t wlen, unsigned threads,
                       const std::function<bool(size_t, size_t)> &differs);
void induce_sort8_par(const uint8_t *text, size_t len, uint32_t *suf, uint32_t *ptrs_head, uint32_t *ptrs_tail,
                      bool left_most, unsigned threads);
}

namespace {

typedef unsigned __int128 u128;

template <class C> struct Chr;
template <> struct Chr<uint8_t> {
    static constexpr uint32_t MAXV = 0xFFu;
    static constexpr int BITS = 8;
};
template <> struct Chr<uint32_t> {
    static constexpr uint32_t MAXV = 0xFFFFFFFFu;
    static constexpr int BITS = 32;
};

/* src/psacak32.rs:12 -- empty symbol of the inner-level workspace. */
constexpr uint32_t EMPTY = 1u << 31;

/* src/psacak32.rs:486-496 -- two's-complement bucket counters in u32. */
inline size_t decode_counter(uint32_t x) { return (uint32_t)(-(int32_t)x); }
inline uint32_t encode_counter(size_t n) { return (uint32_t)(-(int32_t)(uint32_t)n); }

uint64_t mix64(uint64_t z) {
    z += 0x9e3779b97f4a7c15ull;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

struct Trace {
    oracle_level *out;
    uint32_t cap;
    uint32_t count;
    uint32_t *reduced_out;   /* level-0 reduced string capture (nullable) */
    uint64_t reduced_cap;
    uint64_t reduced_len;
    uint64_t reduced_k;
    bool stop_after_level0;  /* only compute the level-0 reduction */
};

void trace_push(Trace *tr, uint32_t level, uint32_t width, uint64_t m,
                uint64_t n_lms, uint64_t k, uint64_t hash) {
    if (!tr) return;
    if (tr->out && tr->count < tr->cap) {
        oracle_level &l = tr->out[tr->count];
        l.level = level; l.width = width; l.m = m; l.n_lms = n_lms;
        l.k = k; l.hash = hash;
    }
    tr->count++;
}

/* src/common.rs:13-25 saca_tiny: sort suffix indices by slice order
 * (a proper prefix sorts first, i.e. the shorter suffix wins ties). */
template <class C>
void saca_tiny(const C *text, size_t n, uint32_t *suf) {
    for (size_t i = 0; i < n; i++) suf[i] = (uint32_t)i;
    std::sort(suf, suf + n, [&](uint32_t a, uint32_t b) {
        return std::lexicographical_compare(text + a, text + n, text + b, text + n);
    });
}

struct TypedChar {
    bool stype;
    bool left_most;
    bool is_lms() const { return stype && left_most; }
};

/* src/common.rs:43-68 foreach_typedchars: right-to-left L/S typing with the
 * equal-character carry; position n-1 is L (compared to the sentinel). */
template <class C, class F>
void foreach_typedchars(const C *text, size_t n, F f) {
    if (n == 0) return;
    bool stype = false;
    for (size_t i = n - 1; i >= 1; --i) {
        bool next_stype = text[i - 1] < text[i] || (text[i - 1] == text[i] && stype);
        f(i, TypedChar{stype, stype != next_stype}, text[i]);
        stype = next_stype;
    }
    f(0, TypedChar{stype, false}, text[0]);
}

/* src/common.rs:72-97 foreach_typedchars_mut: same walk, the callback may
 * rewrite text[i] after its type (and text[i-1]'s) has been derived. */
template <class C, class F>
void foreach_typedchars_mut(C *text, size_t n, F f) {
    if (n == 0) return;
    bool stype = false;
    for (size_t i = n - 1; i >= 1; --i) {
        bool next_stype = text[i - 1] < text[i] || (text[i - 1] == text[i] && stype);
        f(i, TypedChar{stype, stype != next_stype}, text[i]);
        stype = next_stype;
    }
    f(0, TypedChar{stype, false}, text[0]);
}

/* src/common.rs:101-117 foreach_lmschars: LMS positions, decreasing. */
template <class C, class F>
void foreach_lmschars(const C *text, size_t n, F f) {
    if (n < 3) return;
    bool stype = false;
    for (size_t i = n - 2; i >= 1; --i) {
        stype = text[i] < text[i + 1] || (text[i] == text[i + 1] && stype);
        if (stype && text[i - 1] > text[i]) f(i, text[i]);
    }
}

/* src/common.rs:123-134 compact_left. */
size_t compact_left(uint32_t *d, size_t len, uint32_t except) {
    size_t n = 0;
    for (size_t i = 0; i < len; i++) {
        uint32_t x = d[i];
        if (x != except) d[n++] = x;
    }
    return n;
}

/* src/common.rs:139-150 compact_right. */
size_t compact_right(uint32_t *d, size_t len, uint32_t except) {
    size_t p = len;
    for (size_t i = len; i-- > 0;) {
        uint32_t x = d[i];
        if (x != except) d[--p] = x;
    }
    return len - p;
}

/* src/common.rs:155-170 compact_left_range over [lo, hi]. */
size_t compact_left_range(uint32_t *d, size_t len, uint32_t lo, uint32_t hi) {
    size_t n = 0;
    for (size_t i = 0; i < len; i++) {
        uint32_t x = d[i];
        if (x >= lo && x <= hi) d[n++] = x;
    }
    return n;
}

inline void reset_slice(uint32_t *d, size_t len, uint32_t v) {
    for (size_t i = 0; i < len; i++) d[i] = v;
}

/* ---------------------------------------------------------------------- */
/* Naming (src/naming.rs)                                                 */
/* ---------------------------------------------------------------------- */

template <class C> struct Fingerprint {
    size_t len;
    u128 fp;
    bool operator==(const Fingerprint &o) const { return len == o.len && fp == o.fp; }
};

/* src/naming.rs:339-385 UintFingerprint<u128>::get: LMS-substring length
 * (sentinel included, redundant trailing equal S-characters excluded) and the
 * first 16/width characters packed in a u128. */
template <class C>
Fingerprint<C> fp_get(const C *text, size_t n, size_t i) {
    const size_t W = 16 / sizeof(C);
    const int B = Chr<C>::BITS;
    if (i == n) return Fingerprint<C>{1, (u128)Chr<C>::MAXV};
    size_t k = 1;
    u128 fp = (u128)text[i];
    while (i + k < n && text[i + k] >= text[i + k - 1]) {
        if (k < W) { fp <<= B; fp |= (u128)text[i + k]; }
        k++;
    }
    while (i + k < n && text[i + k] <= text[i + k - 1]) {
        if (k < W) { fp <<= B; fp |= (u128)text[i + k]; }
        k++;
    }
    if (i + k == n) {
        k++;
        if (k < W) { fp <<= B; fp |= (u128)Chr<C>::MAXV; }
    } else {
        while (k > 0 && text[i + k - 1] == text[i + k - 2]) {
            k--;
            if (k < W) fp >>= B;
        }
    }
    return Fingerprint<C>{k, fp};
}

/* src/naming.rs:388-408 UintFingerprint<u128>::equals. */
template <class C>
bool fp_equals(const C *text, size_t n, size_t i, Fingerprint<C> fi, size_t j,
               Fingerprint<C> fj) {
    const size_t W = 16 / sizeof(C);
    if (i == j) return true;
    size_t p = i + fi.len, q = j + fj.len;
    if (!(fi == fj) || p > n || q > n) return false;
    if (fi.len <= W) return true;
    i += W;
    j += W;
    return std::equal(text + i, text + p, text + j, text + q);
}

/* src/naming.rs:263-274 translate: names -> bucket pointers (L-type ->
 * bucket head, S-type -> bucket tail - 1). */
void translate(uint32_t *t, size_t n, const uint32_t *tails) {
    foreach_typedchars_mut(t, n, [&](size_t, TypedChar ty, uint32_t &p) {
        size_t c = p;
        if (!ty.stype) p = (c == 0) ? 0 : tails[c - 1];
        else p = tails[c] - 1;
    });
}

/* src/naming.rs:51-93 nonpar_name_lmssubstrings_using with the default
 * UintFingerprint<u128> (src/naming.rs:16): names the n sorted LMS substrings
 * in suf[..n], leaves the translated reduced string in the tail of suf and
 * the bucket tails in suf[..k]; returns k. */
template <class C>
size_t name_lmssubstrings(const C *text, size_t len, uint32_t *suf, size_t n, unsigned threads = 0) {
    if (n == 0) return 0;
    uint32_t *lmssubs = suf;
    uint32_t *work = suf + n;
    size_t wlen = len - n;
    if (threads > 1 && n >= (1u << 16)) {
        /* src/naming.rs:169-259 fastpar naming: flags and names by chunks in
         * parallel (psacak_oracle_par.cpp), bucket tails serially */
        oracle_par::name_chunks_par(lmssubs, n, work, wlen, threads, [&](size_t i0, size_t i1) {
            return !fp_equals(text, len, i0, fp_get(text, len, i0), i1, fp_get(text, len, i1));
        });
        size_t k = 0, h = 0, m = 0;
        for (size_t i = 0; i < n; i++) {
            if (lmssubs[i] & (1u << 31)) {
                lmssubs[k] = (uint32_t)(h + m);
                k++;
                h += m;
                m = 0;
            }
            m++;
        }
        lmssubs[k] = (uint32_t)(h + m);
        k++;
        size_t p = wlen - n;
        compact_right(work, wlen, UINT32_MAX);
        translate(work + p, n, lmssubs);
        return k;
    }
    size_t k = 0, h = 0, m = 1;
    size_t i0 = lmssubs[0];
    Fingerprint<C> fp0 = fp_get(text, len, i0);
    reset_slice(work, wlen, UINT32_MAX);
    work[i0 / 2] = 0;
    for (size_t i = 1; i < n; i++) {
        size_t i1 = lmssubs[i];
        Fingerprint<C> fp1 = fp_get(text, len, i1);
        if (!fp_equals(text, len, i0, fp0, i1, fp1)) {
            lmssubs[k] = (uint32_t)(h + m);
            k++;
            h += m;
            m = 0;
        }
        m++;
        i0 = i1;
        fp0 = fp1;
        work[i1 / 2] = (uint32_t)k;
    }
    lmssubs[k] = (uint32_t)(h + m);
    k++;
    size_t p = wlen - n;
    compact_right(work, wlen, UINT32_MAX);
    translate(work + p, n, lmssubs);
    return k;
}

/* src/naming.rs:413-430 permutate_lmssuffixes. */
template <class C>
void permutate_lmssuffixes(const C *text, size_t len, uint32_t *suf, size_t n) {
    size_t p = len;
    foreach_lmschars(text, len, [&](size_t i, C) { suf[--p] = (uint32_t)i; });
    for (size_t i = 0; i < n; i++) {
        size_t j = suf[i];
        suf[i] = suf[p + j];
    }
}

/* ---------------------------------------------------------------------- */
/* Inner levels, u32 (src/psacak32.rs)                                    */
/* ---------------------------------------------------------------------- */

/* src/psacak32.rs:60-99 put_lmscharacters with in-workspace counters. */
void put_lmscharacters32(const uint32_t *text, uint32_t *suf, size_t len) {
    reset_slice(suf, len, EMPTY);
    foreach_lmschars(text, len, [&](size_t i, uint32_t c) {
        size_t p = c;
        if (suf[p] < EMPTY) {
            size_t n = 0;
            while (p + n < len && suf[p + n] < EMPTY) n++;
            std::memmove(suf + p + 1, suf + p, n * sizeof(uint32_t));
            suf[p] = EMPTY;
        }
        if (suf[p] == EMPTY) {
            if (p > 0 && suf[p - 1] == EMPTY) {
                suf[p] = encode_counter(1);
                suf[p - 1] = (uint32_t)i;
            } else {
                suf[p] = (uint32_t)i;
            }
        } else {
            size_t q = p - decode_counter(suf[p]);
            if (q > 0 && suf[q - 1] == EMPTY) {
                suf[p] -= 1;
                suf[q - 1] = (uint32_t)i;
            } else {
                std::memmove(suf + q + 1, suf + q, (p - q) * sizeof(uint32_t));
                suf[q] = (uint32_t)i;
            }
        }
    });
    for (size_t i = len - 1; i >= 1; --i) {
        if (suf[i] > EMPTY) {
            size_t n = decode_counter(suf[i]);
            std::memmove(suf + i - n + 1, suf + i - n, n * sizeof(uint32_t));
            suf[i - n] = EMPTY;
        }
    }
}

/* src/psacak32.rs:103-121 put_lmssuffixes. */
void put_lmssuffixes32(const uint32_t *text, size_t len, uint32_t *suf, size_t n) {
    reset_slice(suf + n, len - n, EMPTY);
    size_t prev = len, m = 0;
    for (size_t i = n; i-- > 0;) {
        size_t x = suf[i];
        suf[i] = EMPTY;
        size_t p = text[x];
        if (p != prev) m = 0;
        suf[p - m] = (uint32_t)x;
        prev = p;
        m++;
    }
}

/* src/psacak32.rs:137-275 nonpar_induce_sort (u32, counters in suf). */
void induce_sort32(const uint32_t *text, uint32_t *suf, size_t len, bool left_most) {
    /* stage 1: induce L (or LML) from LMS, starting with the sentinel. */
    {
        size_t p = text[len - 1];
        if (p + 1 < len && suf[p + 1] == EMPTY) {
            suf[p] = encode_counter(1);
            suf[p + 1] = (uint32_t)(len - 1);
        } else {
            suf[p] = (uint32_t)(len - 1);
        }
    }
    size_t i = 0;
    while (i < len) {
        if (suf[i] > 0 && suf[i] < EMPTY) {
            size_t j = suf[i] - 1;
            uint32_t c0 = text[j], c1 = text[j + 1];
            size_t p = c0;
            if (c0 >= c1) {
                if (suf[p] < EMPTY) {
                    size_t n = 0;
                    while (n <= p && suf[p - n] <= EMPTY) n++;
                    std::memmove(suf + p - n, suf + p + 1 - n, n * sizeof(uint32_t));
                    suf[p] = EMPTY;
                    if (i > p - n) i -= 1;
                }
                if (suf[p] == EMPTY) {
                    if (p + 1 < len && suf[p + 1] == EMPTY) {
                        suf[p] = encode_counter(1);
                        suf[p + 1] = (uint32_t)j;
                    } else {
                        suf[p] = (uint32_t)j;
                    }
                } else {
                    size_t q = p + 1 + decode_counter(suf[p]);
                    if (q < len && suf[q] == EMPTY) {
                        suf[p] -= 1;
                        suf[q] = (uint32_t)j;
                    } else {
                        std::memmove(suf + p, suf + p + 1, (q - p - 1) * sizeof(uint32_t));
                        suf[q - 1] = (uint32_t)j;
                        if (i > p) i -= 1;
                    }
                }
                if (left_most) {
                    suf[i] = EMPTY;
                } else if (j + 2 < len) {
                    uint32_t c2 = text[j + 2];
                    if (!(c1 > c2 || (c1 == c2 && i > (size_t)c1))) suf[i] = EMPTY;
                }
            }
        }
        i += 1;
    }
    /* clean up bucket counters. */
    for (size_t t = 0; t < len; t++) {
        if (suf[t] > EMPTY) {
            size_t n = decode_counter(suf[t]);
            std::memmove(suf + t, suf + t + 1, n * sizeof(uint32_t));
            suf[t + n] = EMPTY;
        }
    }
    /* stage 2: induce S (or LMS) from L (or LML). */
    i = len - 1;
    for (;;) {
        if (suf[i] > 0 && suf[i] < EMPTY) {
            size_t j = suf[i] - 1;
            uint32_t c0 = text[j], c1 = text[j + 1];
            size_t p = c0;
            if (c0 < c1 || (c0 == c1 && i < p)) {
                if (suf[p] < EMPTY) {
                    size_t n = 0;
                    while (p + n < len && suf[p + n] < EMPTY) n++;
                    std::memmove(suf + p + 1, suf + p, n * sizeof(uint32_t));
                    suf[p] = EMPTY;
                    if (i < p + n) i += 1;
                }
                if (suf[p] == EMPTY) {
                    if (p > 0 && suf[p - 1] == EMPTY) {
                        suf[p] = encode_counter(1);
                        suf[p - 1] = (uint32_t)j;
                    } else {
                        suf[p] = (uint32_t)j;
                    }
                } else {
                    size_t q = p - decode_counter(suf[p]);
                    if (q > 0 && suf[q - 1] == EMPTY) {
                        suf[p] -= 1;
                        suf[q - 1] = (uint32_t)j;
                    } else {
                        std::memmove(suf + q + 1, suf + q, (p - q) * sizeof(uint32_t));
                        suf[q] = (uint32_t)j;
                        if (i < p) i += 1;
                    }
                }
                if (left_most) suf[i] = EMPTY;
            }
        }
        if (i == 0) break;
        i -= 1;
    }
}

/* src/psacak32.rs:24-56 psacak32: one inner level on bucket-pointer text. */
void psacak32_level(const uint32_t *text, uint32_t *suf, size_t len, uint32_t level,
                    Trace *tr, unsigned threads = 0) {
    /* with threads: the pipelined scans (src/psacak32.rs:289-484) from two
     * blocks of 64Ki up, the parallel naming */
    const bool par = threads > 1 && len >= 2 * 64 * 1024;
    if (len <= 3) {
        saca_tiny(text, len, suf);
        trace_push(tr, level, 4, len, 0, 0, 0);
        return;
    }
    put_lmscharacters32(text, suf, len);
    if (par) oracle_par::induce_sort32_par(text, suf, len, true, threads);
    else induce_sort32(text, suf, len, true);
    size_t n = compact_left_range(suf, len, 1, EMPTY - 1);
    size_t k = name_lmssubstrings(text, len, suf, n, threads);
    uint32_t *suf1 = suf;
    uint32_t *text1 = suf + (len - n);
    trace_push(tr, level, 4, len, n, k, k < n ? oracle_hash_u32(text1, n) : 0);
    if (k < n) {
        psacak32_level(text1, suf1, n, level + 1, tr, threads);
    } else {
        for (size_t i = 0; i < n; i++) suf1[text1[i]] = (uint32_t)i;
    }
    permutate_lmssuffixes(text, len, suf, n);
    put_lmssuffixes32(text, len, suf, n);
    if (par) oracle_par::induce_sort32_par(text, suf, len, false, threads);
    else induce_sort32(text, suf, len, false);
}

/* ---------------------------------------------------------------------- */
/* Outer level, u8 (src/psacak8.rs)                                       */
/* ---------------------------------------------------------------------- */

/* src/psacak8.rs:347-406 Buckets. */
struct Buckets {
    uint32_t ptrs[256];
    uint32_t bounds[257];
    uint32_t lmscnts[256];
    void build(const uint8_t *text, size_t n) {
        std::memset(ptrs, 0, sizeof(ptrs));
        std::memset(bounds, 0, sizeof(bounds));
        std::memset(lmscnts, 0, sizeof(lmscnts));
        foreach_typedchars(text, n, [&](size_t, TypedChar t, uint8_t c) {
            bounds[c + 1]++;
            if (t.is_lms()) lmscnts[c]++;
        });
        uint32_t p = 0;
        for (int i = 1; i < 257; i++) {
            uint32_t cnt = bounds[i];
            bounds[i] += p;
            p += cnt;
        }
    }
    void set_head() { std::memcpy(ptrs, bounds, sizeof(ptrs)); }
    void set_tail() { std::memcpy(ptrs, bounds + 1, sizeof(ptrs)); }
};

/* src/psacak8.rs:57-72 put_lmscharacters. */
void put_lmscharacters8(const uint8_t *text, size_t n, uint32_t *suf, Buckets &bkt) {
    bkt.set_tail();
    reset_slice(suf, n, 0);
    uint8_t c_prev = text[n - 1];
    size_t p = bkt.ptrs[c_prev];
    foreach_lmschars(text, n, [&](size_t i, uint8_t c) {
        if (c != c_prev) {
            bkt.ptrs[c_prev] = (uint32_t)p;
            p = bkt.ptrs[c];
            c_prev = c;
        }
        p -= 1;
        suf[p] = (uint32_t)i;
    });
}

/* src/psacak8.rs:91-104 move_within. */
void move_within(uint32_t *s, size_t i, size_t j, size_t k, uint32_t reset) {
    std::memmove(s + k, s + i, (j - i) * sizeof(uint32_t));
    size_t a, b;
    if (k > j) { a = i; b = j; }
    else if (k > i) { a = i; b = k; }
    else if (k + (j - i) > i) { a = k + (j - i); b = j; }
    else { a = i; b = j; }
    reset_slice(s + a, b - a, reset);
}

/* src/psacak8.rs:76-87 put_lmssuffixes. */
void put_lmssuffixes8(uint32_t *suf, size_t len, Buckets &bkt, size_t n) {
    bkt.set_tail();
    reset_slice(suf + n, len - n, 0);
    for (int c = 255; c >= 0; c--) {
        size_t m = bkt.lmscnts[c];
        size_t dest = bkt.ptrs[c] - m;
        move_within(suf, n - m, n, dest, 0);
        n -= m;
    }
}

/* src/psacak8.rs:127-190 nonpar_induce_sort (u8). */
void induce_sort8(const uint8_t *text, size_t len, uint32_t *suf, Buckets &bkt,
                  bool left_most) {
    bkt.set_head();
    uint8_t prev_c0 = text[len - 1];
    size_t p = bkt.ptrs[prev_c0];
    suf[p] = (uint32_t)(len - 1);
    p += 1;
    for (size_t i = 0; i < len; i++) {
        if (suf[i] > 0) {
            size_t j = suf[i] - 1;
            uint8_t c0 = text[j], c1 = text[j + 1];
            if (c0 != prev_c0) {
                bkt.ptrs[prev_c0] = (uint32_t)p;
                p = bkt.ptrs[c0];
                prev_c0 = c0;
            }
            if (c0 >= c1) {
                suf[p] = (uint32_t)j;
                p += 1;
                if (left_most) suf[i] = 0;
            }
        }
    }
    bkt.set_tail();
    prev_c0 = 255;
    p = bkt.ptrs[prev_c0];
    for (size_t i = len; i-- > 0;) {
        if (suf[i] > 0) {
            size_t j = suf[i] - 1;
            uint8_t c0 = text[j], c1 = text[j + 1];
            if (c0 != prev_c0) {
                bkt.ptrs[prev_c0] = (uint32_t)p;
                p = bkt.ptrs[c0];
                prev_c0 = c0;
            }
            if (c0 <= c1 && p <= i) {
                p -= 1;
                suf[p] = (uint32_t)j;
                if (left_most) suf[i] = 0;
            }
        }
    }
}

/* src/psacak8.rs:108-123 induce_sort: the pipelined scans from two blocks of
 * 128Ki up when threads are given, else the serial ones. */
void induce_sort8_any(const uint8_t *text, size_t len, uint32_t *suf, Buckets &bkt, bool left_most,
                      unsigned threads) {
    if (threads > 0 && len >= 2 * 128 * 1024)
        oracle_par::induce_sort8_par(text, len, suf, bkt.bounds, bkt.bounds + 1, left_most, threads);
    else induce_sort8(text, len, suf, bkt, left_most);
}

/* PSACAK_ORACLE_TIMES=1: wall time of each stage on stderr (for sizing the
 * CPU baselines; no effect on results). */
static void stage_mark(const char *what) {
    static int on = -1;
    static std::chrono::steady_clock::time_point last;
    if (on < 0) {
        const char *e = getenv("PSACAK_ORACLE_TIMES");
        on = e && e[0] == '1';
        last = std::chrono::steady_clock::now();
    }
    if (!on) return;
    auto now = std::chrono::steady_clock::now();
    fprintf(stderr, "[oracle] %-28s %8.3f s\n", what, std::chrono::duration<double>(now - last).count());
    last = now;
}

/* src/psacak8.rs:19-53 psacak8. */
void psacak8_impl(const uint8_t *text, size_t len, uint32_t *suf, Trace *tr, unsigned threads = 0) {
    if (len <= 3) {
        saca_tiny(text, len, suf);
        trace_push(tr, 0, 1, len, 0, 0, 0);
        return;
    }
    stage_mark("start");
    Buckets bkt;
    bkt.build(text, len);
    put_lmscharacters8(text, len, suf, bkt);
    stage_mark("typing+placement");
    induce_sort8_any(text, len, suf, bkt, true, threads);
    stage_mark("induce lms-substrings");
    size_t n = compact_left(suf, len, 0);
    size_t k = name_lmssubstrings(text, len, suf, n, threads);
    stage_mark("compact+naming");
    uint32_t *suf1 = suf;
    uint32_t *text1 = suf + (len - n);
    trace_push(tr, 0, 1, len, n, k, k < n ? oracle_hash_u32(text1, n) : 0);
    if (tr && tr->reduced_out) {
        size_t c = n < tr->reduced_cap ? n : tr->reduced_cap;
        std::memcpy(tr->reduced_out, text1, c * sizeof(uint32_t));
        tr->reduced_len = n;
        tr->reduced_k = k;
    }
    if (tr && tr->stop_after_level0) return;
    if (k < n) {
        psacak32_level(text1, suf1, n, 1, tr, threads);
    } else {
        for (size_t i = 0; i < n; i++) suf1[text1[i]] = (uint32_t)i;
    }
    stage_mark("inner levels");
    permutate_lmssuffixes(text, len, suf, n);
    put_lmssuffixes8(suf, len, bkt, n);
    stage_mark("permute+put");
    induce_sort8_any(text, len, suf, bkt, false, threads);
    stage_mark("final induce");
}

/* src/psacak32.rs:912-943 translate_sample: ordered histogram, L -> bucket
 * head, S -> bucket tail - 1; declines when distinct >= length. */
bool translate_sample(const uint32_t *text, size_t n, std::vector<uint32_t> &out) {
    std::map<uint32_t, std::pair<uint32_t, uint32_t>> bkt;
    for (size_t i = 0; i < n; i++) {
        auto it = bkt.find(text[i]);
        if (it != bkt.end()) it->second.first++;
        else bkt.emplace(text[i], std::make_pair(1u, 0u));
    }
    if (bkt.size() >= n) return false;
    uint32_t sum = 0;
    for (auto &kv : bkt) {
        uint32_t count = kv.second.first;
        kv.second.first = sum;
        sum += count;
        kv.second.second = sum;
    }
    out.assign(text, text + n);
    foreach_typedchars_mut(out.data(), n, [&](size_t, TypedChar t, uint32_t &p) {
        const auto &e = bkt.find(p)->second;
        p = t.stype ? e.second - 1 : e.first;
    });
    return true;
}

template <class C>
int check_sa(const C *text, uint64_t n, const uint32_t *sa) {
    if (n == 0) return 1;
    std::vector<uint32_t> rank(n + 1, 0);
    for (uint64_t i = 0; i < n; i++) {
        uint32_t x = sa[i];
        if (x >= n || rank[x] != 0) return 0;
        rank[x] = (uint32_t)(i + 1);
    }
    for (uint64_t i = 1; i < n; i++) {
        uint32_t a = sa[i - 1], b = sa[i];
        if (text[a] > text[b]) return 0;
        if (text[a] == text[b] && rank[a + 1] >= rank[b + 1]) return 0;
    }
    return 1;
}

}  // namespace

/* LCP array by Kasai, Lee, Arimura, Arikawa, Park (CPM 2001): inverse
 * suffix array, then the LCP of each suffix with its predecessor in text
 * order, each start one below the previous value.  lcp[0] = 0. */
template <class C>
void kasai(const C *text, uint64_t n, const uint32_t *sa, uint32_t *lcp) {
    if (n == 0) return;
    std::vector<uint32_t> rank(n);
    for (uint64_t i = 0; i < n; i++) rank[sa[i]] = (uint32_t)i;
    uint64_t h = 0;
    lcp[0] = 0;
    for (uint64_t j = 0; j < n; j++) {
        if (rank[j] == 0) {
            h = 0;
            continue;
        }
        uint64_t k = sa[rank[j] - 1];
        while (j + h < n && k + h < n && text[j + h] == text[k + h]) h++;
        lcp[rank[j]] = (uint32_t)h;
        if (h > 0) h--;
    }
}


extern "C" {

uint64_t oracle_hash_u32(const uint32_t *v, uint64_t n) {
    uint64_t h = 0;
    for (uint64_t i = 0; i < n; i++) h += mix64((i << 32) ^ (uint64_t)v[i]);
    return h;
}

int oracle_psacak8(const uint8_t *text, uint64_t n, uint32_t *sa, oracle_level *trace,
                   uint32_t max_levels, uint32_t *n_levels) {
    /* src/lib.rs:78-79: the length must stay below u32::MAX. */
    if (n >= 0xFFFFFFFFull) return -1;
    Trace tr{trace, max_levels, 0, nullptr, 0, 0, 0, false};
    psacak8_impl(text, (size_t)n, sa, &tr);
    if (n_levels) *n_levels = tr.count;
    return 0;
}

int oracle_psacak32(const uint32_t *text, uint64_t n, uint32_t *sa, oracle_level *trace,
                    uint32_t max_levels, uint32_t *n_levels) {
    /* src/psacak32.rs:25: inner strings are limited to 2^31 - 1 symbols. */
    if (n > 0x7FFFFFFFull) return -1;
    Trace tr{trace, max_levels, 0, nullptr, 0, 0, 0, false};
    std::vector<uint32_t> t;
    if (translate_sample(text, (size_t)n, t)) {
        psacak32_level(t.data(), sa, (size_t)n, 0, &tr);
    } else {
        saca_tiny(text, (size_t)n, sa);
    }
    if (n_levels) *n_levels = tr.count;
    return 0;
}

int oracle_psacak8_par(const uint8_t *text, uint64_t n, uint32_t *sa, uint32_t threads) {
    if (n >= 0xFFFFFFFFull) return -1;
    psacak8_impl(text, (size_t)n, sa, nullptr, threads ? threads : 1);
    return 0;
}

void oracle_saca_tiny8(const uint8_t *text, uint64_t n, uint32_t *sa) {
    saca_tiny(text, (size_t)n, sa);
}

void oracle_saca_tiny32(const uint32_t *text, uint64_t n, uint32_t *sa) {
    saca_tiny(text, (size_t)n, sa);
}

int oracle_translate_sample(const uint32_t *text, uint64_t n, uint32_t *out) {
    std::vector<uint32_t> t;
    if (!translate_sample(text, (size_t)n, t)) return 0;
    std::memcpy(out, t.data(), n * sizeof(uint32_t));
    return 1;
}

int oracle_check_sa8(const uint8_t *text, uint64_t n, const uint32_t *sa) {
    return check_sa(text, n, sa);
}

int oracle_check_sa32(const uint32_t *text, uint64_t n, const uint32_t *sa) {
    return check_sa(text, n, sa);
}

void oracle_lcp8(const uint8_t *text, uint64_t n, const uint32_t *sa, uint32_t *lcp) { kasai(text, n, sa, lcp); }
void oracle_lcp32(const uint32_t *text, uint64_t n, const uint32_t *sa, uint32_t *lcp) { kasai(text, n, sa, lcp); }

/* Burrows-Wheeler transform of text + sentinel, the sentinel's character
 * left out (libdivsufsort's divbwt convention): bwt[0] = text[n-1], then
 * text[sa[i]-1] in suffix order skipping sa[i] = 0, whose row (i + 1) is
 * returned as the primary index. */
uint64_t oracle_bwt8(const uint8_t *text, uint64_t n, const uint32_t *sa, uint8_t *bwt) {
    if (n == 0) return 0;
    uint64_t primary = 0, o = 1;
    bwt[0] = text[n - 1];
    for (uint64_t i = 0; i < n; i++) {
        if (sa[i] == 0) primary = i + 1;
        else bwt[o++] = text[sa[i] - 1];
    }
    return primary;
}

/* Suffix-array indices [lo, hi) whose suffixes start with pat[0, m): two
 * binary searches on the suffix array comparing suffixes with the pattern
 * (a suffix that ends inside the pattern's length while equal so far sorts
 * before it).  The independent check of the FM-index's backward search. */
static int cmp_prefix(const uint8_t *text, uint64_t n, uint64_t p, const uint8_t *pat, uint64_t m) {
    for (uint64_t k = 0; k < m; k++) {
        if (p + k >= n) return -1;
        if (text[p + k] != pat[k]) return text[p + k] < pat[k] ? -1 : 1;
    }
    return 0;
}

void oracle_sa_range8(const uint8_t *text, uint64_t n, const uint32_t *sa, const uint8_t *pat, uint64_t m,
                      uint64_t *lo, uint64_t *hi) {
    uint64_t a = 0, b = n;  // first index with cmp >= 0
    while (a < b) {
        uint64_t mid = a + (b - a) / 2;
        if (cmp_prefix(text, n, sa[mid], pat, m) < 0) a = mid + 1;
        else b = mid;
    }
    uint64_t c = a, d = n;  // first index with cmp > 0
    while (c < d) {
        uint64_t mid = c + (d - c) / 2;
        if (cmp_prefix(text, n, sa[mid], pat, m) <= 0) c = mid + 1;
        else d = mid;
    }
    *lo = a;
    *hi = c;
}

uint64_t oracle_reduced8(const uint8_t *text, uint64_t n, uint32_t *out, uint64_t cap,
                         uint64_t *k) {
    if (n <= 3 || n >= 0xFFFFFFFFull) {
        if (k) *k = 0;
        return 0;
    }
    std::vector<uint32_t> suf(n);
    Trace tr{nullptr, 0, 0, out, cap, 0, 0, true};
    psacak8_impl(text, (size_t)n, suf.data(), &tr);
    if (k) *k = tr.reduced_k;
    return tr.reduced_len;
}

}  // extern "C"
