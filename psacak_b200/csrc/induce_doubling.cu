// induce_doubling.cu -- the induced L-/S-scans of one level as chain doubling.
//
// The reference's scans (src/psacak8.rs:127-190, src/psacak32.rs:137-275)
// place every L-type suffix j at the next free slot of bucket text[j] in the
// order in which its successor j+1 is met by the left-to-right scan, and
// every S-type suffix, right to left, in the order of its successor.  The
// L part of a bucket is therefore sorted by the rank of j+1, which is itself
// an L suffix sorted the same way, until the chain reaches an LMS position
// whose slot is known before the scan starts (the "terminal").  In SA-slot
// space every L-type character can stand for the head of its bucket and the
// terminal for its exact slot; comparing these integer chains
// lexicographically reproduces the scan's order (L before S inside a
// bucket, buckets in character order).  The S scan is the mirror image with
// S-type characters standing for the start of the S part and the L slots
// found by the L scan as terminals.
//
// This file resolves those chains with rank doubling: every unresolved item
// (group start g, position j) is keyed by (g, rank[j + h]) for h = 1, 2, 4,
// ...; a round sorts the keys (LSD radix), splits groups where keys differ
// and gives singleton groups their final slot.  Chains end at a terminal,
// so the number of rounds is log2 of the longest L or S run, not of the
// longest repeat.  Nothing here depends on the size of the alphabet.
#include "ctx.cuh"
#include "induce.cuh"

#include <utility>

namespace psk {

// Per sorted item: last group start (max), last subgroup start (max), kept
// items (sum) and kept subgroups started (sum).
struct Tri {
    uint32_t g, s, k, o;
};
__device__ __forceinline__ Tri shfl_up_t(Tri v, int o) {
    Tri r;
    r.g = __shfl_up_sync(FULL_MASK, v.g, o);
    r.s = __shfl_up_sync(FULL_MASK, v.s, o);
    r.k = __shfl_up_sync(FULL_MASK, v.k, o);
    r.o = __shfl_up_sync(FULL_MASK, v.o, o);
    return r;
}
struct OpTri {
    static constexpr int kFields = 4;  // g, s: max; k, o: sum
    __device__ __forceinline__ static uint32_t field(int f, uint32_t a, uint32_t b) {
        return f < 2 ? (a > b ? a : b) : a + b;
    }
    __device__ __forceinline__ Tri operator()(Tri a, Tri b) const {
        Tri r;
        r.g = a.g > b.g ? a.g : b.g;
        r.s = a.s > b.s ? a.s : b.s;
        r.k = a.k + b.k;
        r.o = a.o + b.o;
        return r;
    }
    __device__ __forceinline__ static Tri identity() { return Tri{0, 0, 0, 0}; }
};

// ---- terminal slots of the LMS positions ---------------------------------

// LMS-substring mode: LMS positions take distinct slots at the tail of their
// bucket in arbitrary order (the reference's put_lmscharacters,
// src/psacak8.rs:57-72 / src/psacak32.rs:60-99).  A lane per 32-position
// word; lanes that meet the same bucket in one step share one atomic
// (frequent symbols would otherwise serialise on their cursor).
template <class C>
__global__ void k_place_lms_any(const C *__restrict__ text, uint64_t nwords, const uint32_t *__restrict__ lms,
                                Geom<C> g, uint32_t *cursor, uint32_t *R) {
    const uint32_t lane = threadIdx.x & 31, lt = lanemask_lt();
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t wb = (uint64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31u); wb < nwords; wb += stride) {
        const uint64_t w = wb + lane;
        uint32_t word = w < nwords ? lms[w] : 0u;
        while (__any_sync(FULL_MASK, word != 0)) {
            const bool on = word != 0;
            uint64_t p = 0;
            C c = 0;
            uint32_t bk = 0xFFFFFFFFu;
            if (on) {
                p = (w << 5) + (uint64_t)(__ffs(word) - 1);
                word &= word - 1;
                c = text[p];
                bk = g.bucket(c);
            }
            const uint32_t peers = __match_any_sync(FULL_MASK, bk);
            const int leader = __ffs(peers) - 1;
            uint32_t base = 0;
            if (on && (int)lane == leader) base = atomicAdd(&cursor[bk], __popc(peers));
            base = __shfl_sync(FULL_MASK, base, leader);
            if (on) R[p] = g.tail(c) - (base + __popc(peers & lt));  // slot tail-1-rank, plus one
        }
    }
}

// Final mode: the sorted LMS suffixes fill the tail of each bucket in order
// (the reference's put_lmssuffixes, src/psacak8.rs:76-87 /
// src/psacak32.rs:103-121).  `last` = index of the last list entry of the
// same bucket, found by a max-scan over the reversed list.
template <class C> struct LastLoad {
    static constexpr int kIPT = 8;
    struct Payload {
        uint32_t p;     // the LMS position
        uint32_t tail;  // tail slot (+1) of its bucket
    };
    const uint64_t *sorted;  // position | symbol << 32, in suffix order
    uint64_t n1;
    Geom<C> g;
    __device__ __forceinline__ uint32_t operator()(uint64_t r, Payload &pl) const {
        uint64_t i = n1 - 1 - r;
        const uint64_t e = sorted[i];
        pl.p = (uint32_t)e;
        const C c = (C)(e >> 32);
        pl.tail = g.tail(c);
        bool last = (i + 1 == n1) || g.bucket((C)(sorted[i + 1] >> 32)) != g.bucket(c);
        return last ? (uint32_t)(r + 1) : 0u;
    }
};
template <class C> struct LastStore {
    uint64_t n1;
    uint32_t *R;
    __device__ __forceinline__ void operator()(uint64_t r, uint32_t excl, uint32_t v,
                                               const typename LastLoad<C>::Payload &pl) const {
        uint32_t inc = excl > v ? excl : v;
        uint64_t i = n1 - 1 - r;
        uint64_t last = n1 - inc;
        R[pl.p] = pl.tail - (uint32_t)(last - i);
    }
};

// ---- work list -----------------------------------------------------------

// The work list is a stable compaction of the positions of one type: a scan
// over the 32-position type words' popcounts gives every word its first
// slot, then a kernel with a thread per position emits the selected ones
// (slot = word's first slot + selected positions before it in the word).
template <bool STYPE> __device__ __forceinline__ uint32_t selected_bits(const uint32_t *types, uint64_t n, uint64_t w) {
    uint32_t bits = STYPE ? types[w] : ~types[w];
    const uint64_t p0 = w << 5;
    if (n - p0 < 32) bits &= (1u << (uint32_t)(n - p0)) - 1u;
    return bits;
}
template <bool STYPE> struct WordLoad {
    const uint32_t *types;
    uint64_t n;
    __device__ __forceinline__ uint32_t operator()(uint64_t w) const { return __popc(selected_bits<STYPE>(types, n, w)); }
};
struct WordStore {
    uint32_t *first;
    __device__ __forceinline__ void operator()(uint64_t w, uint32_t excl, uint32_t) const { first[w] = excl; }
};
template <bool STYPE, class Emit>
__global__ void k_emit_selected(const uint32_t *__restrict__ types, const uint32_t *__restrict__ first, uint64_t n,
                                Emit emit) {
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;  // a multiple of 32: lanes stay word-aligned
    for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += stride) {
        const uint64_t w = j >> 5;
        const uint32_t bits = selected_bits<STYPE>(types, n, w);
        if ((bits >> lane) & 1u) emit(j, first[w] + __popc(bits & ((1u << lane) - 1u)));
    }
}

// Work item = (dense group id, position); the group id of round 1 is the
// symbol's name and gstart[id] the first SA slot of its L (or S) part.
template <class C, bool STYPE> struct WEmit {
    const C *text;
    Geom<C> g;
    uint32_t *Wg, *Wv, *R;
    __device__ __forceinline__ void operator()(uint64_t j, uint32_t slot) const {
        C c = text[j];
        uint32_t grp = STYPE ? g.sgroup(c) : g.lgroup(c);
        Wg[slot] = g.name(j, c);
        Wv[slot] = (uint32_t)j;
        R[j] = grp + 1;
    }
};

// Group starts of a whole-string sort's first round (the bucket heads), and
// the item count where the rounds read it on the device.
__global__ void k_copy_heads(const uint32_t *bheads, uint64_t nbuckets, uint32_t *gstart, uint32_t *dcount,
                             uint32_t n) {
    if (blockIdx.x == 0 && threadIdx.x == 0) *dcount = n;
    for (uint64_t c = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; c < nbuckets; c += (uint64_t)gridDim.x * blockDim.x)
        gstart[c] = bheads[c];
}

template <class C, bool STYPE>
__global__ void k_group_starts(Geom<C> g, uint64_t nbuckets, uint32_t *gstart) {
    for (uint64_t c = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; c < nbuckets; c += (uint64_t)gridDim.x * blockDim.x)
        gstart[c] = STYPE ? g.sstart_of((uint32_t)c) : g.lstart_of((uint32_t)c);
}

// Keys of one round: (group id, rank of j + h).  The block also counts the
// digits of every radix pass of the keys (bits [0, nbits)) into `hist`, so
// the sort needs no histogram pass of its own.
// `dcnt` (nullable): the item count is on the device, cnt_max bounds it.
__global__ void __launch_bounds__(256) k_keys(const uint32_t *__restrict__ Wg, const uint32_t *__restrict__ Wv,
                                              uint64_t cnt_max, const uint32_t *dcnt, const uint32_t *__restrict__ R,
                                              uint64_t n, uint64_t h, int KB, uint64_t *keys, uint32_t *vals,
                                              int nbits, uint32_t *hist, uint32_t *err) {
    __shared__ uint32_t sh[RADIX_MAX_PASSES * 256];
    const uint64_t cnt = dcnt ? (*dcnt < cnt_max ? *dcnt : cnt_max) : cnt_max;
    const int npasses = (nbits + 7) / 8;
    for (int i = threadIdx.x; i < npasses * 256; i += blockDim.x) sh[i] = 0;
    __syncthreads();
    constexpr int U = 4;  // items per thread step: their rank gathers overlap
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t ib = (uint64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31u); ib < cnt; ib += stride * U) {
        uint32_t v[U], g[U], r[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
            const uint64_t i = ib + u * stride + (threadIdx.x & 31);
            v[u] = i < cnt ? Wv[i] : 0u;
            g[u] = i < cnt ? Wg[i] : 0u;
        }
#pragma unroll
        for (int u = 0; u < U; u++) {
            const uint64_t i = ib + u * stride + (threadIdx.x & 31);
            r[u] = 0;
            if (i < cnt) {
                const uint64_t q = (uint64_t)v[u] + h;
                if (q <= n) r[u] = R[q];
                else dev_fail(err, DEVERR_RANGE);
            }
        }
#pragma unroll
        for (int u = 0; u < U; u++) {
            const uint64_t i = ib + u * stride + (threadIdx.x & 31);
            const bool valid = i < cnt;
            const uint64_t key = ((uint64_t)g[u] << KB) | r[u];
            if (valid) {
                keys[i] = key;
                vals[i] = v[u];
            }
            radix_count_digits(sh, key, valid, 0, npasses, nbits);
        }
    }
    __syncthreads();
    radix_flush_digits(sh, npasses, hist);
}

// Keys of the first round of a whole-string sort, where every position j is
// an item (item j = position j): the group (the name of j) above the names
// of j + 1 .. j + P - 1, each + 1 in NB bits (0 at and past the end of the
// string).  These order the suffixes by their first P symbols, so the round
// after it doubles from h = P instead of h = 1: the early rounds, in which
// nearly every item is still unresolved, run fewer times.  The kernel also
// gives every position its first rank, the slot of its bucket's head + 1.
// Digits are counted as in k_keys.
__global__ void __launch_bounds__(256) k_keys_packed(const uint32_t *__restrict__ names,
                                                     const uint32_t *__restrict__ bheads, uint64_t n, int P, int NB,
                                                     uint64_t *keys, uint32_t *vals, uint32_t *R, int nbits,
                                                     uint32_t *hist) {
    __shared__ uint32_t sh[RADIX_MAX_PASSES * 256];
    const int npasses = (nbits + 7) / 8;
    const int KB = (P - 1) * NB;
    for (int i = threadIdx.x; i < npasses * 256; i += blockDim.x) sh[i] = 0;
    __syncthreads();
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t ib = (uint64_t)blockIdx.x * blockDim.x; ib < n; ib += stride) {
        const uint64_t j = ib + threadIdx.x;
        const bool valid = j < n;
        uint64_t key = 0;
        if (valid) {
            const uint32_t g = names[j];
            uint64_t r = 0;
            for (int t = 1; t < P; t++) {
                const uint64_t q = j + t;
                r = (r << NB) | (q < n ? names[q] + 1u : 0u);
            }
            key = ((uint64_t)g << KB) | r;
            keys[j] = key;
            vals[j] = (uint32_t)j;
            R[j] = bheads[g] + 1;
        }
        radix_count_digits(sh, key, valid, 0, npasses, nbits);
    }
    __syncthreads();
    radix_flush_digits(sh, npasses, hist);
}

// The load also fetches the item's position and its group's first slot
// (the store's only reads), so their latency overlaps the scan.
struct RoundPayload {
    uint32_t val;  // position
    uint32_t gs;   // first slot of the item's group
};
// Two phases (see lbscan.cuh): the item's key, its neighbours' keys and its
// position for every item of the thread first, then the group-start gathers.
struct RoundPre {
    uint64_t k, kp, kn;  // this key, the previous one, the next one (see `has`)
    uint32_t val;
    uint32_t has;  // bit 0: a previous item exists, bit 1: a next one
};
struct RoundLoad {
    using Payload = RoundPayload;
    using Pre = RoundPre;
    static constexpr int kIPT = 6;
    const uint64_t *keys;
    const uint32_t *vals;
    const uint32_t *gstart;  // group id -> first slot (this round)
    uint64_t cnt, n, ngroups;  // ngroups: a bound of the group ids
    int KB;
    uint32_t *err;
    const uint32_t *dcnt;  // nullable: the item count on the device (cnt bounds it)
    __device__ __forceinline__ void pre(uint64_t i, RoundPre &p) const {
        const uint64_t cnt = dcnt ? (*dcnt < this->cnt ? *dcnt : this->cnt) : this->cnt;
        p.k = keys[i];
        p.val = vals[i];
        p.has = (i > 0 ? 1u : 0u) | (i + 1 < cnt ? 2u : 0u);
        p.kp = (p.has & 1u) ? keys[i - 1] : 0ull;
        p.kn = (p.has & 2u) ? keys[i + 1] : 0ull;
    }
    __device__ __forceinline__ Tri operator()(uint64_t i, const RoundPre &p, RoundPayload &pl) const {
        const uint64_t k = p.k;
        const uint64_t gid = k >> KB;
        pl.val = p.val;
        pl.gs = 0;
        if (gid < ngroups && pl.val < n) pl.gs = gstart[gid];
        else pl.val = 0xFFFFFFFFu;  // reported by the store
        bool gb = true, sb = true, sbn = true;
        if (p.has & 1u) {
            gb = (p.kp >> KB) != (k >> KB);
            sb = p.kp != k;
        }
        if (p.has & 2u) sbn = p.kn != k;
        Tri t;
        t.g = gb ? (uint32_t)(i + 1) : 0u;
        t.s = sb ? (uint32_t)(i + 1) : 0u;
        bool keep = !(sb && sbn);
        t.k = keep ? 1u : 0u;
        t.o = (keep && sb) ? 1u : 0u;
        return t;
    }
};
// Algorithmic bytes of the round scan per item: its key and position read
// (12), its new rank written (4) and, for a kept item, its work-list entry
// written (8; a resolved item writes its 4-byte slot instead).
constexpr uint64_t ROUND_SCAN_BYTES = 24;
struct RoundStore {
    uint32_t *gnext;  // kept subgroup ordinal -> first slot (next round)
    uint32_t *R, *sa, *Wg, *Wv;
    uint64_t n;
    uint32_t *err;
    __device__ __forceinline__ void operator()(uint64_t i, Tri excl, Tri v, const RoundPayload &pl) const {
        uint32_t gs = (excl.g > v.g ? excl.g : v.g) - 1;
        uint32_t ss = (excl.s > v.s ? excl.s : v.s) - 1;
        const uint32_t val = pl.val;
        if (val >= n) {
            dev_fail(err, DEVERR_RANGE);
            return;
        }
        uint32_t newg = pl.gs + (ss - gs);
        if (newg >= n) {
            dev_fail(err, DEVERR_RANGE);
            return;
        }
        // Every item's rank is its group's first slot + 1 when the round
        // starts; items of the group's first subgroup keep it.
        if (ss != gs) R[val] = newg + 1;
        if (v.k) {
            uint32_t ord = excl.o + v.o - 1;
            Wg[excl.k] = ord;
            Wv[excl.k] = val;
            if (v.o) gnext[ord] = newg;
        } else {
            sa[newg] = val;
        }
    }
};

// ---- rounds over a work list ordered by group ----------------------------
//
// Every round after a list's first reads the list that the previous round's
// scan wrote, in sorted order, so the items of a group are contiguous and
// groups follow one another in key order.  Only the ranks inside each group
// need sorting.  Past the first few rounds nearly all groups are a handful of
// items, so a CTA sorts the small groups that start in its tile in shared
// memory (each item's slot = the group's start + the items of the group with
// a smaller (rank, index)), and the items of groups larger than SEG_MAX go
// through a compaction, the radix sort and a scatter back into place.  The
// output is the same (key, position) sequence as a full sort up to the order
// of equal keys, which the scan that follows does not depend on.
constexpr int SEG_BLOCK = 256;
constexpr int SEG_TILE = 2048;  // list items whose groups a CTA decides
constexpr int SEG_MAX = 64;     // largest group sorted in shared memory
constexpr int SEG_WIN = SEG_TILE + 2 * SEG_MAX;
constexpr int SEG_WORDS = (SEG_WIN + 1 + 31) / 32;
constexpr int SEG_OWN = SEG_TILE + SEG_MAX;  // items of the groups a CTA owns
constexpr int SEG_STEPS = (SEG_OWN + SEG_BLOCK - 1) / SEG_BLOCK;
// Use the in-place path when the previous round left at most this many
// items per kept group on average.
constexpr uint32_t SEG_AVG_MAX = 16;

// Highest set bit of the boundary bitmap in [lo, x], or -1.
__device__ __forceinline__ int seg_prev(const uint32_t *bm, int x, int lo) {
    int w = x >> 5;
    uint32_t m = bm[w] & (0xFFFFFFFFu >> (31 - (x & 31)));
    while (true) {
        if (m) {
            const int p = (w << 5) + 31 - __clz(m);
            return p >= lo ? p : -1;
        }
        if ((w << 5) <= lo) return -1;
        m = bm[--w];
    }
}
// Lowest set bit of the boundary bitmap in [x + 1, hi], or -1.
__device__ __forceinline__ int seg_next(const uint32_t *bm, int x, int hi) {
    const int p0 = x + 1;
    if (p0 > hi) return -1;
    int w = p0 >> 5;
    uint32_t m = bm[w] & (0xFFFFFFFFu << (p0 & 31));
    while (true) {
        if (m) {
            const int p = (w << 5) + __ffs(m) - 1;
            return p <= hi ? p : -1;
        }
        if (((w + 1) << 5) > hi) return -1;
        m = bm[++w];
    }
}

// Keys of one round over a group-ordered list (see above).  CTA b decides
// the list items [t0, t1) = [b * SEG_TILE, ...): it reads the group ids of
// the window [t0 - SEG_MAX - 1, t1 + SEG_MAX), marks where groups start, and
//  * sorts every group of at most SEG_MAX items that starts in [t0, t1)
//    (such a group ends before t1 + SEG_MAX),
//  * writes the items of [t0, t1) that belong to larger groups in place and
//    flags them in `big` (a group whose start lies more than SEG_MAX items
//    back, or whose end lies more than SEG_MAX items ahead, is large),
//  * adds its flagged items to *bigcnt.
// Items of small groups that start before t0 belong to the previous CTA.
__global__ void __launch_bounds__(SEG_BLOCK) k_seg_keys(const uint32_t *__restrict__ Wg,
                                                        const uint32_t *__restrict__ Wv, uint64_t cnt,
                                                        const uint32_t *__restrict__ R, uint64_t n, uint64_t h,
                                                        int KB, uint64_t *keys, uint32_t *vals, uint8_t *big,
                                                        uint32_t *bigcnt, uint32_t *err) {
    __shared__ uint32_t s_g[SEG_WIN + 1];  // s_g[x + 1] = Wg[wlo + x]; s_g[0] = Wg[wlo - 1]
    __shared__ uint32_t s_bm[SEG_WORDS];   // bit x: list item wlo + x starts a group (x == L: the list's end)
    __shared__ uint32_t s_r[SEG_OWN], s_v[SEG_OWN];
    __shared__ uint32_t s_red[33];
    const uint64_t t0 = (uint64_t)blockIdx.x * SEG_TILE;
    const uint64_t t1 = t0 + SEG_TILE < cnt ? t0 + SEG_TILE : cnt;
    const uint64_t wlo = t0 > (uint64_t)SEG_MAX ? t0 - SEG_MAX : 0;
    const uint64_t whi = t1 + SEG_MAX < cnt ? t1 + SEG_MAX : cnt;
    const int L = (int)(whi - wlo);
    const int xt0 = (int)(t0 - wlo), xt1 = (int)(t1 - wlo);
    for (int x = threadIdx.x; x <= L; x += SEG_BLOCK) {
        if (x == 0) s_g[0] = wlo > 0 ? Wg[wlo - 1] : 0xFFFFFFFFu;
        else s_g[x] = Wg[wlo + x - 1];
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nw = (L + 1 + 31) >> 5;
    for (int base = warp * 32; base < nw * 32; base += SEG_BLOCK) {  // warp-uniform
        const int x = base + lane;
        bool b = false;
        if (x < L) b = (wlo + x == 0) || s_g[x + 1] != s_g[x];
        else if (x == L) b = whi == cnt;
        const uint32_t m = __ballot_sync(FULL_MASK, b);
        if (lane == 0) s_bm[base >> 5] = m;
    }
    __syncthreads();
    // each owned or flagged item: its rank gather
    int ga[SEG_STEPS], gb[SEG_STEPS];
    uint32_t nbig = 0;
#pragma unroll
    for (int u = 0; u < SEG_STEPS; u++) {
        const int x = xt0 + u * SEG_BLOCK + (int)threadIdx.x;
        ga[u] = -1;
        gb[u] = -1;
        if (x >= L) continue;
        const int lo = x - SEG_MAX + 1 > 0 ? x - SEG_MAX + 1 : 0;
        const int a = seg_prev(s_bm, x, lo);
        const int b = a >= 0 ? seg_next(s_bm, x, a + SEG_MAX < L ? a + SEG_MAX : L) : -1;
        const bool small = b >= 0;
        const bool owned = small && a >= xt0 && a < xt1;
        const bool flagged = !small && x < xt1;
        if (x < xt1) big[wlo + x] = flagged ? 1 : 0;
        if (!owned && !flagged) continue;
        const uint32_t v = Wv[wlo + x];
        const uint64_t q = (uint64_t)v + h;
        uint32_t r = 0;
        if (q <= n) r = R[q];
        else dev_fail(err, DEVERR_RANGE);
        s_r[x - xt0] = r;
        s_v[x - xt0] = v;
        if (owned) {
            ga[u] = a;
            gb[u] = b;
        } else {
            keys[wlo + x] = ((uint64_t)s_g[x + 1] << KB) | r;
            vals[wlo + x] = v;
            nbig++;
        }
    }
    __syncthreads();
#pragma unroll
    for (int u = 0; u < SEG_STEPS; u++) {
        if (ga[u] < 0) continue;
        const int x = xt0 + u * SEG_BLOCK + (int)threadIdx.x;
        const uint32_t r = s_r[x - xt0];
        int less = 0;
        for (int y = ga[u]; y < gb[u]; y++) {
            const uint32_t ry = s_r[y - xt0];
            less += (ry < r || (ry == r && y < x)) ? 1 : 0;
        }
        const uint64_t p = wlo + (uint64_t)(ga[u] + less);
        keys[p] = ((uint64_t)s_g[x + 1] << KB) | r;
        vals[p] = s_v[x - xt0];
    }
    uint32_t tot = 0;
    block_exclusive_sum<uint32_t, SEG_BLOCK>(nbig, s_red, &tot);
    if (threadIdx.x == 0 && tot) atomicAdd(bigcnt, tot);
}

// The flagged items, in list order, with their list index.
struct BigPred {
    const uint8_t *big;
    __device__ __forceinline__ bool operator()(uint64_t i) const { return big[i] != 0; }
};
struct BigEmit {
    const uint64_t *keys;
    const uint32_t *vals;
    uint64_t *bk;
    uint32_t *bv, *src;
    __device__ __forceinline__ void operator()(uint64_t i, uint32_t slot) const {
        bk[slot] = keys[i];
        bv[slot] = vals[i];
        src[slot] = (uint32_t)i;
    }
};
// The sorted flagged items back into the list.  A large group's items were
// gathered in list order and sort to a contiguous run of the same length,
// so the q-th sorted item takes the list index of the q-th gathered one.
__global__ void k_seg_back(const uint64_t *__restrict__ bk, const uint32_t *__restrict__ bv,
                           const uint32_t *__restrict__ src, uint64_t nb, uint64_t cnt, uint64_t *keys,
                           uint32_t *vals, uint32_t *err) {
    for (uint64_t q = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; q < nb; q += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t i = src[q];
        if (i >= cnt) {
            dev_fail(err, DEVERR_RANGE);
            continue;
        }
        keys[i] = bk[q];
        vals[i] = bv[q];
    }
}

// Keys of a group-ordered round (k_seg_keys, then the large groups' sort).
static status_t seg_round_keys(Ctx &ctx, const uint32_t *Wg, const uint32_t *Wv, uint64_t cnt, const uint32_t *R,
                               uint64_t n, uint64_t h, int KB, int GB, uint64_t *keys, uint32_t *vals,
                               cudaStream_t s) {
    uint32_t *d_big = ctx.d_scalars + 13;
    DBuf<uint8_t> big;
    PSK_TRY(big.init(ctx, cnt));
    PSK_CUDA(cudaMemsetAsync(d_big, 0, sizeof(uint32_t), s));
    const uint64_t g = ceil_div(cnt, SEG_TILE);
    PSK_PROF_LAUNCH(s, "double_seg_keys", cnt, 21ull * cnt,
                    (k_seg_keys<<<(uint32_t)g, SEG_BLOCK, 0, s>>>(Wg, Wv, cnt, R, n, h, KB, keys, vals, big, d_big,
                                                                  ctx.d_err)));
    PSK_LAUNCH_CHECK();
    uint32_t nb = 0;
    PSK_TRY(ctx.read_u32(d_big, &nb));
    if (ctx.stage_timing)
        fprintf(stderr, "[psacak]   group-ordered round h=%llu: %llu items, %u in groups over %d\n",
                (unsigned long long)h, (unsigned long long)cnt, nb, SEG_MAX);
    if (nb == 0) return PSACAK_OK;
    DBuf<uint64_t> bk0, bk1;
    DBuf<uint32_t> bv0, bv1, src;
    PSK_TRY(bk0.init(ctx, nb));
    PSK_TRY(bk1.init(ctx, nb));
    PSK_TRY(bv0.init(ctx, nb));
    PSK_TRY(bv1.init(ctx, nb));
    PSK_TRY(src.init(ctx, nb));
    PSK_TRY(ctx.compact(BigPred{big}, BigEmit{keys, vals, bk0, bv0, src}, cnt, ctx.d_scalars + 14, "seg_gather"));
    int in1 = 0;
    PSK_TRY((ctx.radix_sort<uint64_t, uint32_t>(bk0, bv0, bk1, bv1, nb, 0, KB + GB, &in1)));
    const uint64_t gg = ceil_div(nb, 256);
    PSK_PROF_LAUNCH(s, "seg_back", nb, 28ull * nb,
                    (k_seg_back<<<(uint32_t)(gg < 16384 ? gg : 16384), 256, 0, s>>>(
                        in1 ? bk1.get() : bk0.get(), in1 ? bv1.get() : bv0.get(), src, nb, cnt, keys, vals,
                        ctx.d_err)));
    PSK_LAUNCH_CHECK();
    return PSACAK_OK;
}

static status_t doubling_rounds(Ctx &ctx, uint64_t n, uint64_t nbuckets, uint32_t cnt, const uint32_t *d_cnt0,
                                uint32_t *R, uint32_t *sa, uint32_t *Wg, uint32_t *Wv, uint64_t *k0, uint32_t *v0,
                                uint64_t *k1, uint32_t *v1, uint32_t *gA, uint32_t *gB, const uint32_t *names1,
                                const uint32_t *bheads1, char tag, cudaStream_t s);

// One scan (L or S): resolves the chains of every item of the given type.
template <class C, bool STYPE>
static status_t doubling_scan(Ctx &ctx, const C *text, uint64_t n, const uint32_t *types, Geom<C> geom,
                              uint64_t nbuckets, uint32_t *R, uint32_t *sa, uint32_t *Wg, uint32_t *Wv, uint64_t *k0,
                              uint32_t *v0, uint64_t *k1, uint32_t *v1, uint32_t *gA, uint32_t *gB, cudaStream_t s) {
    uint32_t *d_cnt = ctx.d_scalars;
    {
        uint64_t gb = ceil_div(nbuckets, 256);
        k_group_starts<C, STYPE><<<(uint32_t)(gb < 4096 ? gb : 4096), 256, 0, s>>>(geom, nbuckets, gA);
        PSK_KCOUNT();
        PSK_LAUNCH_CHECK();
    }
    {
        const uint64_t nwords = ceil_div(n, 32);
        DBuf<uint32_t> first;
        PSK_TRY(first.init(ctx, nwords));
        PSK_TRY((ctx.scan<uint32_t, OpSum<uint32_t>>(WordLoad<STYPE>{types, n}, WordStore{first}, nwords, d_cnt,
                                                     OpSum<uint32_t>(), "double_words")));
        const uint64_t g = ceil_div(n, 256);
        PSK_PROF_LAUNCH(s, "double_items", n, 0,
                        (k_emit_selected<STYPE, WEmit<C, STYPE>><<<(uint32_t)(g < 16384 ? g : 16384), 256, 0, s>>>(
                            types, first, n, WEmit<C, STYPE>{text, geom, Wg, Wv, R})));
        PSK_LAUNCH_CHECK();
    }
    uint32_t cnt = 0;
    PSK_TRY(ctx.read_u32(d_cnt, &cnt));
    return doubling_rounds(ctx, n, nbuckets, cnt, d_cnt, R, sa, Wg, Wv, k0, v0, k1, v1, gA, gB, nullptr, nullptr,
                           STYPE ? 'S' : 'L', s);
}

// Rounds of a work list shorter than this run DOUBLING_SPEC_ROUNDS at a
// time without a host round trip between them: the counts stay on the
// device (each kernel reads the current one and the launches are sized for
// the count at the start of the block), the key width covers any group id
// the block can meet, and every radix pass runs.  A round left with no
// items costs a handful of empty launches, less than a read-back.
constexpr uint32_t DOUBLING_SPEC_MAX = 1u << 20;
// Most symbols packed into the first round's keys (k_keys_packed).
constexpr int DOUBLING_PACK_MAX = 16;
constexpr int DOUBLING_SPEC_ROUNDS = 2;

// Rank-doubling rounds over the work list (Wg = dense group id, Wv =
// position) until every item has its own slot.  `d_cnt0`: the device word
// holding cnt (the work list's count).
static status_t doubling_rounds(Ctx &ctx, uint64_t n, uint64_t nbuckets, uint32_t cnt, const uint32_t *d_cnt0,
                                uint32_t *R, uint32_t *sa, uint32_t *Wg, uint32_t *Wv, uint64_t *k0, uint32_t *v0,
                                uint64_t *k1, uint32_t *v1, uint32_t *gA, uint32_t *gB, const uint32_t *names1,
                                const uint32_t *bheads1, char tag, cudaStream_t s) {
    const int KB = bitlen(n);
    uint64_t ngroups = nbuckets;
    // round totals alternate between two device slots: a round reads its
    // count from the one the previous round wrote
    Tri *d_tri[2] = {(Tri *)(ctx.d_scalars + 4), (Tri *)(ctx.d_scalars + 8)};
    int tb = 0;
    const uint32_t *dcnt = d_cnt0;
    // The work list (Wg, Wv) lives as two u32 arrays inside the key array of
    // the radix pair that is spare: it enters in (k1, v1), the keys are built
    // into the other pair, and each round writes the next list into whichever
    // pair the sort did not leave its result in.
    uint64_t *kA = k0, *kB = k1;
    uint32_t *vA = v0, *vB = v1;
    if (Wg != (uint32_t *)k1 || Wv != Wg + n)
        return set_error(PSACAK_EINTERNAL, "doubling rounds: work list outside its radix pair");
    uint64_t h = 1;
    while (cnt > 0) {
        if (h > n) return set_error(PSACAK_EINTERNAL, "doubling scan did not converge (n=%llu)", (unsigned long long)n);
        const bool spec = cnt < DOUBLING_SPEC_MAX;
        const int rounds = spec ? DOUBLING_SPEC_ROUNDS : 1;
        for (int r = 0; r < rounds && h <= n; r++) {
            PSK_TRY(ctx.checkpoint());
            // group ids: < ngroups in the block's first round, and later
            // below the items left (kept subgroups never outnumber them)
            const uint64_t gbound = r == 0 ? ngroups : (cnt > 0 ? cnt : 1);
            const int GB = bitlen(gbound > 0 ? gbound - 1 : 0);
            const uint32_t *dc = spec ? dcnt : nullptr;
            // the first round of a whole-string sort keys by packed names:
            // as many symbols as fit beside the group id in 64 bits
            const bool packed = h == 1 && names1 && bheads1;
            const int NB = bitlen(nbuckets);
            int P = packed ? 1 + (64 - GB) / NB : 1;
            if (P > DOUBLING_PACK_MAX) P = DOUBLING_PACK_MAX;
            const int KBr = packed ? (P - 1) * NB : KB;
            // a list written by the previous round is ordered by group
            const bool seg = !spec && h > 1 && ngroups > 0 && (uint64_t)cnt <= (uint64_t)SEG_AVG_MAX * ngroups;
            int in1 = 0;
            if (seg) {
                PSK_TRY(seg_round_keys(ctx, Wg, Wv, cnt, R, n, h, KBr, GB, kA, vA, s));
            } else {
                uint64_t gblocks = ceil_div(cnt, 256 * 16);
                PSK_CUDA(cudaMemsetAsync(ctx.d_hist, 0, RADIX_MAX_PASSES * 256 * sizeof(uint32_t), s));
                if (packed) {
                    if (cnt != n) return set_error(PSACAK_EINTERNAL, "doubling: first round over %u of %llu items",
                                                   cnt, (unsigned long long)n);
                    PSK_PROF_LAUNCH(s, "double_keys", cnt, 20ull * cnt,
                                    (k_keys_packed<<<(uint32_t)(gblocks < 1184 ? gblocks : 1184), 256, 0, s>>>(
                                        names1, bheads1, n, P, NB, kA, vA, R, KBr + GB, ctx.d_hist)));
                } else {
                    PSK_PROF_LAUNCH(s, "double_keys", cnt, 20ull * cnt,
                                    (k_keys<<<(uint32_t)(gblocks < 1184 ? gblocks : 1184), 256, 0, s>>>(
                                        Wg, Wv, cnt, dc, R, n, h, KBr, kA, vA, KBr + GB, ctx.d_hist, ctx.d_err)));
                }
                PSK_LAUNCH_CHECK();
                PSK_TRY((ctx.radix_sort<uint64_t, uint32_t>(kA, vA, kB, vB, cnt, 0, KBr + GB, &in1, true, dc)));
            }
            uint64_t *ks = in1 ? kB : kA, *kfree = in1 ? kA : kB;
            uint32_t *vs = in1 ? vB : vA, *vfree = in1 ? vA : vB;
            Wg = (uint32_t *)kfree;
            Wv = Wg + n;
            Tri *tout = d_tri[tb];
            PSK_TRY((ctx.scan<Tri, OpTri>(RoundLoad{ks, vs, gA, cnt, n, gbound, KBr, ctx.d_err, dc},
                                          RoundStore{gB, R, sa, Wg, Wv, n, ctx.d_err}, cnt, tout, OpTri(),
                                          "scan_rounds", dc, ROUND_SCAN_BYTES * (uint64_t)cnt)));
            kA = ks;
            vA = vs;
            kB = kfree;
            vB = vfree;
            dcnt = &tout->k;
            tb ^= 1;
            std::swap(gA, gB);
            if (ctx.stage_timing)
                fprintf(stderr, "[psacak]   doubling %c-scan h=%llu: <= %u items, %d key bits%s\n", tag,
                        (unsigned long long)h, cnt, KBr + GB,
                        spec ? " (count on the device)" : seg ? " (group-ordered)" : "");
            h = packed ? (uint64_t)P : h << 1;
        }
        uint32_t tri[4];
        PSK_TRY(ctx.read_u32(dcnt - 2, tri, 4));  // the last round's totals (g, s, k, o)
        cnt = tri[2];
        ngroups = tri[3];
    }
    return PSACAK_OK;
}

template <class C>
status_t induce_doubling(Ctx &ctx, const C *text, uint64_t n, const uint32_t *types, const uint32_t *lms,
                         Geom<C> geom, uint64_t nbuckets, InduceMode mode, const uint64_t *sorted_lms, uint64_t n1,
                         uint32_t *cursor, uint32_t *sa, cudaStream_t s) {
    DBuf<uint32_t> R, v0, v1, gA, gB;
    DBuf<uint64_t> k0, k1;
    // group-start tables: indexed by bucket id (round 1) or kept-group ordinal
    const uint64_t gcap = n > nbuckets ? n : nbuckets;
    PSK_TRY(gA.init(ctx, gcap));
    PSK_TRY(gB.init(ctx, gcap));
    PSK_TRY(R.init(ctx, n + 1));
    PSK_TRY(v0.init(ctx, n));
    PSK_TRY(v1.init(ctx, n));
    PSK_TRY(k0.init(ctx, n));
    PSK_TRY(k1.init(ctx, n));
    uint32_t *Wg = (uint32_t *)k1.get(), *Wv = Wg + n;  // the work list (see doubling_rounds)
    PSK_CUDA(cudaMemsetAsync(R.get() + n, 0, sizeof(uint32_t), s));  // the sentinel ranks lowest
    const uint64_t nwords = ceil_div(n, 32);
    if (mode == INDUCE_LMS_SUBSTRINGS) {
        uint64_t g = ceil_div(nwords, 256);
        PSK_PROF_LAUNCH(s, "place_lms", nwords, 0,
                        (k_place_lms_any<C><<<(uint32_t)(g < 8192 ? g : 8192), 256, 0, s>>>(text, nwords, lms, geom,
                                                                                            cursor, R)));
        PSK_LAUNCH_CHECK();
    } else if (n1 > 0) {
        PSK_TRY((ctx.scan<uint32_t, OpMax<uint32_t>>(LastLoad<C>{sorted_lms, n1, geom},
                                                     LastStore<C>{n1, R}, n1,
                                                     (uint32_t *)nullptr, OpMax<uint32_t>(), "scan_last")));
    }
    PSK_TRY((doubling_scan<C, false>(ctx, text, n, types, geom, nbuckets, R, sa, Wg, Wv, k0, v0, k1, v1, gA, gB, s)));
    PSK_TRY((doubling_scan<C, true>(ctx, text, n, types, geom, nbuckets, R, sa, Wg, Wv, k0, v0, k1, v1, gA, gB, s)));
    return PSACAK_OK;
}

// Suffix array of a u32 string directly by prefix doubling (no recursion):
// the items are all positions, grouped by bucket, ranks doubled until every
// suffix is alone.  Rounds = log2 of the longest repeat, so this only pays
// for short strings, where it replaces the remaining recursion levels.
status_t sort_by_doubling(Ctx &ctx, const uint32_t *names, const uint32_t *bheads, uint64_t nbuckets, uint64_t n,
                          uint32_t *sa, cudaStream_t s) {
    DBuf<uint32_t> R, v0, v1, gA, gB;
    DBuf<uint64_t> k0, k1;
    const uint64_t gcap = n > nbuckets ? n : nbuckets;
    PSK_TRY(gA.init(ctx, gcap));
    PSK_TRY(gB.init(ctx, gcap));
    PSK_TRY(R.init(ctx, n + 1));
    PSK_TRY(v0.init(ctx, n));
    PSK_TRY(v1.init(ctx, n));
    PSK_TRY(k0.init(ctx, n));
    PSK_TRY(k1.init(ctx, n));
    uint32_t *Wg = (uint32_t *)k1.get(), *Wv = Wg + n;  // the work list (see doubling_rounds)
    PSK_CUDA(cudaMemsetAsync(R.get() + n, 0, sizeof(uint32_t), s));
    uint64_t gb = ceil_div(nbuckets, 256);
    k_copy_heads<<<(uint32_t)(gb < 4096 ? gb : 4096), 256, 0, s>>>(bheads, nbuckets, gA, ctx.d_scalars, (uint32_t)n);
    PSK_KCOUNT();
    PSK_LAUNCH_CHECK();
    // the first round builds its keys and ranks from the names directly
    return doubling_rounds(ctx, n, nbuckets, (uint32_t)n, ctx.d_scalars, R, sa, Wg, Wv, k0, v0, k1, v1, gA, gB,
                           names, bheads, 'A', s);
}

template status_t induce_doubling<uint8_t>(Ctx &, const uint8_t *, uint64_t, const uint32_t *, const uint32_t *,
                                           Geom<uint8_t>, uint64_t, InduceMode, const uint64_t *, uint64_t, uint32_t *,
                                           uint32_t *, cudaStream_t);
template status_t induce_doubling<uint32_t>(Ctx &, const uint32_t *, uint64_t, const uint32_t *, const uint32_t *,
                                            Geom<uint32_t>, uint64_t, InduceMode, const uint64_t *, uint64_t,
                                            uint32_t *, uint32_t *, cudaStream_t);

}  // namespace psk
