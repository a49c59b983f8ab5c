// induce_bucket.cu -- bucket-ordered induced scans of a byte level.
//
// The reference's scans (src/psacak8.rs:127-190 serially, :201-344 with the
// fetch/induce/flush pipeline of src/pipeline.rs) visit the suffix array slot
// by slot.  Every L-type suffix lands in a bucket at least as large as the
// one being scanned, so once buckets 0..c-1 have been scanned the L part of
// bucket c is complete except for suffixes induced from bucket c itself, and
// those are exactly the runs of equal characters (c0 == c1).  The GPU form
// processes one bucket at a time, with all of the bucket's slots in
// parallel:
//
//  1. chain expansion: the suffixes already in the L part ("seeds", in scan
//     order) are followed by the suffixes that extend them with one more c,
//     then two more, ...  -- breadth-first, which is the order in which the
//     serial scan appends them.  Each seed's run length is measured, the
//     (depth, seed) cells are laid out by a stable radix sort on depth.
//  2. multisplit: the bucket's entries (L part, then its LMS slots) are read
//     in scan order; each entry whose predecessor is L-type in a larger
//     bucket sends that predecessor to the next free slot of its bucket, in
//     scan order (a stable counting scatter with per-bucket cursors -- the
//     reference's bucket pointers), staged through shared memory so writes
//     go out in runs.
//
// The S scan is the mirror image (buckets from 255 down, S parts filled from
// their tails).  No entry needs the reference's left_most clearing: an entry
// induces only when its predecessor has the type being induced, which is
// what the clearing arranges in the serial scan.
#include "ctx.cuh"
#include "induce.cuh"

#include <utility>

namespace psk {

constexpr int MS_BLOCK = 256;
constexpr int MS_IPT = 16;
constexpr int MS_TILE = MS_BLOCK * MS_IPT;
constexpr int MS_WARPS = MS_BLOCK / 32;

// Scan order of one bucket as a map from scan index q to SA slot: segment A
// then segment B, each walked forward (dir > 0) or backward.
struct BucketSeq {
    uint32_t a_start, a_len, b_start, b_len;
    int dir;
    __device__ __forceinline__ uint32_t slot(uint32_t q) const {
        if (q < a_len) return dir > 0 ? a_start + q : a_start - q;
        q -= a_len;
        return dir > 0 ? b_start + q : b_start - q;
    }
    // the same with the direction known at compile time (DIR = dir)
    template <int DIR> __device__ __forceinline__ uint32_t slot_dir(uint32_t q) const {
        const uint32_t s0 = q < a_len ? a_start : b_start;
        const uint32_t qq = q < a_len ? q : q - a_len;
        return DIR > 0 ? s0 + qq : s0 - qq;
    }
};

// ---- placement of the LMS positions --------------------------------------

// LMS-substring mode placement: LMS positions go to the tail of their bucket
// in arbitrary order.  Each CTA walks a contiguous range of 32-position words
// (a warp per word, a lane per position, so the text is read coalesced;
// PL_UNROLL words per warp step so that their loads overlap), counts its LMS
// per character in shared memory, reserves one range per character with a
// single global atomic, then writes into it.
constexpr int PL_BLOCK = 256;
constexpr int PL_WARPS = PL_BLOCK / 32;
constexpr int PL_UNROLL = 4;
__global__ void __launch_bounds__(PL_BLOCK) k_place_lms_any8(const uint8_t *__restrict__ text, uint64_t nwords,
                                                             const uint32_t *__restrict__ lms,
                                                             const ByteGeom *__restrict__ g, uint32_t *cursor,
                                                             uint32_t *sa, uint32_t *wins, uint64_t wchunk) {
    __shared__ uint32_t s_cnt[256], s_base[256], s_tail[256];
    s_cnt[threadIdx.x] = 0;
    s_tail[threadIdx.x] = g->tail[threadIdx.x];
    __syncthreads();
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5, lt = lanemask_lt();
    const uint64_t w0 = (uint64_t)blockIdx.x * wchunk;
    const uint64_t w1 = w0 + wchunk < nwords ? w0 + wchunk : nwords;
    for (int pass = 0; pass < 2; pass++) {
        for (uint64_t wb = w0 + warp; wb < w1; wb += PL_WARPS * PL_UNROLL) {
            uint32_t word[PL_UNROLL], c[PL_UNROLL], pw[PL_UNROLL];
#pragma unroll
            for (int u = 0; u < PL_UNROLL; u++) {
                const uint64_t w = wb + (uint64_t)u * PL_WARPS;
                word[u] = w < w1 ? lms[w] : 0u;
            }
#pragma unroll
            for (int u = 0; u < PL_UNROLL; u++) {
                const uint64_t p = ((wb + (uint64_t)u * PL_WARPS) << 5) + lane;  // LMS positions are > 0
                const bool on = (word[u] >> lane) & 1u;
                c[u] = on ? text[p] : 256u;
                pw[u] = (pass == 1 && on) ? win_fill(text, (uint32_t)p) : 0u;
            }
#pragma unroll
            for (int u = 0; u < PL_UNROLL; u++) {
                if (!word[u]) continue;  // warp-uniform
                const uint32_t cc = c[u];
                const bool on = cc < 256;
                const uint32_t peers = __match_any_sync(FULL_MASK, cc);
                const int leader = __ffs(peers) - 1;
                uint32_t got = 0;
                if (on && (int)lane == leader) got = atomicAdd(&s_cnt[cc], __popc(peers));
                got = __shfl_sync(FULL_MASK, got, leader);
                if (pass == 1 && on) {
                    const uint32_t slot = s_tail[cc] - 1 - (s_base[cc] + got + __popc(peers & lt));
                    sa[slot] = (uint32_t)(((wb + (uint64_t)u * PL_WARPS) << 5) + lane);
                    wins[slot] = pw[u];
                }
            }
        }
        __syncthreads();
        if (pass == 0) {
            uint32_t c = threadIdx.x;
            s_base[c] = s_cnt[c] ? atomicAdd(&cursor[c], s_cnt[c]) : 0u;
            s_cnt[c] = 0;
            __syncthreads();
        }
    }
}

// Final mode placement: the sorted LMS suffixes fill the tail of each
// bucket in order.  Entry i of the list is position | predecessor window
// << 32; its bucket is the one whose LMS range holds i (a binary
// search over the 256 ranges in shared memory), so the text is not read.
__global__ void __launch_bounds__(256) k_place_lms_sorted8(const uint64_t *__restrict__ sorted, uint64_t n1,
                                                           const ByteGeom *__restrict__ g, uint32_t *sa,
                                                           uint32_t *wins) {
    __shared__ uint32_t s_start[256], s_off[256];  // slot of list entry i = s_off[c] + i
    s_start[threadIdx.x] = g->lmsstart[threadIdx.x];
    s_off[threadIdx.x] = g->tail[threadIdx.x] - g->lmscount[threadIdx.x] - g->lmsstart[threadIdx.x];
    __syncthreads();
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n1; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t v = sorted[i];
        // largest c with s_start[c] <= i (empty buckets share the next start)
        uint32_t c = 0;
#pragma unroll
        for (uint32_t step = 128; step > 0; step >>= 1)
            if (s_start[c + step] <= (uint32_t)i) c += step;
        const uint32_t slot = s_off[c] + (uint32_t)i;
        sa[slot] = (uint32_t)v;
        wins[slot] = (uint32_t)(v >> 32);
    }
}

// cursors: L scan starts at the bucket heads, S scan at the tails; the
// sentinel suffix n-1 is the first entry of its bucket (src/psacak8.rs:131-135).
__global__ void k_init_cursors(const ByteGeom *__restrict__ g, const uint8_t *__restrict__ text, uint64_t n,
                               uint32_t *curL, uint32_t *curS, uint32_t *sa, uint32_t *wins) {
    int c = threadIdx.x;
    uint8_t last = text[n - 1];
    curL[c] = g->head[c] + (c == last ? 1u : 0u);
    curS[c] = g->tail[c];
    if (c == 0) {
        sa[g->head[last]] = (uint32_t)(n - 1);
        wins[g->head[last]] = n >= 2 ? win_fill(text, (uint32_t)(n - 1)) : 0u;
    }
}

// ---- chain expansion -----------------------------------------------------
//
// The cells of a part (seed q, depth d = 1..runs[q]) go breadth-first: all
// depth-1 cells in seed order, then depth 2, ...  The cell (q, d) therefore
// lands at  first + C_1 + ... + C_{d-1} + #{q' < q : runs[q'] >= d},  where
// C_d = #{q : runs[q] >= d}.
//
// Step 1, one look-back scan over the seeds: the load measures each seed's
// run (the characters c in front of it; its window holds the first three), the
// scan counts runs >= 1 and >= 2, and the store places every depth-1 cell and
// lists the seeds with runs >= 2 as a sub-problem: seed x - 1 with run r - 1,
// whose cells are exactly the original depths 2, 3, ...  Step 2 solves the
// (much smaller) sub-list with a four-counter scan that places its depths
// 1..CHAIN_DIRECT directly; only deeper cells (long runs of one character,
// such as N-blocks) go through a sort on depth.
constexpr uint32_t CHAIN_DIRECT = 3;
constexpr uint32_t CHAIN_CAP = 4;             // run characters measured inside the seed scan
constexpr uint32_t CHAIN_LONG = 0x80000000u;  // run flag: longer than CHAIN_CAP, not yet measured

struct ChainPair {
    uint32_t c1, c2;
};
__device__ __forceinline__ ChainPair shfl_up_t(ChainPair v, int o) {
    ChainPair r;
    r.c1 = __shfl_up_sync(FULL_MASK, v.c1, o);
    r.c2 = __shfl_up_sync(FULL_MASK, v.c2, o);
    return r;
}
struct OpPair {
    static constexpr int kFields = 2;
    __device__ __forceinline__ static uint32_t field(int, uint32_t a, uint32_t b) { return a + b; }
    __device__ __forceinline__ ChainPair operator()(ChainPair a, ChainPair b) const {
        return ChainPair{a.c1 + b.c1, a.c2 + b.c2};
    }
    __device__ __forceinline__ static ChainPair identity() { return ChainPair{0, 0}; }
};

struct ChainPayload {
    uint32_t x, r;
    uint8_t e;
};
// Seeds in scan order: L part = sa[start + q]; S part = sa[start - q].
struct SeedLoad {
    using Payload = ChainPayload;
    static constexpr int kIPT = 8;
    const uint8_t *text;
    const uint32_t *sa;
    const uint32_t *wins;
    uint32_t start;
    int dir;
    uint8_t c;
    __device__ __forceinline__ ChainPair operator()(uint64_t q, ChainPayload &p) const {
        const uint32_t slot = dir > 0 ? start + (uint32_t)q : start - (uint32_t)q;
        const uint32_t x = sa[slot];
        uint32_t r = 0;
        uint8_t b = 0;
        if (x > 0) {
            const uint32_t w = wins[slot];
            b = (uint8_t)w;
            if (b == c) {
                // measured up to CHAIN_CAP characters here (the window's
                // look-ahead bytes first); a longer run is finished by
                // k_chain_totals over the sub-list, so that no tile waits on
                // a long run (the next tiles' look-back would)
                const uint32_t ahead = w >> 24;
                r = 1;
                while (r < x && r < CHAIN_CAP) {
                    b = r <= ahead ? (uint8_t)(w >> (8 * r)) : text[x - r - 1];
                    if (b != c) break;
                    r++;
                }
                if (r == x) b = 0;
                else if (r == CHAIN_CAP && b == c) r |= CHAIN_LONG;
            }
        }
        p.x = x;
        p.r = r;
        p.e = b;
        const uint32_t rr = r & ~CHAIN_LONG;
        return ChainPair{rr >= 1 ? 1u : 0u, rr >= 2 ? 1u : 0u};
    }
};
struct SeedStore {
    uint32_t *sa;
    uint32_t *wins;
    uint32_t *subx, *subr;
    uint8_t *sube;
    uint32_t first, limit;  // slot of the first cell; C_1
    int dir;
    uint8_t c;
    uint32_t *err;
    __device__ __forceinline__ void operator()(uint64_t, ChainPair ex, ChainPair, const ChainPayload &p) const {
        const uint32_t r = p.r & ~CHAIN_LONG;
        if (r == 0) return;
        if (ex.c1 >= limit) {
            dev_fail(err, DEVERR_RANGE);
            return;
        }
        const uint32_t slot = dir > 0 ? first + ex.c1 : first - ex.c1;
        sa[slot] = p.x - 1;
        wins[slot] = run_win(1, r, c, p.e);
        if (r >= 2) {
            subx[ex.c2] = p.x - 1;
            subr[ex.c2] = (r - 1) | (p.r & CHAIN_LONG);  // a long run's length is finished later
            sube[ex.c2] = p.e;
        }
    }
};

// Per-seed counters of the sub-list scan.
struct ChainCounts {
    uint32_t c1, c2, c3, deep;
};
__device__ __forceinline__ ChainCounts shfl_up_t(ChainCounts v, int o) {
    ChainCounts r;
    r.c1 = __shfl_up_sync(FULL_MASK, v.c1, o);
    r.c2 = __shfl_up_sync(FULL_MASK, v.c2, o);
    r.c3 = __shfl_up_sync(FULL_MASK, v.c3, o);
    r.deep = __shfl_up_sync(FULL_MASK, v.deep, o);
    return r;
}
struct OpChain {
    static constexpr int kFields = 4;
    __device__ __forceinline__ static uint32_t field(int, uint32_t a, uint32_t b) { return a + b; }
    __device__ __forceinline__ ChainCounts operator()(ChainCounts a, ChainCounts b) const {
        return ChainCounts{a.c1 + b.c1, a.c2 + b.c2, a.c3 + b.c3, a.deep + b.deep};
    }
    __device__ __forceinline__ static ChainCounts identity() { return ChainCounts{0, 0, 0, 0}; }
};
__device__ __forceinline__ ChainCounts chain_counts(uint32_t r) {
    return ChainCounts{r >= 1 ? 1u : 0u, r >= 2 ? 1u : 0u, r >= 3 ? 1u : 0u, r > CHAIN_DIRECT ? r - CHAIN_DIRECT : 0u};
}

// Totals of a sub-list: totals[0] = longest run (atomic max), totals[1..4] =
// its ChainCounts sums.  Runs flagged CHAIN_LONG are measured to the end
// first (seed x = xs[q] has at least the flagged length of c in front).
__global__ void __launch_bounds__(256) k_chain_totals(const uint8_t *__restrict__ text, const uint32_t *__restrict__ xs,
                                                      uint32_t *runs, uint8_t *endc, uint8_t c, uint32_t m,
                                                      uint32_t *totals) {
    __shared__ uint32_t s_red[8][5];
    uint32_t mx = 0;
    ChainCounts acc{0, 0, 0, 0};
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < m; q += gridDim.x * blockDim.x) {
        uint32_t r = runs[q];
        if (r & CHAIN_LONG) {
            const uint32_t x = xs[q];
            r &= ~CHAIN_LONG;
            uint8_t b = c;
            while (r < x && (b = text[x - r - 1]) == c) r++;
            if (r == x) b = 0;
            runs[q] = r;
            endc[q] = b;
        }
        mx = r > mx ? r : mx;
        acc = OpChain()(acc, chain_counts(r));
    }
    for (int o = 16; o > 0; o >>= 1) {
        uint32_t t = __shfl_down_sync(FULL_MASK, mx, o);
        mx = t > mx ? t : mx;
        acc.c1 += __shfl_down_sync(FULL_MASK, acc.c1, o);
        acc.c2 += __shfl_down_sync(FULL_MASK, acc.c2, o);
        acc.c3 += __shfl_down_sync(FULL_MASK, acc.c3, o);
        acc.deep += __shfl_down_sync(FULL_MASK, acc.deep, o);
    }
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
        s_red[w][0] = mx;
        s_red[w][1] = acc.c1;
        s_red[w][2] = acc.c2;
        s_red[w][3] = acc.c3;
        s_red[w][4] = acc.deep;
    }
    __syncthreads();
    if (threadIdx.x < 5) {
        uint32_t v = 0;
        for (int ww = 0; ww < (int)(blockDim.x >> 5); ww++) {
            const uint32_t t = s_red[ww][threadIdx.x];
            v = threadIdx.x == 0 ? (t > v ? t : v) : v + t;
        }
        if (v) {
            if (threadIdx.x == 0) atomicMax(&totals[0], v);
            else atomicAdd(&totals[threadIdx.x], v);
        }
    }
}

// Sub-list scan: per seed its ChainCounts; the store writes the seed's cells
// of depth 1..3 (entry and predecessor window) and the offset of its deep
// cells.
struct ChainLoad {
    using Payload = ChainPayload;
    static constexpr int kIPT = 6;
    const uint32_t *xs;
    const uint32_t *runs;
    const uint8_t *endc;
    __device__ __forceinline__ ChainCounts operator()(uint64_t q, ChainPayload &p) const {
        p.x = xs[q];
        p.r = runs[q];
        p.e = endc[q];
        return chain_counts(p.r);
    }
};
struct ChainStore {
    uint32_t *sa;
    uint32_t *wins;
    uint32_t *deep_off;  // null when the sub-list has no deep cells
    uint32_t first;      // slot of the first cell
    uint32_t base2, base3;  // C_1 and C_1 + C_2
    uint32_t limit;         // cells of depth <= 3 (C_1 + C_2 + C_3)
    int dir;
    uint8_t c;
    uint32_t *err;
    __device__ __forceinline__ void put(uint32_t k, uint32_t val, uint32_t w) const {
        if (k >= limit) {
            dev_fail(err, DEVERR_RANGE);
            return;
        }
        const uint32_t slot = dir > 0 ? first + k : first - k;
        sa[slot] = val;
        wins[slot] = w;
    }
    __device__ __forceinline__ void operator()(uint64_t q, ChainCounts ex, ChainCounts, const ChainPayload &p) const {
        const uint32_t r = p.r;
        if (r >= 1) put(ex.c1, p.x - 1, run_win(1, r, c, p.e));
        if (r >= 2) put(base2 + ex.c2, p.x - 2, run_win(2, r, c, p.e));
        if (r >= 3) put(base3 + ex.c3, p.x - 3, run_win(3, r, c, p.e));
        if (deep_off) deep_off[q] = ex.deep;
    }
};

// Deep cell q (row-major over sub-list seeds, depths > 3) -> (depth - 3,
// value (seed - depth) | the window of that suffix << 32).
__global__ void k_expand_deep(const uint32_t *__restrict__ xs, uint32_t nseeds, const uint32_t *__restrict__ off,
                              const uint32_t *__restrict__ runs, const uint8_t *__restrict__ endc, uint8_t c,
                              uint32_t ncells, uint32_t *keys, uint64_t *vals) {
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < ncells; q += gridDim.x * blockDim.x) {
        // last seed s with off[s] <= q (seeds without deep cells share the next one's offset)
        uint32_t lo = 0, hi = nseeds - 1;
        while (lo < hi) {
            uint32_t mid = (lo + hi + 1) >> 1;
            if (off[mid] <= q) lo = mid;
            else hi = mid - 1;
        }
        uint32_t dd = q - off[lo] + 1;
        uint32_t d = dd + CHAIN_DIRECT;
        uint32_t x = xs[lo];
        keys[q] = dd;
        vals[q] = (uint64_t)(x - d) | (uint64_t)run_win(d, runs[lo], c, endc[lo]) << 32;
    }
}

__global__ void k_place_cells(const uint64_t *__restrict__ vals, uint32_t ncells, uint32_t first, int dir,
                              uint32_t *sa, uint32_t *wins) {
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < ncells; q += gridDim.x * blockDim.x) {
        uint32_t slot = dir > 0 ? first + q : first - q;
        uint64_t v = vals[q];
        sa[slot] = (uint32_t)v;
        wins[slot] = (uint32_t)(v >> 32);
    }
}

// ---- multisplit ----------------------------------------------------------

// The bucket's entries in scan order; an entry x induces its predecessor
// x-1 when that character c0 = text[x-1] is larger (L scan) or smaller (S
// scan) than the bucket's character c, and the predecessor goes to slot
// cur_in[c0] + rank (L) or cur_in[c0] - 1 - rank (S) -- the reference's
// bucket-pointer increment/decrement, in scan order.
//
// In the LMS-substring round the S scan also extracts the sorted LMS
// substrings: an S-part entry whose predecessor is larger is an LMS
// suffix (the reference keeps exactly these after its left_most clearing
// and compacts them, src/psacak8.rs:35).  They get the spare digit 255
// (never an S-scan target: targets are smaller than c) and go to the
// bucket's range of the sorted LMS list, highest first.
constexpr uint32_t LMS_DIGIT = 255;

// Items carry the target position (low 32 bits) and its predecessor window
// (high 32 bits, win_next), stored beside the entry in wins: the decision
// and the target bucket come from the window, and the text is read only
// when an induced suffix's window has no look-ahead byte left.
template <bool LSCAN> struct BucketPolicy {
    using Item = uint64_t;
    // 4 CTAs per SM (64 registers; the compiler keeps a few values in local
    // memory): the scatter waits on its loads and on the look-back, and the
    // fourth CTA measured 31.1 ms against 33.9 ms at 3 CTAs and 80 registers
    // for the 1 GiB build's scatters.
    static constexpr int kMinBlocks = 4;
    const uint8_t *text;
    uint32_t *sa;
    BucketSeq seq;
    uint32_t c;
    const uint32_t *cur_in;
    uint32_t *cur_out;
    unsigned long long *induced;
    uint64_t n;
    uint32_t *err;
    uint32_t *lms_out;   // S scan, LMS-substring round: sorted LMS list (else null)
    uint32_t lms_hi;     // index of this bucket's last entry in that list
    uint32_t lms_cap;    // entries of the list
    uint32_t *wins;      // wins[slot] = predecessor window of sa[slot] for every placed entry
    uint32_t targets[8];  // bit d: digit d can receive entries (buckets with a part of the scan's type)
    __device__ __forceinline__ bool active(uint32_t d) const { return (targets[d >> 5] >> (d & 31)) & 1u; }
    struct Pre {
        uint32_t x;
        uint32_t w;
    };
    __device__ __forceinline__ void pre(uint64_t i, Pre &p) const {
        const uint32_t slot = seq.template slot_dir<LSCAN ? 1 : -1>((uint32_t)i);
        p.x = sa[slot];
        p.w = wins[slot];
    }
    __device__ __forceinline__ void load(uint64_t i, const Pre &p, Item &it, uint32_t &d) const {
        const uint32_t x = p.x;
        d = 256;
        if (x > 0) {
            const uint32_t c0 = p.w & 0xFFu;
            if (LSCAN ? c0 > c : c0 < c) {
                d = c0;
                it = (uint64_t)(x - 1) | (uint64_t)win_next(p.w, text, x) << 32;
            } else if (!LSCAN && lms_out && c0 > c && i < seq.a_len) {
                d = LMS_DIGIT;
                it = x;
            }
        }
    }
    // rank r of digit d goes to cur_in[d] + r (L), cur_in[d] - 1 - r (S) or,
    // for the extracted LMS suffixes, lms_hi - r
    static constexpr int kOutSign = LSCAN ? 1 : -1;
    __device__ __forceinline__ uint64_t out0(uint32_t d) const {
        if (!LSCAN && lms_out && d == LMS_DIGIT) return (uint64_t)lms_hi;
        return LSCAN ? (uint64_t)cur_in[d] : (uint64_t)cur_in[d] - 1;
    }
    __device__ __forceinline__ void store(uint64_t idx, const Item &it, uint32_t d) const {
        if (!LSCAN && lms_out && d == LMS_DIGIT) {
            if (idx < lms_cap) lms_out[idx] = (uint32_t)it;
            else dev_fail(err, DEVERR_RANGE);
            return;
        }
        if (idx < n) {
            sa[idx] = (uint32_t)it;
            wins[idx] = (uint32_t)(it >> 32);
        } else {
            dev_fail(err, DEVERR_RANGE);
        }
    }
    __device__ __forceinline__ void finish(uint32_t d, uint32_t total) const {
        if (!LSCAN && lms_out && d == LMS_DIGIT) {
            cur_out[d] = cur_in[d];
            if (total) atomicAdd(induced + 1, (unsigned long long)total);
            return;
        }
        cur_out[d] = LSCAN ? cur_in[d] + total : cur_in[d] - total;
        if (total) atomicAdd(induced, (unsigned long long)total);
    }
};

static inline uint32_t grid_cap(uint64_t n, uint32_t cap) {
    uint64_t g = ceil_div(n ? n : 1, 256);
    return (uint32_t)(g < cap ? g : cap);
}

// Chain expansion of one bucket part.  `start` is the slot of the first
// seed in scan order, `nseeds` the seeds present, `part` the full size of
// the part; fills the remaining part - nseeds slots.
static status_t expand_chains(Ctx &ctx, const uint8_t *text, uint32_t *sa, uint32_t start, int dir, uint32_t nseeds,
                              uint32_t part, uint8_t c, uint32_t *subx, uint32_t *subr, uint8_t *sube, uint32_t *off,
                              uint32_t *wins, cudaStream_t s) {
    if (part == 0) return PSACAK_OK;
    if (nseeds == 0 || nseeds > part)
        return set_error(PSACAK_EINTERNAL, "bucket %u: %u seeds for a part of %u", c, nseeds, part);
    if (nseeds == part) return PSACAK_OK;  // nothing chained: no seed has c in front of it
    const uint32_t first = dir > 0 ? start + nseeds : start - nseeds;
    const uint32_t cells = part - nseeds;
    // step 1: depth-1 cells and the sub-list of runs >= 2
    ChainPair *d_pair = (ChainPair *)(ctx.d_scalars + 24);
    PSK_TRY((ctx.scan<ChainPair, OpPair>(SeedLoad{text, sa, wins, start, dir, c},
                                         SeedStore{sa, wins, subx, subr, sube, first, cells, dir, c, ctx.d_err}, nseeds,
                                         d_pair, OpPair(), "chain_seeds")));
    uint32_t h[5];
    PSK_TRY(ctx.read_u32((const uint32_t *)d_pair, h, 2));
    const uint32_t C1 = h[0], m = h[1];
    if (m == 0) {
        if (C1 != cells) return set_error(PSACAK_EINTERNAL, "bucket %u: %u chained != %u", c, C1, cells);
        return PSACAK_OK;
    }
    // step 2: the sub-list (seeds x - 1 with runs r - 1) from slot first + C1
    uint32_t *d_tot = ctx.d_scalars + 26;  // [max run, C'_1, C'_2, C'_3, deep cells]
    PSK_CUDA(cudaMemsetAsync(d_tot, 0, 5 * sizeof(uint32_t), s));
    PSK_PROF_LAUNCH(s, "chain_totals", m, 0,
                    (k_chain_totals<<<grid_cap(m, 1184), 256, 0, s>>>(text, subx, subr, sube, c, m, d_tot)));
    PSK_TRY(ctx.read_u32(d_tot, h, 5));
    const uint32_t maxrun = h[0], D1 = h[1], D2 = h[2], D3 = h[3], ndeep = h[4];
    if ((uint64_t)C1 + D1 + D2 + D3 + ndeep != cells || D1 != m)
        return set_error(PSACAK_EINTERNAL, "bucket %u: %u + %u + %u + %u + %u chained != %u", c, C1, D1, D2, D3, ndeep,
                         cells);
    const uint32_t sfirst = dir > 0 ? first + C1 : first - C1;
    const uint32_t direct = D1 + D2 + D3;
    PSK_TRY((ctx.scan<ChainCounts, OpChain>(ChainLoad{subx, subr, sube},
                                            ChainStore{sa, wins, ndeep ? off : nullptr, sfirst, D1, D1 + D2, direct, dir,
                                                       c, ctx.d_err},
                                            m, (ChainCounts *)nullptr, OpChain(), "chain_place")));
    if (ndeep == 0) return PSACAK_OK;
    // step 3: cells deeper than the direct depths, sorted on depth (buffers
    // sized to this part's deep cells)
    DBuf<uint32_t> k0, k1;
    DBuf<uint64_t> v0, v1;
    PSK_TRY(k0.init(ctx, ndeep));
    PSK_TRY(k1.init(ctx, ndeep));
    PSK_TRY(v0.init(ctx, ndeep));
    PSK_TRY(v1.init(ctx, ndeep));
    PSK_PROF_LAUNCH(s, "chain_deep", ndeep, 0,
                    (k_expand_deep<<<grid_cap(ndeep, 8192), 256, 0, s>>>(subx, m, off, subr, sube, c, ndeep, k0,
                                                                           v0)));
    PSK_LAUNCH_CHECK();
    int in1 = 0;
    PSK_TRY((ctx.radix_sort<uint32_t, uint64_t>(k0.get(), v0.get(), k1.get(), v1.get(), ndeep, 0,
                                                bitlen(maxrun - CHAIN_DIRECT), &in1)));
    const uint32_t dfirst = dir > 0 ? sfirst + direct : sfirst - direct;
    PSK_PROF_LAUNCH(s, "chain_place_deep", ndeep, 13ull * ndeep,
                    (k_place_cells<<<grid_cap(ndeep, 8192), 256, 0, s>>>(in1 ? v1.get() : v0.get(), ndeep, dfirst, dir,
                                                                          sa, wins)));
    PSK_LAUNCH_CHECK();
    return PSACAK_OK;
}

// Multisplit of one bucket; the cursors move from cur[0..256) to
// cur[256..512) (the caller swaps the halves afterwards).
// `hg`: the level's bucket geometry, which bounds the digits an entry of
// bucket c can send: larger buckets with an L part (L scan), smaller ones
// with an S part (S scan), and the extraction digit.
template <bool LSCAN>
static status_t multisplit(Ctx &ctx, const uint8_t *text, uint32_t *sa, uint64_t n, BucketSeq seq, uint8_t c,
                           const uint32_t *cur_in, uint32_t *cur_out, uint32_t *wins, cudaStream_t s,
                           const ByteGeom &hg, uint32_t *lms_out = nullptr, uint32_t lms_hi = 0,
                           uint32_t lms_cap = 0) {
    uint32_t nitems = seq.a_len + seq.b_len;
    if (nitems == 0) {
        k_copy_words<<<1, 256, 0, s>>>(cur_in, cur_out, 256);
        PSK_KCOUNT();
        PSK_LAUNCH_CHECK();
        return PSACAK_OK;
    }
    PSK_TRY(ctx.ensure_onesweep(ceil_div(nitems, 8 * OS_BLOCK) + 1));
    BucketPolicy<LSCAN> pol{text, sa, seq, c, cur_in, cur_out, ctx.d_induced, n, ctx.d_err, lms_out, lms_hi, lms_cap,
                            wins, {}};
    for (uint32_t d = 0; d < 256; d++) {
        const bool target = LSCAN ? (d > c && hg.lcount[d] > 0) : (d < c && hg.scount[d] > 0);
        if (target || (!LSCAN && lms_out && d == LMS_DIGIT)) pol.targets[d >> 5] |= 1u << (d & 31);
    }
    // algorithmic bytes: each entry and its window read (8); inducing
    // entries write entry + window (8, added from the device count) and read
    // the text byte in front of their target (1, with it).
    return onesweep_ipt<BucketPolicy<LSCAN>>(pol, nitems, ctx.tile_ipt(), ctx.os, ctx.d_err, s, "induce_scatter",
                                              8ull * nitems);
}

status_t induce_bucket8(Ctx &ctx, const uint8_t *text, uint64_t n, const uint32_t *lms, const ByteGeom &hg,
                        const ByteGeom *dgeom, InduceMode mode, const uint64_t *sorted_win, uint64_t n1,
                        uint32_t *sa, cudaStream_t s, uint32_t *lms_out) {
    uint32_t maxpart = 1, maxbucket = 1;
    for (int c = 0; c < 256; c++) {
        uint32_t cnt = hg.tail[c] - hg.head[c];
        maxbucket = cnt > maxbucket ? cnt : maxbucket;
        maxpart = hg.lcount[c] > maxpart ? hg.lcount[c] : maxpart;
        maxpart = hg.scount[c] > maxpart ? hg.scount[c] : maxpart;
    }
    DBuf<uint32_t> cur, cur2, runs, off, subx;
    DBuf<uint8_t> endc;
    DBuf<uint32_t> wins;
    PSK_TRY(cur.init(ctx, 512));
    PSK_TRY(cur2.init(ctx, 512));
    PSK_TRY(endc.init(ctx, maxpart));
    PSK_TRY(wins.init(ctx, n));
    PSK_TRY(runs.init(ctx, maxpart));
    PSK_TRY(subx.init(ctx, maxpart));
    PSK_TRY(off.init(ctx, maxpart));
    uint32_t *curL = cur.get(), *curS = cur.get() + 256;
    uint32_t *alt = cur2.get();

    // LMS positions at the bucket tails (put_lmscharacters / put_lmssuffixes).
    if (mode == INDUCE_LMS_SUBSTRINGS) {
        PSK_CUDA(cudaMemsetAsync(curL, 0, 256 * sizeof(uint32_t), s));
        const uint64_t nwords = ceil_div(n, 32);
        const uint64_t G = ceil_div(nwords, 2048) < 4ull * ctx.scan_ctas ? ceil_div(nwords, 2048) : 4ull * ctx.scan_ctas;
        const uint64_t wchunk = ceil_div(nwords, G);
        PSK_PROF_LAUNCH(s, "place_lms", nwords, 0,
                        (k_place_lms_any8<<<(uint32_t)G, PL_BLOCK, 0, s>>>(text, nwords, lms, dgeom, curL, sa, wins.get(),
                                                                         wchunk)));
    } else if (n1 > 0) {
        PSK_PROF_LAUNCH(s, "place_lms", n1, 0,
                        (k_place_lms_sorted8<<<grid_cap(n1, 8192), 256, 0, s>>>(sorted_win, n1, dgeom, sa,
                                                                                  wins.get())));
    }
    k_init_cursors<<<1, 256, 0, s>>>(dgeom, text, n, curL, curS, sa, wins.get());
    PSK_KCOUNT();
    PSK_LAUNCH_CHECK();

    // The final SA goes to the host while the scans run: a bucket's L part
    // is final once its chains are expanded in the L scan (later writes go
    // to larger buckets or to S parts), its S part once its chains are
    // expanded in the S scan.
    const bool sink = mode == INDUCE_FINAL && ctx.sink_host && sa == ctx.sink_dev;
    // L scan: buckets in increasing order.
    for (int c = 0; c < 256; c++) {
        const uint32_t head = hg.head[c], tail = hg.tail[c];
        if (tail == head) continue;
        const uint32_t lc = hg.lcount[c], lmsc = hg.lmscount[c];
        if (lc > 0) {
            uint32_t cl = 0;
            PSK_TRY(ctx.read_u32(curL + c, &cl));
            PSK_TRY(expand_chains(ctx, text, sa, head, +1, cl - head, lc, (uint8_t)c, subx, runs, endc, off, wins, s));
            if (sink) PSK_TRY(ctx.sink_part(head, lc));
        }
        BucketSeq seq{head, lc, tail - lmsc, lmsc, +1};
        PSK_TRY(multisplit<true>(ctx, text, sa, n, seq, (uint8_t)c, curL, alt, wins, s, hg));
        std::swap(curL, alt);
    }
    alt = cur2.get() + 256;
    // S scan: buckets in decreasing order, S parts filled from their tails.
    for (int c = 255; c >= 0; c--) {
        const uint32_t head = hg.head[c], tail = hg.tail[c];
        if (tail == head) continue;
        const uint32_t lc = hg.lcount[c], sc = hg.scount[c];
        if (sc > 0) {
            uint32_t cs = 0;
            PSK_TRY(ctx.read_u32(curS + c, &cs));
            PSK_TRY(expand_chains(ctx, text, sa, tail - 1, -1, tail - cs, sc, (uint8_t)c, subx, runs, endc, off, wins,
                                  s));
            if (sink) PSK_TRY(ctx.sink_part(head + lc, sc));
        }
        BucketSeq seq{tail - 1, sc, head + lc - 1, lc, -1};
        const bool extract = mode == INDUCE_LMS_SUBSTRINGS && lms_out && hg.lmscount[c] > 0;
        PSK_TRY(multisplit<false>(ctx, text, sa, n, seq, (uint8_t)c, curS, alt, wins, s, hg,
                                  extract ? lms_out : nullptr, hg.lmsstart[c] + hg.lmscount[c] - 1, (uint32_t)n1));
        std::swap(curS, alt);
    }
    if (sink) ctx.sink_done = true;
    return PSACAK_OK;
}

}  // namespace psk
