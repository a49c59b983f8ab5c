// induce.cuh -- induced L-/S-scans of one level.
#pragma once

#include "level.cuh"

namespace psk {

struct Ctx;

// Geometry of the buckets of a byte level (SA-position space), uploaded from
// the host after the level histogram is read back.
struct ByteGeom {
    uint32_t head[256];    // first SA slot of bucket c
    uint32_t tail[256];    // one past the last slot of bucket c
    uint32_t lcount[256];  // L-type suffixes of bucket c
    uint32_t scount[256];  // S-type suffixes of bucket c
    uint32_t lmscount[256];
    uint32_t lmsstart[256];  // first index of bucket c in the sorted LMS list
};

// Geometry of a translated integer level: every L-type symbol is its bucket
// head and every S-type symbol is its bucket tail - 1 (the reference's
// translate, src/naming.rs:263-274).  scnt[v] = S-type count of the bucket
// whose tail - 1 is v.
struct WordGeom {
    const uint32_t *scnt;
};

template <class C> struct Geom;
template <> struct Geom<uint8_t> {
    const ByteGeom *g;
    __device__ __forceinline__ uint32_t name(uint64_t, uint8_t c) const { return c; }
    // first slot of the L (S) part of the bucket with dense id c
    __device__ __forceinline__ uint32_t lstart_of(uint32_t c) const { return g->head[c]; }
    __device__ __forceinline__ uint32_t sstart_of(uint32_t c) const { return g->tail[c] - g->scount[c]; }
    __device__ __forceinline__ uint32_t lgroup(uint8_t c) const { return g->head[c]; }
    __device__ __forceinline__ uint32_t sgroup(uint8_t c) const { return g->tail[c] - g->scount[c]; }
    __device__ __forceinline__ uint32_t tail(uint8_t c) const { return g->tail[c]; }
    __device__ __forceinline__ uint32_t bucket(uint8_t c) const { return c; }
};
template <> struct Geom<uint32_t> {
    const uint32_t *scnt;
    const uint32_t *names;  // dense bucket id of every position
    const uint32_t *heads;  // bucket boundaries by dense id (nbuckets + 1 entries)
    __device__ __forceinline__ uint32_t name(uint64_t j, uint32_t) const { return names[j]; }
    __device__ __forceinline__ uint32_t lstart_of(uint32_t c) const { return heads[c]; }
    __device__ __forceinline__ uint32_t sstart_of(uint32_t c) const {
        uint32_t tail = heads[c + 1];
        return tail - scnt[tail - 1];
    }
    __device__ __forceinline__ uint32_t lgroup(uint32_t v) const { return v; }
    __device__ __forceinline__ uint32_t sgroup(uint32_t v) const { return v + 1 - scnt[v]; }
    __device__ __forceinline__ uint32_t tail(uint32_t v) const { return v + 1; }
    __device__ __forceinline__ uint32_t bucket(uint32_t v) const { return v; }
};

enum InduceMode { INDUCE_LMS_SUBSTRINGS = 0, INDUCE_FINAL = 1 };

// Chain-doubling induced sort.  In INDUCE_LMS_SUBSTRINGS mode the LMS
// positions start in arbitrary order at their bucket tails; in INDUCE_FINAL
// mode `sorted_lms` (n1 entries, ascending suffix order, each position |
// its symbol << 32, permute_lms_sym) gives their order.
// Writes every SA slot.  `cursor` is n (u32 levels) or 256 (byte levels)
// zeroed uint32 used to place LMS positions in the first mode.
// `nbuckets` = number of distinct symbols (dense ids 0..nbuckets-1).
template <class C>
status_t induce_doubling(Ctx &ctx, const C *text, uint64_t n, const uint32_t *types, const uint32_t *lms,
                         Geom<C> geom, uint64_t nbuckets, InduceMode mode, const uint64_t *sorted_lms, uint64_t n1,
                         uint32_t *cursor, uint32_t *sa, cudaStream_t s);

// Suffix array of a u32 level directly by prefix doubling (recursion finisher).
status_t sort_by_doubling(Ctx &ctx, const uint32_t *names, const uint32_t *bheads, uint64_t nbuckets, uint64_t n,
                          uint32_t *sa, cudaStream_t s);

// Bucket-ordered induced sort of a byte level (the reference's induce scan
// processed one bucket at a time): every bucket's L part is completed and
// then scattered to the higher buckets in scan order; the S scan mirrors it.
// In INDUCE_LMS_SUBSTRINGS mode with `lms_out` set, the S scan also writes the
// n1 LMS positions in sorted-substring order to lms_out.
// In INDUCE_FINAL mode `sorted_win` lists the sorted LMS suffixes as
// position | predecessor window << 32 (win_fill).
status_t induce_bucket8(Ctx &ctx, const uint8_t *text, uint64_t n, const uint32_t *lms,
                        const ByteGeom &hgeom, const ByteGeom *dgeom, InduceMode mode, const uint64_t *sorted_win,
                        uint64_t n1, uint32_t *sa, cudaStream_t s, uint32_t *lms_out = nullptr);

}  // namespace psk
