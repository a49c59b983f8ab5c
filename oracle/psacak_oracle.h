/*
 * psacak_oracle.h -- CPU restatement of hucsmn/psacak's serial pSACAK path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the parity checker for the
 * B200 builder: only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg may load it.  The product path (psacak_b200) never calls it.
 *
 * Every function follows the serial (non-pipelined) path of the reference
 * crate; the file:line of the reference item each function restates is given
 * beside its definition in psacak_oracle.c.  The reference's own parallel
 * paths are proven equal to these serial paths by the reference's tests
 * (src/psacak8.rs:536-590, src/psacak32.rs:854-910, src/naming.rs:438-471).
 */
#ifndef PSACAK_ORACLE_H
#define PSACAK_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Per-recursion-level record.  level 0 is the input text.  m = level length,
 * n_lms = number of LMS positions, k = number of distinct LMS-substring
 * names, hash = order-dependent hash of the translated reduced string that
 * the level hands to the next one (0 when k == n_lms and no recursion). */
typedef struct {
    uint32_t level;
    uint32_t width;   /* symbol width in bytes: 1 (u8) or 4 (u32) */
    uint64_t m;
    uint64_t n_lms;
    uint64_t k;
    uint64_t hash;
} oracle_level;

/* psacak / psacak_inplace (src/lib.rs:64-82): SA of `text` without the
 * sentinel.  Returns 0, or -1 when n >= 2^32-1.  `trace` (nullable) receives
 * up to `max_levels` records; the number of levels is returned in *n_levels. */
int oracle_psacak8(const uint8_t *text, uint64_t n, uint32_t *sa,
                   oracle_level *trace, uint32_t max_levels, uint32_t *n_levels);

/* Integer-alphabet entry: the reference's test helper calc_psacak32
 * (src/psacak32.rs:873-881): translate_sample then psacak32, or saca_tiny
 * when the number of distinct symbols is >= n.  Returns 0, or -1 when
 * n > 2^31-1. */
int oracle_psacak32(const uint32_t *text, uint64_t n, uint32_t *sa,
                    oracle_level *trace, uint32_t max_levels, uint32_t *n_levels);

/* psacak8 with the reference's pipelined induced scans (src/pipeline.rs,
 * src/psacak8.rs:201-344) on `threads` threads for texts of two blocks
 * (2 x 128Ki) and more: the all-core CPU baseline.  Same result as
 * oracle_psacak8.  Returns 0, or -1 when n >= 2^32-1. */
int oracle_psacak8_par(const uint8_t *text, uint64_t n, uint32_t *sa, uint32_t threads);

/* Derived arrays (no counterpart in the reference): LCP by Kasai et al.
 * (lcp[0] = 0), BWT in libdivsufsort's divbwt convention (returns the
 * primary index; bwt has n bytes). */
void oracle_lcp8(const uint8_t *text, uint64_t n, const uint32_t *sa, uint32_t *lcp);
void oracle_lcp32(const uint32_t *text, uint64_t n, const uint32_t *sa, uint32_t *lcp);
uint64_t oracle_bwt8(const uint8_t *text, uint64_t n, const uint32_t *sa, uint8_t *bwt);

/* Suffix-array indices [lo, hi) of the suffixes that start with pat[0, m),
 * by binary search on the suffix array (checks the FM-index search). */
void oracle_sa_range8(const uint8_t *text, uint64_t n, const uint32_t *sa, const uint8_t *pat, uint64_t m,
                      uint64_t *lo, uint64_t *hi);

/* saca_tiny (src/common.rs:13-25): naive comparison sort of the suffixes. */
void oracle_saca_tiny8(const uint8_t *text, uint64_t n, uint32_t *sa);
void oracle_saca_tiny32(const uint32_t *text, uint64_t n, uint32_t *sa);

/* The translate_sample mapping alone (src/psacak32.rs:912-943).  Returns 1
 * and fills `out` when distinct < n, else returns 0. */
int oracle_translate_sample(const uint32_t *text, uint64_t n, uint32_t *out);

/* Burkhardt-Kaerkkaeinen O(n) suffix-array check (CPM 2003): `sa` is a
 * permutation and adjacent suffixes are in order.  Returns 1 if correct. */
int oracle_check_sa8(const uint8_t *text, uint64_t n, const uint32_t *sa);
int oracle_check_sa32(const uint32_t *text, uint64_t n, const uint32_t *sa);

/* Order-dependent hash used for level traces: sum over i of
 * mix64(((uint64)i << 32) ^ v[i]) modulo 2^64. */
uint64_t oracle_hash_u32(const uint32_t *v, uint64_t n);

/* Reduced string of level 0 of psacak8 (after naming and translate).
 * Writes up to `cap` symbols, returns the reduced length n_lms and stores the
 * name count in *k. */
uint64_t oracle_reduced8(const uint8_t *text, uint64_t n, uint32_t *out,
                         uint64_t cap, uint64_t *k);

#ifdef __cplusplus
}
#endif
#endif
