/*
 * psacak_b200_debug.h -- internal stages of the builder, exported for the
 * stage-by-stage parity tests and for tuning.  Device pointers; every call
 * synchronises the context stream before returning.
 *
 * None of these has a counterpart in hucsmn/psacak's public API; each names
 * the reference item whose output it exposes.
 */
#ifndef PSACAK_B200_DEBUG_H
#define PSACAK_B200_DEBUG_H

#include "psacak_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Stable LSD radix sort of (key, value) pairs on bits [begin_bit, end_bit),
 * in place.  The primitive under every sort of the chain-doubling scan. */
PSACAK_API int psacak_debug_radix_sort_u64(psacak_ctx *ctx, uint64_t *d_keys, uint32_t *d_vals, uint64_t n,
                                           int begin_bit, int end_bit);
PSACAK_API int psacak_debug_radix_sort_u32(psacak_ctx *ctx, uint32_t *d_keys, uint32_t *d_vals, uint64_t n,
                                           int begin_bit, int end_bit);

/* Exclusive prefix sum of n uint32 (the chunked scan used everywhere). */
PSACAK_API int psacak_debug_exclusive_sum(psacak_ctx *ctx, const uint32_t *d_in, uint32_t *d_out, uint64_t n);

/* L/S types and LMS flags of a text (width 1 or 4) as packed bitmaps of
 * ceil(n/32) words: the reference's foreach_typedchars
 * (src/common.rs:43-68) and foreach_lmschars (src/common.rs:101-117). */
PSACAK_API int psacak_debug_types(psacak_ctx *ctx, const void *d_text, uint64_t n, int width, uint32_t *d_types,
                                  uint32_t *d_lms);

/* Level 0 of psacak8 up to the reduced string: typing, LMS-substring sort,
 * naming and translation (src/psacak8.rs:28-36, src/naming.rs:20-93,
 * :263-274).  Writes the translated reduced string (n_lms entries, capacity
 * `cap`) and returns n_lms and the name count k. */
PSACAK_API int psacak_debug_reduced8(psacak_ctx *ctx, const uint8_t *d_text, uint64_t n, uint32_t *d_red,
                                     uint64_t cap, uint64_t *n_lms, uint64_t *k,
                                     const psacak_schedule *sched);

/* Limits for the failure-path tests.  spin_limit: polls after which every
 * bounded device wait of the calls on `ctx` gives up and the call returns
 * PSACAK_ETIMEOUT (0 = the compiled limits, 2^22..2^24 polls; at most
 * 2^31).  workspace_cap: most device workspace bytes a build on `ctx` may
 * hold at once; a larger request fails with PSACAK_ENOMEM, as a failed
 * allocation does (0 = no cap). */
PSACAK_API int psacak_debug_set_limits(psacak_ctx *ctx, uint32_t spin_limit, uint64_t workspace_cap);

/* Exclusive sum of n words of d_in into d_out by the single-pass look-back
 * scan of every build, launched without its first tile: that tile's status
 * words are never published, so the look-back of every other tile waits on
 * a flag that nothing sets until its wait runs out.  Returns
 * PSACAK_ETIMEOUT (after the bounded waits; keep the spin limit short) and
 * leaves the context usable.  n must span at least two tiles (> 4096). */
PSACAK_API int psacak_debug_stalled_scan(psacak_ctx *ctx, const uint32_t *d_in, uint32_t *d_out, uint64_t n);

#ifdef __cplusplus
}
#endif
#endif
