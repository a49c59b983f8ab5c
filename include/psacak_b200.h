/*
 * psacak_b200.h -- C ABI of the B200 suffix-array builder.
 *
 * The builder keeps hucsmn/psacak's method (SACA-K L/S typing, LMS
 * placement, induced L-/S-scans, LMS-substring naming, recursion on the
 * reduced u32 string, final induction) and runs it as sm_100a CUDA kernels.
 * Every SA it returns is the suffix array of the input without the sentinel
 * position, exactly as the reference's src/lib.rs:30-43 documents; a text has
 * a single such array, so the output is bit-for-bit the reference's.
 *
 * All entry points return PSACAK_OK (0) or a negative PSACAK_E* status and
 * never abort the process; psacak_last_error_string() describes the last
 * failure on the calling thread.
 */
#ifndef PSACAK_B200_H
#define PSACAK_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define PSACAK_API __attribute__((visibility("default")))
#else
#define PSACAK_API
#endif

#define PSACAK_OK 0
#define PSACAK_EINVAL (-1)    /* null pointer, length limit, bad argument */
#define PSACAK_ENOMEM (-2)    /* device or pinned host allocation failed */
#define PSACAK_ECUDA (-3)     /* a CUDA runtime call failed */
#define PSACAK_ETIMEOUT (-4)  /* a bounded device-side wait ran out */
#define PSACAK_EINTERNAL (-5) /* a device-side consistency check failed */
#define PSACAK_ECANCELED (-6) /* psacak_cancel ended the build */

/* Induced-scan engine selection (psacak_schedule.engine). */
#define PSACAK_ENGINE_AUTO 0     /* bucket scan for byte levels, doubling otherwise */
#define PSACAK_ENGINE_BUCKET 1   /* bucket-ordered scan (alphabets <= 256 only) */
#define PSACAK_ENGINE_DOUBLING 2 /* chain-doubling scan (any alphabet) */

/* Tunables of one build.  Zero fields mean "use the default" (finish_below:
 * 0 = never; inner_finish_below: 0 = finish_below).  A NULL schedule is the
 * zero schedule with finish_below = PSACAK_DEFAULT_FINISH_BELOW for byte
 * texts and PSACAK_DEFAULT_FINISH_BELOW32 for integer texts,
 * inner_finish_below = PSACAK_DEFAULT_INNER_FINISH_BELOW and tile_items =
 * PSACAK_DEFAULT_TILE_ITEMS: shorter texts are sorted directly by prefix
 * doubling, longer ones by induced sorting at the top level and prefix
 * doubling from the first reduced string on.  Measured on a B200 for
 * 2^20..2^28 symbols: byte texts (genome-like, i.i.d. and Markov ACGT) sort
 * faster by prefix doubling below about 2^24 bytes and by induced sorting
 * above; integer texts (i.i.d. over 2^16, Zipf with planted repeats) sort
 * 1.7x..3x faster by prefix doubling at every length, so the integer
 * cut-off equals the inner one.  The inner cut-off is the fastest measured
 * for a 1 GiB genome-like text.  Every schedule gives the same suffix
 * array; it only changes speed. */
#define PSACAK_DEFAULT_FINISH_BELOW (1u << 24)
#define PSACAK_DEFAULT_FINISH_BELOW32 (1u << 30)
#define PSACAK_DEFAULT_INNER_FINISH_BELOW (1u << 30)
#define PSACAK_DEFAULT_TILE_ITEMS 16u
typedef struct {
    uint32_t engine;           /* PSACAK_ENGINE_* for level 0 */
    uint32_t inner_engine;     /* PSACAK_ENGINE_* for levels >= 1 */
    uint32_t scan_ctas_per_sm; /* CTAs per SM of the grid-stride helper kernels (0 = 4) */
    uint32_t batch_chunk_mib;  /* batch builds: max MiB per concatenated build (0 = 3072) */
    uint32_t tile_items;       /* items per thread of the bucket scatter and compactions: 8, 12 or 16 (0 = 8) */
    uint32_t finish_below;     /* recursion strategy: levels shorter than this (the text itself
                                  included) are sorted directly by prefix doubling instead of
                                  induced sorting and recursion (0 = never) */
    uint32_t inner_finish_below; /* the same cut-off for the reduced strings (levels >= 1),
                                    0 = finish_below */
    uint32_t reserved[1];
} psacak_schedule;

/* One record per recursion level of the last build on a context. */
typedef struct {
    uint32_t level;  /* 0 = input text */
    uint32_t width;  /* symbol width in bytes of this level: 1 or 4 */
    uint64_t m;      /* level length */
    uint64_t n_lms;  /* LMS positions = length of the reduced string */
    uint64_t k;      /* distinct LMS-substring names */
    uint64_t hash;   /* hash of the translated reduced string (0 when k == n_lms) */
} psacak_level_info;

typedef struct psacak_ctx psacak_ctx;

/* Creates a builder context on CUDA device `device`.  A context owns a
 * stream, a grow-only device workspace and a pinned staging buffer; calls
 * on one context are serialised, distinct contexts are independent. */
PSACAK_API int psacak_ctx_create(int device, psacak_ctx **out);
PSACAK_API int psacak_ctx_destroy(psacak_ctx *ctx);

/* Description of the last error on the calling thread ("" if none). */
PSACAK_API const char *psacak_last_error_string(void);

/* Library version, e.g. "0.1.0". */
PSACAK_API const char *psacak_version(void);

/*
 * psacak_init -- makes `device` the device of the calling thread's default
 * context (the one psacak8 / psacak32 use) and creates that context now, so
 * that the first build does not pay for CUDA start-up, the pinned buffers
 * and the helper threads.  Optional: without it the default context is
 * created on device 0 by the first build.  PSACAK_EINVAL for a device that
 * does not exist.
 * psacak_shutdown -- releases the calling thread's default context (device
 * workspace, pinned buffers, host copy threads).  A later psacak8 / psacak32
 * call creates a new one.  The reference has neither: its calls keep no state
 * between them (src/lib.rs:64-82).
 */
PSACAK_API int psacak_init(int device);
PSACAK_API int psacak_shutdown(void);

/*
 * psacak8 -- suffix array of a byte string, host pointers.
 * Replaces psacak_inplace(text: &[u8], suf: &mut [u32]) (src/lib.rs:77-82)
 * and psacak (src/lib.rs:64-69), which drive psacak8 (src/psacak8.rs:19).
 * `sa` receives n entries.  n must be < 2^32 - 1 (src/lib.rs:65, :79);
 * PSACAK_EINVAL otherwise.  Uses a per-thread default context on device 0.
 */
PSACAK_API int psacak8(const uint8_t *text, uint64_t n, uint32_t *sa);

/*
 * psacak32 -- suffix array of an integer-alphabet string, host pointers.
 * Replaces the reference's integer-alphabet path: translate_sample
 * (src/psacak32.rs:912-943) followed by psacak32 (src/psacak32.rs:24), with
 * saca_tiny when distinct symbols >= n (src/psacak32.rs:873-881).  The
 * translation runs on the device.  n must be <= 2^31 - 1
 * (src/psacak32.rs:25).
 */
PSACAK_API int psacak32(const uint32_t *text, uint64_t n, uint32_t *sa);

/* Same as psacak8 / psacak32 on an explicit context (host pointers). */
PSACAK_API int psacak8_ctx(psacak_ctx *ctx, const uint8_t *text, uint64_t n, uint32_t *sa,
                const psacak_schedule *sched);
PSACAK_API int psacak32_ctx(psacak_ctx *ctx, const uint32_t *text, uint64_t n, uint32_t *sa,
                 const psacak_schedule *sched);

/* Device-pointer forms: `d_text` and `d_sa` live on the context's device;
 * `stream` is a cudaStream_t (NULL = the context's own stream).  The call
 * returns after the build has finished on that stream. */
PSACAK_API int psacak8_dev(psacak_ctx *ctx, const uint8_t *d_text, uint64_t n, uint32_t *d_sa,
                void *stream, const psacak_schedule *sched);
PSACAK_API int psacak32_dev(psacak_ctx *ctx, const uint32_t *d_text, uint64_t n, uint32_t *d_sa,
                 void *stream, const psacak_schedule *sched);

/*
 * psacak8_batch -- suffix arrays of n_texts independent byte strings in one
 * build.  The reference has only the per-text call (src/lib.rs:77); this is
 * that call applied to every text, with one SA per text in sas[i] (lens[i]
 * entries each).  Host pointers.
 */
PSACAK_API int psacak8_batch(psacak_ctx *ctx, const uint8_t *const *texts, const uint64_t *lens,
                  uint32_t n_texts, uint32_t *const *sas, const psacak_schedule *sched);

/*
 * psacak8_batch_dev -- device form of psacak8_batch: the texts are packed back
 * to back in d_texts, text i occupying bytes [offsets[i], offsets[i+1]) (a
 * host array of n_texts + 1 entries); text i's SA is written to
 * d_sas[offsets[i] .. offsets[i+1]).  All texts are sorted by one build of
 * their concatenation with a separator smaller than every byte, then split
 * by text.
 */
PSACAK_API int psacak8_batch_dev(psacak_ctx *ctx, const uint8_t *d_texts, const uint64_t *offsets, uint32_t n_texts,
                                 uint32_t *d_sas, void *stream, const psacak_schedule *sched);

/*
 * psacak_cancel -- asks the build running on `ctx` to stop.  Safe to call
 * from any thread while another thread is inside a call on `ctx`.  The build
 * polls the request at its checkpoints (each recursion level, each round of
 * the chain-doubling scans, each chunk or text of a batch), lets the work it
 * has queued finish and returns PSACAK_ECANCELED; its output arrays are then
 * unspecified and the context stays usable.  A request made while no build
 * runs on `ctx` ends the next one at its first checkpoint.  The reference
 * has no counterpart (its calls cannot be interrupted, src/lib.rs:64-82).
 */
PSACAK_API int psacak_cancel(psacak_ctx *ctx);

/* Per-level records of the last build on `ctx` (see psacak_level_info). */
PSACAK_API int psacak_get_trace(psacak_ctx *ctx, psacak_level_info *out, uint32_t cap, uint32_t *count);

/*
 * Device-side suffix-array check (Burkhardt & Kaerkkaeinen, CPM 2003, O(n)):
 * *ok = 1 iff d_sa is a permutation of [0, n) and adjacent suffixes are in
 * order.  The reference's CLI check (src/bin/psacak.rs:73-80) is the
 * quadratic form of the same test.
 */
PSACAK_API int psacak_check_sa8_dev(psacak_ctx *ctx, const uint8_t *d_text, uint64_t n,
                         const uint32_t *d_sa, int *ok, void *stream);
PSACAK_API int psacak_check_sa32_dev(psacak_ctx *ctx, const uint32_t *d_text, uint64_t n,
                          const uint32_t *d_sa, int *ok, void *stream);

/* Per-kernel-class device time of the builds made while profiling is on
 * (CUDA events around every launch; adds a little host overhead).
 * `bytes` is the algorithmic traffic of the class: the bytes its launches
 * must move by construction (each input read once, each output written
 * once), independent of caching. */
typedef struct {
    char name[32];
    uint64_t launches;
    uint64_t items;   /* units processed (entries, positions, keys) */
    uint64_t bytes;   /* algorithmic bytes, 0 where not defined */
    double ms;        /* summed device time */
} psacak_kernel_stat;

PSACAK_API int psacak_profile_enable(psacak_ctx *ctx, int on);
PSACAK_API int psacak_profile_reset(psacak_ctx *ctx);
PSACAK_API int psacak_profile_get(psacak_ctx *ctx, psacak_kernel_stat *out, uint32_t cap, uint32_t *count);

/* Largest n accepted by psacak_check_sa8_noalloc (8 MiB of fixed scratch). */
#define PSACAK_NOALLOC_CHECK_MAX (1u << 21)

/*
 * psacak_check_sa8_noalloc -- the check of psacak_check_sa8_dev for callers
 * that cannot allocate device memory: a serving loop in which cudaMalloc /
 * cudaFree would synchronise the device and stall its other streams, or a
 * host process that owns the device memory budget and forbids allocations by
 * its plugins.  No counterpart in the reference.  It allocates nothing: its
 * scratch is an array of PSACAK_NOALLOC_CHECK_MAX entries compiled into the
 * library (held on every GPU that loads the library until exit), so n above
 * that limit returns PSACAK_EINVAL.  No context is used; `stream` is a
 * cudaStream_t (NULL = default stream) on the current device.  The first call
 * on a device looks up the array's device address (cudaGetSymbolAddress).
 * All calls share the array: calls that overlap on the GPU race.  Returns
 * after the check has finished on `stream`.
 */
PSACAK_API int psacak_check_sa8_noalloc(const uint8_t *d_text, uint64_t n, const uint32_t *d_sa, int *ok,
                                        void *stream);

/*
 * Arrays derived from a suffix array `d_sa` of n entries (sentinel excluded,
 * as psacak8 / psacak32 produce it), on the device.  hucsmn/psacak has no
 * counterpart; these are the usual consumers of its output.  All pointers
 * are device pointers except `primary`; work is ordered on `stream` (NULL =
 * the context's stream) and the call returns when it has finished.
 *
 * psacak_isa_dev: inverse suffix array, d_isa[d_sa[i]] = i.
 * psacak_bwt8_dev: Burrows-Wheeler transform of text + sentinel without the
 *   sentinel character (libdivsufsort's divbwt convention): d_bwt[0] =
 *   text[n-1], then text[SA[i]-1] for every i with SA[i] > 0 in SA order;
 *   *primary = 1 + the i with SA[i] = 0 (the sentinel's row).  n bytes out.
 * psacak_lcp8_dev / psacak_lcp32_dev: LCP array, d_lcp[0] = 0 and d_lcp[i]
 *   = length of the longest common prefix of the suffixes SA[i-1] and
 *   SA[i].  Work O(n log n) for any text (permuted-LCP method).
 */
PSACAK_API int psacak_isa_dev(psacak_ctx *ctx, const uint32_t *d_sa, uint64_t n, uint32_t *d_isa, void *stream);
PSACAK_API int psacak_bwt8_dev(psacak_ctx *ctx, const uint8_t *d_text, uint64_t n, const uint32_t *d_sa,
                               uint8_t *d_bwt, uint64_t *primary, void *stream);
PSACAK_API int psacak_lcp8_dev(psacak_ctx *ctx, const uint8_t *d_text, uint64_t n, const uint32_t *d_sa,
                               uint32_t *d_lcp, void *stream);
PSACAK_API int psacak_lcp32_dev(psacak_ctx *ctx, const uint32_t *d_text, uint64_t n, const uint32_t *d_sa,
                                uint32_t *d_lcp, void *stream);

/*
 * FM-index of a byte text, over its BWT (psacak_bwt8_dev's output: n bytes
 * and the primary index), on the device.  No counterpart in hucsmn/psacak;
 * its suffix array (sentinel excluded, src/lib.rs:30-43) fixes the rows.
 *
 * psacak_fm_bytes: size of the index of an n-byte text (2 + 4/256 bytes per
 *   text byte plus a 2 KiB header): the caller allocates it, 16-byte
 *   aligned.
 * psacak_fm_build_dev: fills d_fm (C array and rank checkpoints: a count of
 *   every byte value per 2^16 positions and, relative to it, per 256).
 * psacak_fm_count_dev: backward search of n_patterns patterns, pattern i
 *   being bytes [d_offsets[i], d_offsets[i+1]) of d_patterns (d_offsets a
 *   device array of n_patterns + 1 entries): d_ranges[2i], d_ranges[2i+1]
 *   = the half-open range of suffix-array indices whose suffixes start with
 *   the pattern (the occurrences are SA[lo .. hi), their number hi - lo; an
 *   empty pattern matches [0, n)).  d_bwt is the BWT the index was built
 *   from.
 */
PSACAK_API uint64_t psacak_fm_bytes(uint64_t n);
PSACAK_API int psacak_fm_build_dev(psacak_ctx *ctx, const uint8_t *d_bwt, uint64_t n, uint64_t primary, void *d_fm,
                                   void *stream);
PSACAK_API int psacak_fm_count_dev(psacak_ctx *ctx, const void *d_fm, const uint8_t *d_bwt,
                                   const uint8_t *d_patterns, const uint64_t *d_offsets, uint32_t n_patterns,
                                   uint32_t *d_ranges, void *stream);

/* Number of kernels the library launched (all contexts of the process). */
PSACAK_API uint64_t psacak_kernel_launches(psacak_ctx *ctx);

/* Number of host round trips inside builds (all contexts of the process):
 * times the host waited for a count or histogram computed on the device
 * before it could choose the next launches.  They set the latency floor of
 * short and mid-size builds. */
PSACAK_API uint64_t psacak_round_trips(psacak_ctx *ctx);

#ifdef __cplusplus
}
#endif
#endif
