/*
 * synth.c -- seeded synthetic texts for the psacak_b200 tests and benchmark.
 *
 * Host-only C (no GPU).  All generators draw from xoshiro256** seeded by
 * splitmix64(seed), so every input is reproducible from its seed.  The
 * shapes stand in for the reference's benchmark corpus (Pizza&Chili files
 * and the uniform random files of bench/generate.sh), which are not
 * available offline.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#if defined(_WIN32)
#define SYNTH_API __declspec(dllexport)
#else
#define SYNTH_API __attribute__((visibility("default")))
#endif

typedef struct {
    uint64_t s[4];
} xo_t;

static inline uint64_t rotl64(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }

static uint64_t splitmix64(uint64_t *x) {
    uint64_t z = (*x += 0x9e3779b97f4a7c15ull);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

static void xo_seed(xo_t *r, uint64_t seed) {
    uint64_t x = seed;
    for (int i = 0; i < 4; i++) r->s[i] = splitmix64(&x);
}

static inline uint64_t xo_next(xo_t *r) {
    uint64_t *s = r->s;
    uint64_t result = rotl64(s[1] * 5, 7) * 9;
    uint64_t t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = rotl64(s[3], 45);
    return result;
}

static inline double xo_unit(xo_t *r) { return (double)(xo_next(r) >> 11) * 0x1.0p-53; }

static inline uint64_t xo_below(xo_t *r, uint64_t k) {
    return (uint64_t)(((unsigned __int128)xo_next(r) * k) >> 64);
}

/* geometric on {1,2,...} with the given mean */
static uint64_t xo_geometric(xo_t *r, double mean) {
    if (mean <= 1.0) return 1;
    double u = xo_unit(r);
    if (u <= 0.0) u = 0x1.0p-53;
    return 1 + (uint64_t)floor(log(u) / log(1.0 - 1.0 / mean));
}

static uint64_t xo_loguniform(xo_t *r, double lo, double hi) {
    double v = exp(log(lo) + xo_unit(r) * (log(hi) - log(lo)));
    uint64_t x = (uint64_t)v;
    return x < (uint64_t)lo ? (uint64_t)lo : x;
}

/* Mixes (seed, index) into a per-item seed. */
SYNTH_API uint64_t psacak_synth_hash2(uint64_t seed, uint64_t i) {
    uint64_t x = seed ^ (0xd1b54a32d192ed03ull * (i + 1));
    return splitmix64(&x);
}

/* i.i.d. uniform bytes over `alphabet[0..k)`. */
SYNTH_API void psacak_synth_iid(uint8_t *out, uint64_t n, const uint8_t *alphabet, uint32_t k,
                                uint64_t seed) {
    xo_t r;
    xo_seed(&r, seed);
    for (uint64_t i = 0; i < n; i++) out[i] = alphabet[xo_below(&r, k)];
}

static const uint8_t ACGT[4] = {'A', 'C', 'G', 'T'};

static inline int base_code(uint8_t c) {
    switch (c) {
        case 'C': return 1;
        case 'G': return 2;
        case 'T': return 3;
        default: return 0;
    }
}

/* Markov table: `ctx` rows of 4 cumulative probabilities, rows drawn from a
 * flat Dirichlet (normalised exponentials). */
static void markov_table(xo_t *r, double *cum, int ctx) {
    for (int c = 0; c < ctx; c++) {
        double w[4], s = 0;
        for (int b = 0; b < 4; b++) {
            double u = xo_unit(r);
            if (u <= 0) u = 0x1.0p-53;
            w[b] = -log(u);
            s += w[b];
        }
        double acc = 0;
        for (int b = 0; b < 4; b++) {
            acc += w[b] / s;
            cum[c * 4 + b] = acc;
        }
        cum[c * 4 + 3] = 1.0;
    }
}

static inline uint8_t markov_draw(xo_t *r, const double *row) {
    double u = xo_unit(r);
    int b = 0;
    while (b < 3 && u >= row[b]) b++;
    return ACGT[b];
}

/* Integer form of a Markov table: per context three 32-bit thresholds. */
static void markov_thresholds(const double *cum, uint32_t *thr, int ctx) {
    for (int c = 0; c < ctx; c++)
        for (int b = 0; b < 3; b++) {
            double v = cum[c * 4 + b] * 4294967296.0;
            thr[c * 3 + b] = v >= 4294967295.0 ? 0xFFFFFFFFu : (uint32_t)v;
        }
}

/* Index (0..3) of the base drawn by the 32-bit uniform u. */
static inline int markov_draw32(uint32_t u, const uint32_t *t) {
    return (u >= t[0]) + (u >= t[1]) + (u >= t[2]);
}

typedef struct {
    uint64_t n_bases;   /* positions emitted by the Markov chain */
    uint64_t n_nrun;    /* positions inside N runs */
    uint64_t n_copied;  /* positions copied from an earlier segment */
    uint64_t n_mutated; /* copied positions that received a point mutation */
    uint64_t n_segments;
} psacak_synth_genome_stats;

/*
 * Genome-like text: order-3 Markov chain over ACGT (transition rows drawn
 * once from the seed), runs of 'N' covering about 5% of positions (run
 * length geometric, mean 1000), and segments copied from earlier positions
 * covering about 30% (length log-uniform on [100, 50000], each copied base
 * replaced by a uniform ACGT base with probability 0.01).  Segment kinds
 * are drawn with P(N run) = 0.1213, P(copy) = 0.0906, otherwise a Markov
 * segment of geometric length with mean 2000; these probabilities give the
 * 5% / 30% / 65% position shares in expectation.
 */
SYNTH_API void psacak_synth_genome(uint8_t *out, uint64_t n, uint64_t seed,
                                   psacak_synth_genome_stats *st) {
    xo_t r;
    xo_seed(&r, seed);
    double cum[64 * 4];
    markov_table(&r, cum, 64);
    uint32_t thr[64 * 3];
    markov_thresholds(cum, thr, 64);
    psacak_synth_genome_stats s;
    memset(&s, 0, sizeof(s));
    uint64_t p = 0;
    int ctx = 0;
    while (p < n) {
        double u = xo_unit(&r);
        s.n_segments++;
        if (u < 0.1213) {
            uint64_t len = xo_geometric(&r, 1000.0);
            if (len > n - p) len = n - p;
            memset(out + p, 'N', len);
            p += len;
            s.n_nrun += len;
            ctx = 0;
            continue;
        }
        if (u < 0.1213 + 0.0906 && p >= 100) {
            uint64_t len = xo_loguniform(&r, 100.0, 50000.0);
            if (len > p) len = p;
            if (len > n - p) len = n - p;
            uint64_t src = xo_below(&r, p - len + 1);
            memmove(out + p, out + src, len);
            /* point mutations: each copied base with probability 0.01,
               drawn as geometric gaps between mutated bases */
            for (uint64_t t = xo_geometric(&r, 100.0) - 1; t < len; t += xo_geometric(&r, 100.0)) {
                out[p + t] = ACGT[xo_below(&r, 4)];
                s.n_mutated++;
            }
            p += len;
            s.n_copied += len;
            ctx = 0;
            for (uint64_t t = (p >= 3 ? p - 3 : 0); t < p; t++) ctx = ((ctx << 2) | base_code(out[t])) & 63;
            continue;
        }
        uint64_t len = xo_geometric(&r, 2000.0);
        if (len > n - p) len = n - p;
        for (uint64_t t = 0; t < len; t += 2) {
            uint64_t x = xo_next(&r);
            int b = markov_draw32((uint32_t)(x >> 32), thr + ctx * 3);
            out[p + t] = ACGT[b];
            ctx = ((ctx << 2) | b) & 63;
            if (t + 1 < len) {
                b = markov_draw32((uint32_t)x, thr + ctx * 3);
                out[p + t + 1] = ACGT[b];
                ctx = ((ctx << 2) | b) & 63;
            }
        }
        p += len;
        s.n_bases += len;
    }
    if (st) *st = s;
}

/* Order-2 Markov chain over ACGT, transition rows drawn from the seed. */

SYNTH_API void psacak_synth_markov2(uint8_t *out, uint64_t n, uint64_t seed) {
    xo_t r;
    xo_seed(&r, seed);
    double cum[16 * 4];
    markov_table(&r, cum, 16);
    uint32_t thr[16 * 3];
    markov_thresholds(cum, thr, 16);
    int ctx = 0;
    for (uint64_t i = 0; i < n; i += 2) {
        uint64_t x = xo_next(&r);
        int b = markov_draw32((uint32_t)(x >> 32), thr + ctx * 3);
        out[i] = ACGT[b];
        ctx = ((ctx << 2) | b) & 15;
        if (i + 1 < n) {
            b = markov_draw32((uint32_t)x, thr + ctx * 3);
            out[i + 1] = ACGT[b];
            ctx = ((ctx << 2) | b) & 15;
        }
    }
}

/* `count` lengths, log-uniform on [lo, hi]. */
SYNTH_API void psacak_synth_loguniform(uint64_t *out, uint64_t count, uint64_t lo, uint64_t hi,
                                       uint64_t seed) {
    xo_t r;
    xo_seed(&r, seed);
    for (uint64_t i = 0; i < count; i++) {
        uint64_t v = xo_loguniform(&r, (double)lo, (double)hi);
        out[i] = v > hi ? hi : v;
    }
}

/*
 * u32 symbols over an alphabet of `alphabet` ids with Zipf(s) rank
 * frequencies (ranks mapped to ids by a seeded permutation), with planted
 * exact repeats: a segment is a repeat with probability q (length
 * log-uniform on [rep_min, rep_max], copied from a uniform earlier offset),
 * otherwise an i.i.d. Zipf segment of geometric length with mean 50000.
 * q is chosen so that repeats cover `repeat_frac` of the positions in
 * expectation.
 */
SYNTH_API int psacak_synth_zipf32(uint32_t *out, uint64_t n, uint32_t alphabet, double s,
                                  double repeat_frac, uint32_t rep_min, uint32_t rep_max,
                                  uint64_t seed) {
    if (alphabet == 0) return -1;
    xo_t r;
    xo_seed(&r, seed);
    double *cdf = (double *)malloc(sizeof(double) * alphabet);
    uint32_t *perm = (uint32_t *)malloc(sizeof(uint32_t) * alphabet);
    if (!cdf || !perm) {
        free(cdf);
        free(perm);
        return -1;
    }
    double acc = 0;
    for (uint32_t k = 0; k < alphabet; k++) {
        acc += pow((double)(k + 1), -s);
        cdf[k] = acc;
    }
    for (uint32_t k = 0; k < alphabet; k++) cdf[k] /= acc;
    cdf[alphabet - 1] = 1.0;
    for (uint32_t k = 0; k < alphabet; k++) perm[k] = k;
    for (uint32_t k = alphabet - 1; k > 0; k--) {
        uint32_t j = (uint32_t)xo_below(&r, (uint64_t)k + 1);
        uint32_t t = perm[k];
        perm[k] = perm[j];
        perm[j] = t;
    }
    double q = 0.0;
    if (repeat_frac > 0 && rep_max >= rep_min && rep_min > 0) {
        double mean_rep = rep_max > rep_min
                              ? ((double)rep_max - rep_min) / (log((double)rep_max) - log((double)rep_min))
                              : (double)rep_min;
        double mean_seg = 50000.0;
        q = repeat_frac * mean_seg / ((1 - repeat_frac) * mean_rep + repeat_frac * mean_seg);
    }
    uint64_t p = 0;
    while (p < n) {
        if (q > 0 && xo_unit(&r) < q && p >= rep_min) {
            uint64_t len = xo_loguniform(&r, (double)rep_min, (double)rep_max);
            if (len > p) len = p;
            if (len > n - p) len = n - p;
            uint64_t src = xo_below(&r, p - len + 1);
            memcpy(out + p, out + src, len * sizeof(uint32_t));
            p += len;
            continue;
        }
        uint64_t len = xo_geometric(&r, 50000.0);
        if (len > n - p) len = n - p;
        for (uint64_t t = 0; t < len; t++) {
            double u = xo_unit(&r);
            uint32_t lo = 0, hi = alphabet - 1;
            while (lo < hi) {
                uint32_t mid = lo + (hi - lo) / 2;
                if (cdf[mid] > u) hi = mid;
                else lo = mid + 1;
            }
            out[p + t] = perm[lo];
        }
        p += len;
    }
    free(cdf);
    free(perm);
    return 0;
}
