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
};

// ---- placement of the LMS positions --------------------------------------

__global__ void k_place_lms_any8(const uint8_t *__restrict__ text, uint64_t nwords, const uint32_t *__restrict__ lms,
                                 const ByteGeom *__restrict__ g, uint32_t *cursor, uint32_t *sa) {
    for (uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; w < nwords; w += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t word = lms[w];
        while (word) {
            int b = __ffs(word) - 1;
            word &= word - 1;
            uint64_t p = (w << 5) + b;
            uint8_t c = text[p];
            uint32_t slot = atomicAdd(&cursor[c], 1u);
            sa[g->tail[c] - 1 - slot] = (uint32_t)p;
        }
    }
}

__global__ void k_place_lms_sorted8(const uint8_t *__restrict__ text, const uint32_t *__restrict__ sorted,
                                    uint64_t n1, const ByteGeom *__restrict__ g, uint32_t *sa) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n1; i += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t p = sorted[i];
        uint8_t c = text[p];
        sa[g->tail[c] - g->lmscount[c] + ((uint32_t)i - g->lmsstart[c])] = p;
    }
}

// cursors: L scan starts at the bucket heads, S scan at the tails; the
// sentinel suffix n-1 is the first entry of its bucket (src/psacak8.rs:131-135).
__global__ void k_init_cursors(const ByteGeom *__restrict__ g, const uint8_t *__restrict__ text, uint64_t n,
                               uint32_t *curL, uint32_t *curS, uint32_t *sa) {
    int c = threadIdx.x;
    uint8_t last = text[n - 1];
    curL[c] = g->head[c] + (c == last ? 1u : 0u);
    curS[c] = g->tail[c];
    if (c == 0) sa[g->head[last]] = (uint32_t)(n - 1);
}

// ---- chain expansion -----------------------------------------------------

// Seeds in scan order: L part = sa[start + q]; S part = sa[start - q].
// runs[q] = number of equal characters c in front of the seed.
__global__ void k_seed_runs(const uint8_t *__restrict__ text, const uint32_t *__restrict__ sa, uint32_t start, int dir,
                            uint32_t nseeds, uint8_t c, uint32_t *runs, uint32_t *maxrun) {
    uint32_t mx = 0;
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < nseeds; q += gridDim.x * blockDim.x) {
        uint32_t x = sa[dir > 0 ? start + q : start - q];
        uint32_t r = 0;
        while (r < x && text[x - r - 1] == c) r++;
        runs[q] = r;
        mx = r > mx ? r : mx;
    }
    for (int o = 16; o > 0; o >>= 1) {
        uint32_t t = __shfl_down_sync(FULL_MASK, mx, o);
        mx = t > mx ? t : mx;
    }
    if ((threadIdx.x & 31) == 0 && mx) atomicMax(maxrun, mx);
}

struct RunLoad {
    const uint32_t *runs;
    __device__ __forceinline__ uint32_t operator()(uint64_t i) const { return runs[i]; }
};
struct RunStore {
    uint32_t *off;
    __device__ __forceinline__ void operator()(uint64_t i, uint32_t excl, uint32_t) const { off[i] = excl; }
};

// Cell q (row-major over seeds) -> (depth d, value seed - d).
__global__ void k_expand_cells(const uint32_t *__restrict__ sa, uint32_t start, int dir, uint32_t nseeds,
                               const uint32_t *__restrict__ off, uint32_t ncells, uint32_t *keys, uint32_t *vals) {
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < ncells; q += gridDim.x * blockDim.x) {
        // last seed s with off[s] <= q
        uint32_t lo = 0, hi = nseeds - 1;
        while (lo < hi) {
            uint32_t mid = (lo + hi + 1) >> 1;
            if (off[mid] <= q) lo = mid;
            else hi = mid - 1;
        }
        uint32_t d = q - off[lo] + 1;
        uint32_t x = sa[dir > 0 ? start + lo : start - lo];
        keys[q] = d;
        vals[q] = x - d;
    }
}

__global__ void k_place_cells(const uint32_t *__restrict__ vals, uint32_t ncells, uint32_t first, int dir,
                              uint32_t *sa) {
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < ncells; q += gridDim.x * blockDim.x)
        sa[dir > 0 ? first + q : first - q] = vals[q];
}

// ---- multisplit ----------------------------------------------------------

// Per-CTA digit histogram of the entries that induce; the digit (the
// predecessor's character) is kept in `dg` for the scatter pass.
template <bool LSCAN>
__global__ void __launch_bounds__(MS_BLOCK) k_ms_up(const uint8_t *__restrict__ text, const uint32_t *__restrict__ sa,
                                                    BucketSeq seq, uint32_t nitems, uint8_t c, uint64_t chunk,
                                                    uint8_t *dg, uint32_t *hist, uint32_t G) {
    __shared__ uint32_t sh[MS_WARPS][256];
    for (int i = threadIdx.x; i < MS_WARPS * 256; i += MS_BLOCK) (&sh[0][0])[i] = 0;
    __syncthreads();
    const int w = threadIdx.x >> 5;
    uint64_t start = (uint64_t)blockIdx.x * chunk;
    uint64_t end = start + chunk < nitems ? start + chunk : nitems;
    const uint32_t invalid = LSCAN ? 0u : 255u;
    for (uint64_t base = start; base < end; base += MS_BLOCK) {
        uint64_t q = base + threadIdx.x;
        uint32_t d = 256;
        if (q < end) {
            uint32_t x = sa[seq.slot((uint32_t)q)];
            uint32_t dd = invalid;
            if (x > 0) {
                uint32_t c0 = text[x - 1];
                if (LSCAN ? c0 > c : c0 < c) dd = c0;
            }
            dg[q] = (uint8_t)dd;
            if (dd != invalid) d = dd;
        }
        uint32_t peers = __match_any_sync(FULL_MASK, d);
        if (d < 256 && (int)(threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(&sh[w][d], __popc(peers));
    }
    __syncthreads();
    for (int d = threadIdx.x; d < 256; d += MS_BLOCK) {
        uint32_t s = 0;
        for (int ww = 0; ww < MS_WARPS; ww++) s += sh[ww][d];
        hist[(uint64_t)d * G + blockIdx.x] = s;
    }
}

// Turns the histograms into per-CTA start slots and advances the cursors.
__global__ void k_ms_offsets(uint32_t *hist, uint32_t G, uint32_t *cursor, int dir, unsigned long long *induced) {
    int d = threadIdx.x;
    uint32_t run = cursor[d], tot = 0;
    for (uint32_t b = 0; b < G; b++) {
        uint32_t h = hist[(uint64_t)d * G + b];
        hist[(uint64_t)d * G + b] = run;
        run = dir > 0 ? run + h : run - h;
        tot += h;
    }
    cursor[d] = run;
    if (tot) atomicAdd(induced, (unsigned long long)tot);
}

template <bool LSCAN>
__global__ void __launch_bounds__(MS_BLOCK) k_ms_down(const uint32_t *__restrict__ sa_in, BucketSeq seq,
                                                      uint32_t nitems, uint64_t chunk, const uint8_t *__restrict__ dg,
                                                      const uint32_t *__restrict__ hist, uint32_t G, uint32_t *sa_out,
                                                      uint64_t n, uint32_t *err) {
    __shared__ uint32_t s_val[MS_TILE];
    __shared__ uint8_t s_dig[MS_TILE];
    __shared__ uint32_t s_off[256];
    __shared__ uint32_t s_tstart[256];
    __shared__ uint32_t s_tcount[256];
    __shared__ uint16_t s_wcnt[MS_WARPS][256];
    __shared__ uint32_t s_scan[33];
    const int w = threadIdx.x >> 5;
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t lt = lanemask_lt();
    const uint32_t invalid = LSCAN ? 0u : 255u;
    uint64_t start = (uint64_t)blockIdx.x * chunk;
    uint64_t end = start + chunk < nitems ? start + chunk : nitems;
    s_off[threadIdx.x] = hist[(uint64_t)threadIdx.x * G + blockIdx.x];
    for (uint64_t base = start; base < end; base += MS_TILE) {
        for (int i = threadIdx.x; i < MS_WARPS * 256; i += MS_BLOCK) (&s_wcnt[0][0])[i] = 0;
        __syncthreads();
        uint32_t v[MS_IPT];
        uint16_t rk[MS_IPT];
        uint32_t dgt[MS_IPT];
#pragma unroll
        for (int r = 0; r < MS_IPT; r++) {
            uint64_t q = base + (uint64_t)w * 32 * MS_IPT + (uint64_t)r * 32 + lane;
            uint32_t d = 256;
            if (q < end) {
                uint32_t dd = dg[q];
                if (dd != invalid) {
                    d = dd;
                    v[r] = sa_in[seq.slot((uint32_t)q)] - 1;
                }
            }
            dgt[r] = d;
            uint32_t peers = __match_any_sync(FULL_MASK, d);
            uint32_t prior = d < 256 ? s_wcnt[w][d] : 0;
            rk[r] = (uint16_t)(prior + __popc(peers & lt));
            __syncwarp();
            if (d < 256 && (int)lane == __ffs(peers) - 1) s_wcnt[w][d] = (uint16_t)(prior + __popc(peers));
            __syncwarp();
        }
        __syncthreads();
        {
            uint32_t d = threadIdx.x, sum = 0;
#pragma unroll
            for (int ww = 0; ww < MS_WARPS; ww++) {
                uint32_t cc = s_wcnt[ww][d];
                s_wcnt[ww][d] = (uint16_t)sum;
                sum += cc;
            }
            s_tcount[d] = sum;
            uint32_t ex, tot;
            block_scan<uint32_t, OpSum<uint32_t>, MS_BLOCK>(sum, OpSum<uint32_t>(), s_scan, &ex, &tot);
            s_tstart[d] = ex;
            if (d == 0) s_scan[32] = tot;
        }
        __syncthreads();
        const uint32_t tile_valid = s_scan[32];
#pragma unroll
        for (int r = 0; r < MS_IPT; r++) {
            if (dgt[r] < 256) {
                uint32_t pos = s_tstart[dgt[r]] + s_wcnt[w][dgt[r]] + rk[r];
                s_val[pos] = v[r];
                s_dig[pos] = (uint8_t)dgt[r];
            }
        }
        __syncthreads();
        for (uint32_t i = threadIdx.x; i < tile_valid; i += MS_BLOCK) {
            uint32_t d = s_dig[i];
            uint32_t rank = i - s_tstart[d];
            uint64_t o = LSCAN ? (uint64_t)s_off[d] + rank : (uint64_t)s_off[d] - 1 - rank;
            if (o < n) sa_out[o] = s_val[i];
            else dev_fail(err, DEVERR_RANGE);
        }
        __syncthreads();
        {
            uint32_t d = threadIdx.x;
            s_off[d] = LSCAN ? s_off[d] + s_tcount[d] : s_off[d] - s_tcount[d];
        }
        __syncthreads();
    }
}

static inline uint32_t grid_cap(uint64_t n, uint32_t cap) {
    uint64_t g = ceil_div(n ? n : 1, 256);
    return (uint32_t)(g < cap ? g : cap);
}

// Chain expansion of one bucket part.  `start` is the slot of the first
// seed in scan order, `nseeds` the seeds present, `part` the full size of
// the part; fills the remaining part - nseeds slots.
static status_t expand_chains(Ctx &ctx, const uint8_t *text, uint32_t *sa, uint32_t start, int dir, uint32_t nseeds,
                              uint32_t part, uint8_t c, uint32_t *runs, uint32_t *off, uint32_t *k0, uint32_t *v0,
                              uint32_t *k1, uint32_t *v1, cudaStream_t s) {
    if (nseeds == part) return PSACAK_OK;
    if (nseeds == 0 || nseeds > part)
        return set_error(PSACAK_EINTERNAL, "bucket %u: %u seeds for a part of %u", c, nseeds, part);
    uint32_t *d_max = ctx.d_scalars + 8;
    uint32_t *d_tot = ctx.d_scalars + 9;
    PSK_CUDA(cudaMemsetAsync(d_max, 0, sizeof(uint32_t), s));
    PSK_PROF_LAUNCH(s, "chain_runs", nseeds, 0,
                    (k_seed_runs<<<grid_cap(nseeds, 4096), 256, 0, s>>>(text, sa, start, dir, nseeds, c, runs, d_max)));
    PSK_LAUNCH_CHECK();
    PSK_TRY((chunk_scan<uint32_t, OpSum<uint32_t>>(RunLoad{runs}, RunStore{off}, nseeds, ctx.d_partial, d_tot,
                                                   OpSum<uint32_t>(), ctx.scan_ctas, s)));
    uint32_t h[2];
    PSK_TRY(ctx.read_u32(d_max, h, 2));
    const uint32_t maxrun = h[0], ncells = h[1];
    if (nseeds + ncells != part)
        return set_error(PSACAK_EINTERNAL, "bucket %u: %u seeds + %u chained != %u", c, nseeds, ncells, part);
    PSK_PROF_LAUNCH(s, "chain_expand", ncells, 0,
                    (k_expand_cells<<<grid_cap(ncells, 8192), 256, 0, s>>>(sa, start, dir, nseeds, off, ncells, k0, v0)));
    PSK_LAUNCH_CHECK();
    int in1 = 0;
    PSK_TRY((radix_sort_pairs<uint32_t, uint32_t>(k0, v0, k1, v1, ncells, 0, bitlen(maxrun), ctx.d_hist, &in1,
                                                  ctx.radix_ctas, s)));
    uint32_t first = dir > 0 ? start + nseeds : start - nseeds;
    PSK_PROF_LAUNCH(s, "chain_place", ncells, 8ull * ncells,
                    (k_place_cells<<<grid_cap(ncells, 8192), 256, 0, s>>>(in1 ? v1 : v0, ncells, first, dir, sa)));
    PSK_LAUNCH_CHECK();
    return PSACAK_OK;
}

template <bool LSCAN>
static status_t multisplit(Ctx &ctx, const uint8_t *text, uint32_t *sa, uint64_t n, BucketSeq seq, uint8_t c,
                           uint32_t *cursor, uint8_t *dg, cudaStream_t s) {
    uint32_t nitems = seq.a_len + seq.b_len;
    if (nitems == 0) return PSACAK_OK;
    Chunking ch = make_chunking(nitems, MS_TILE, ctx.radix_ctas < RADIX_MAX_CTAS ? ctx.radix_ctas : RADIX_MAX_CTAS);
    // algorithmic bytes: up reads each entry (4) and its predecessor's
    // character (1) and writes the digit (1); down reads the digit (1) and,
    // for inducing entries, the entry (4) and writes it to its bucket (4) --
    // the inducing count is added from the device at the end of the build.
    PSK_PROF_LAUNCH(s, "induce_up", nitems, 6ull * nitems,
                    (k_ms_up<LSCAN><<<ch.G, MS_BLOCK, 0, s>>>(text, sa, seq, nitems, c, ch.chunk, dg, ctx.d_hist,
                                                              ch.G)));
    PSK_PROF_LAUNCH(s, "induce_offsets", 256, 0,
                    (k_ms_offsets<<<1, 256, 0, s>>>(ctx.d_hist, ch.G, cursor, LSCAN ? 1 : -1, ctx.d_induced)));
    PSK_PROF_LAUNCH(s, "induce_down", nitems, 1ull * nitems,
                    (k_ms_down<LSCAN><<<ch.G, MS_BLOCK, 0, s>>>(sa, seq, nitems, ch.chunk, dg, ctx.d_hist, ch.G, sa, n,
                                                                ctx.d_err)));
    PSK_LAUNCH_CHECK();
    return PSACAK_OK;
}

status_t induce_bucket8(Ctx &ctx, const uint8_t *text, uint64_t n, const uint32_t *lms, const ByteGeom &hg,
                        const ByteGeom *dgeom, InduceMode mode, const uint32_t *sorted_lms, uint64_t n1,
                        uint32_t *sa, cudaStream_t s) {
    uint32_t maxpart = 1, maxbucket = 1;
    for (int c = 0; c < 256; c++) {
        uint32_t cnt = hg.tail[c] - hg.head[c];
        maxbucket = cnt > maxbucket ? cnt : maxbucket;
        maxpart = hg.lcount[c] > maxpart ? hg.lcount[c] : maxpart;
        maxpart = hg.scount[c] > maxpart ? hg.scount[c] : maxpart;
    }
    DBuf<uint32_t> cur, runs, off, k0, v0, k1, v1;
    DBuf<uint8_t> dg;
    PSK_TRY(cur.init(ctx, 512));
    PSK_TRY(runs.init(ctx, maxpart));
    PSK_TRY(off.init(ctx, maxpart));
    PSK_TRY(k0.init(ctx, maxpart));
    PSK_TRY(v0.init(ctx, maxpart));
    PSK_TRY(k1.init(ctx, maxpart));
    PSK_TRY(v1.init(ctx, maxpart));
    PSK_TRY(dg.init(ctx, maxbucket));
    uint32_t *curL = cur.get(), *curS = cur.get() + 256;

    // LMS positions at the bucket tails (put_lmscharacters / put_lmssuffixes).
    if (mode == INDUCE_LMS_SUBSTRINGS) {
        PSK_CUDA(cudaMemsetAsync(curL, 0, 256 * sizeof(uint32_t), s));
        const uint64_t nwords = ceil_div(n, 32);
        PSK_PROF_LAUNCH(s, "place_lms", nwords, 0,
                        (k_place_lms_any8<<<grid_cap(nwords, 8192), 256, 0, s>>>(text, nwords, lms, dgeom, curL, sa)));
    } else if (n1 > 0) {
        PSK_PROF_LAUNCH(s, "place_lms", n1, 0,
                        (k_place_lms_sorted8<<<grid_cap(n1, 8192), 256, 0, s>>>(text, sorted_lms, n1, dgeom, sa)));
    }
    k_init_cursors<<<1, 256, 0, s>>>(dgeom, text, n, curL, curS, sa);
    PSK_KCOUNT();
    PSK_LAUNCH_CHECK();

    // L scan: buckets in increasing order.
    for (int c = 0; c < 256; c++) {
        const uint32_t head = hg.head[c], tail = hg.tail[c];
        if (tail == head) continue;
        const uint32_t lc = hg.lcount[c], lmsc = hg.lmscount[c];
        if (lc > 0) {
            uint32_t cl = 0;
            PSK_TRY(ctx.read_u32(curL + c, &cl));
            PSK_TRY(expand_chains(ctx, text, sa, head, +1, cl - head, lc, (uint8_t)c, runs, off, k0, v0, k1, v1, s));
        }
        BucketSeq seq{head, lc, tail - lmsc, lmsc, +1};
        PSK_TRY(multisplit<true>(ctx, text, sa, n, seq, (uint8_t)c, curL, dg, s));
    }
    // S scan: buckets in decreasing order, S parts filled from their tails.
    for (int c = 255; c >= 0; c--) {
        const uint32_t head = hg.head[c], tail = hg.tail[c];
        if (tail == head) continue;
        const uint32_t lc = hg.lcount[c], sc = hg.scount[c];
        if (sc > 0) {
            uint32_t cs = 0;
            PSK_TRY(ctx.read_u32(curS + c, &cs));
            PSK_TRY(expand_chains(ctx, text, sa, tail - 1, -1, tail - cs, sc, (uint8_t)c, runs, off, k0, v0, k1, v1,
                                  s));
        }
        BucketSeq seq{tail - 1, sc, head + lc - 1, lc, -1};
        PSK_TRY(multisplit<false>(ctx, text, sa, n, seq, (uint8_t)c, curS, dg, s));
    }
    return PSACAK_OK;
}

}  // namespace psk
