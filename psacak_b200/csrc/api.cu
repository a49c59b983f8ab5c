// api.cu -- level recursion (the reference's psacak8 / psacak32 drivers) and
// the C ABI of include/psacak_b200.h.
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <memory>
#include <vector>

#include "ctx.cuh"
#include "hostio.cuh"
#include "induce.cuh"
#include "small.cuh"
#include "../../include/psacak_b200_debug.h"

namespace psk {

const char *last_error();
void clear_error();

// ---------------------------------------------------------------------------
// Small kernels used by the driver.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint64_t mix64(uint64_t z) {
    z += 0x9e3779b97f4a7c15ull;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

// Order-dependent hash of a u32 array: sum of mix64((i << 32) ^ v[i]).
__global__ void k_hash_u32(const uint32_t *__restrict__ v, uint64_t n, unsigned long long *out) {
    __shared__ unsigned long long sm[32];
    unsigned long long acc = 0;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        acc += mix64((i << 32) ^ (uint64_t)v[i]);
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(FULL_MASK, acc, o);
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        acc = threadIdx.x < blockDim.x / 32 ? sm[threadIdx.x] : 0ull;
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(FULL_MASK, acc, o);
        if (threadIdx.x == 0) atomicAdd(out, acc);
    }
}

// S-type counts of translated buckets: scnt[text[j]] += 1 for S positions.
// Lanes holding the same symbol share one atomic (frequent symbols would
// otherwise serialise on their counter).
__global__ void k_count_s(const uint32_t *__restrict__ text, uint64_t n, const uint32_t *__restrict__ types,
                          uint32_t *scnt) {
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t jb = (uint64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31u); jb < n; jb += stride) {
        const uint64_t j = jb + lane;
        const bool s = j < n && bm_get(types, j);
        const uint32_t v = s ? text[j] : 0xFFFFFFFFu;
        const uint32_t peers = __match_any_sync(FULL_MASK, v);
        if (s && (int)lane == __ffs(peers) - 1) atomicAdd(&scnt[v], __popc(peers));
    }
}

// Byte text as u32 bucket ids, with the byte histogram in heads[0..256).
__global__ void k_byte_names(const uint8_t *__restrict__ text, uint64_t n, uint32_t *names, uint32_t *heads) {
    __shared__ uint32_t h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint8_t c = text[i];
        names[i] = c;
        atomicAdd(&h[c], 1u);
    }
    __syncthreads();
    if (h[threadIdx.x]) atomicAdd(&heads[threadIdx.x], h[threadIdx.x]);
}
// Counts in heads[0..256) -> bucket heads (exclusive prefix), heads[256] = n.
__global__ void k_byte_heads(uint32_t *heads, uint32_t n) {
    __shared__ uint32_t s_scan[33];
    uint32_t ex;
    block_scan<uint32_t, OpSum<uint32_t>, 256>(heads[threadIdx.x], OpSum<uint32_t>(), s_scan, &ex, (uint32_t *)nullptr);
    heads[threadIdx.x] = ex;
    if (threadIdx.x == 0) heads[256] = n;
}

struct SortedLmsPred {
    const uint32_t *sa;
    const uint32_t *lms;
    uint64_t n;
    uint32_t *err;
    __device__ __forceinline__ bool operator()(uint64_t i) const {
        uint32_t x = sa[i];
        if (x >= n) {
            dev_fail(err, DEVERR_RANGE);
            return false;
        }
        return bm_get(lms, x);
    }
};
struct SortedLmsEmit {
    const uint32_t *sa;
    uint32_t *out;
    __device__ __forceinline__ void operator()(uint64_t i, uint32_t slot) const { out[slot] = sa[i]; }
};

static inline uint32_t grid_for(uint64_t n, uint32_t cap = 16384) {
    uint64_t g = ceil_div(n ? n : 1, 256);
    return (uint32_t)(g < cap ? g : cap);
}

static void trace_push(Ctx &ctx, uint32_t level, uint32_t width, uint64_t m, uint64_t n1, uint64_t k, uint64_t hash);

// Hash of the reduced string handed to the next level, for the trace:
// computed into the level's slot of ctx.d_hashes and read back with the
// others after the build (Ctx::resolve_trace), so it costs no round trip.
static status_t trace_push_hashed(Ctx &ctx, uint32_t level, uint32_t width, uint64_t m, uint64_t n1, uint64_t k,
                                  const uint32_t *v) {
    const uint32_t slot = (uint32_t)ctx.pending_hash.size();
    unsigned long long *d = slot < Ctx::HASH_SLOTS ? ctx.d_hashes + slot : (unsigned long long *)(ctx.d_scalars + 32);
    PSK_CUDA(cudaMemsetAsync(d, 0, sizeof(unsigned long long), ctx.stream));
    k_hash_u32<<<grid_for(n1, 2048), 256, 0, ctx.stream>>>(v, n1, d);
    PSK_KCOUNT();
    PSK_LAUNCH_CHECK();
    if (slot < Ctx::HASH_SLOTS) {
        trace_push(ctx, level, width, m, n1, k, 0);
        ctx.pending_hash.push_back({ctx.trace.size() - 1, slot});
        return PSACAK_OK;
    }
    uint32_t h[2];  // deeper than the slots: read now
    PSK_TRY(ctx.read_u32((const uint32_t *)d, h, 2));
    trace_push(ctx, level, width, m, n1, k, ((uint64_t)h[1] << 32) | h[0]);
    return PSACAK_OK;
}

static void trace_push(Ctx &ctx, uint32_t level, uint32_t width, uint64_t m, uint64_t n1, uint64_t k, uint64_t hash) {
    psacak_level_info li;
    li.level = level;
    li.width = width;
    li.m = m;
    li.n_lms = n1;
    li.k = k;
    li.hash = hash;
    ctx.trace.push_back(li);
}

static int engine_for(const Ctx &ctx, uint32_t level, bool bytes) {
    uint32_t e = level == 0 ? ctx.sched.engine : ctx.sched.inner_engine;
    if (e == PSACAK_ENGINE_BUCKET && !bytes) e = PSACAK_ENGINE_DOUBLING;
    if (e == PSACAK_ENGINE_AUTO) e = bytes ? PSACAK_ENGINE_BUCKET : PSACAK_ENGINE_DOUBLING;
    return (int)e;
}

// ---------------------------------------------------------------------------
// One recursion level (the reference's psacak8, src/psacak8.rs:19-53, and
// psacak32, src/psacak32.rs:24-56): sort the LMS substrings by an induced
// sort, name them, recurse on the reduced string (or invert it directly when
// all names are unique), map the reduced SA back to LMS positions and run
// the final induced sort.
// ---------------------------------------------------------------------------
template <class C>
status_t build_level(Ctx &ctx, const C *text, const uint32_t *names, const uint32_t *bheads, uint64_t nbuckets,
                     uint64_t n, uint32_t *sa, uint32_t level) {
    cudaStream_t s = ctx.stream;
    const uint32_t width = sizeof(C);
    PSK_TRY(ctx.checkpoint());
    if (n <= 3) {
        PSK_TRY(tiny_sa(text, n, sa, s));
        trace_push(ctx, level, width, n, 0, 0, 0);
        return PSACAK_OK;
    }
    const bool bytes = sizeof(C) == 1;
    if constexpr (sizeof(C) == 4) {
        // recursion finisher: short strings are sorted by prefix doubling
        // (the input's own cut-off at level 0, the inner one below it)
        const uint32_t finish = level > 0 && ctx.sched.inner_finish_below ? ctx.sched.inner_finish_below
                                                                          : ctx.sched.finish_below;
        if (names && bheads && finish && n < finish) {
            trace_push(ctx, level, width, n, 0, 0, 0);
            if (n <= SMALL_MAX && nbuckets <= 65535)  // in one CTA's shared memory
                return small_sa<uint32_t>(ctx, names, SmallJobs{nullptr, nullptr, 1, n, n}, (uint32_t)nbuckets, sa, s);
            return sort_by_doubling(ctx, names, bheads, nbuckets, n, sa, s);
        }
    } else {
        // the same for a short byte text: the bytes are the bucket ids
        if (ctx.sched.finish_below && n < ctx.sched.finish_below) {
            if (n <= SMALL_MAX) {  // in one CTA's shared memory
                trace_push(ctx, level, width, n, 0, 0, 0);
                return small_sa<uint8_t>(ctx, (const uint8_t *)text, SmallJobs{nullptr, nullptr, 1, n, n}, 256, sa, s);
            }
            DBuf<uint32_t> bnames, bh;
            PSK_TRY(bnames.init(ctx, n));
            PSK_TRY(bh.init(ctx, 257));
            PSK_CUDA(cudaMemsetAsync(bh.get(), 0, 257 * sizeof(uint32_t), s));
            k_byte_names<<<grid_for(n, 4096), 256, 0, s>>>(text, n, bnames, bh);
            PSK_KCOUNT();
            k_byte_heads<<<1, 256, 0, s>>>(bh, (uint32_t)n);
            PSK_KCOUNT();
            PSK_LAUNCH_CHECK();
            trace_push(ctx, level, width, n, 0, 0, 0);
            return sort_by_doubling(ctx, bnames, bh, 256, n, sa, s);
        }
    }
    const uint64_t nwords = ceil_div(n, 32);
    const uint64_t ntiles = ceil_div(n, TYPE_TILE);
    DBuf<uint32_t> types, lms, wcnt, pref, tscratch;
    PSK_TRY(types.init(ctx, nwords + 1));
    PSK_TRY(lms.init(ctx, nwords + 1));
    PSK_TRY(wcnt.init(ctx, nwords + 1));
    PSK_TRY(pref.init(ctx, nwords + 1));
    PSK_TRY(tscratch.init(ctx, 2 * ntiles + 1024));
    DBuf<ByteHist> hist;
    DBuf<ByteGeom> dgeom;
    if (bytes) {
        PSK_TRY(hist.init(ctx, 1));
        PSK_TRY(dgeom.init(ctx, 1));
    }
    ctx.mark("enter", level);
    PSK_TRY(ctx.ensure_scan(n));
    const ScanEnv env = ctx.scan_env();
    PSK_TRY(type_text<C>(text, n, types, lms, wcnt, bytes ? hist.get() : nullptr, tscratch, env, ctx.scan_ctas, s));
    tscratch.reset();
    PSK_TRY(lms_prefix(wcnt, nwords, pref, ctx.d_scalars, env, s));
    wcnt.reset();
    uint32_t n1u = 0;
    PSK_TRY(ctx.read_u32(ctx.d_scalars, &n1u));
    const uint64_t n1 = n1u;

    ByteGeom hg;
    Geom<C> geom;
    DBuf<uint32_t> scnt, cursor;
    if constexpr (sizeof(C) == 1) {
        ByteHist hh;
        PSK_CUDA(cudaMemcpyAsync(&hh, hist.get(), sizeof(ByteHist), cudaMemcpyDeviceToHost, s));
        PSK_ROUND_TRIP();
        PSK_TRY(ctx.sync());
        uint32_t acc = 0, lacc = 0;
        for (int c = 0; c < 256; c++) {
            hg.head[c] = acc;
            acc += hh.count[c];
            hg.tail[c] = acc;
            hg.lcount[c] = hh.lcount[c];
            hg.scount[c] = hh.count[c] - hh.lcount[c];
            hg.lmscount[c] = hh.lmscount[c];
            hg.lmsstart[c] = lacc;
            lacc += hh.lmscount[c];
        }
        if (acc != n || lacc != n1)
            return set_error(PSACAK_EINTERNAL, "level histogram does not add up (%u/%llu, %u/%llu)", acc,
                             (unsigned long long)n, lacc, (unsigned long long)n1);
        PSK_CUDA(cudaMemcpyAsync(dgeom.get(), &hg, sizeof(ByteGeom), cudaMemcpyHostToDevice, s));
        geom.g = dgeom.get();
        PSK_TRY(cursor.init(ctx, 256));
        PSK_CUDA(cudaMemsetAsync(cursor.get(), 0, 256 * sizeof(uint32_t), s));
    } else {
        PSK_TRY(scnt.init(ctx, n));
        PSK_CUDA(cudaMemsetAsync(scnt.get(), 0, n * sizeof(uint32_t), s));
        k_count_s<<<grid_for(n), 256, 0, s>>>(text, n, types, scnt);
        PSK_KCOUNT();
        PSK_LAUNCH_CHECK();
        geom.scnt = scnt.get();
        geom.names = names;
        geom.heads = bheads;
        PSK_TRY(cursor.init(ctx, n));
        PSK_CUDA(cudaMemsetAsync(cursor.get(), 0, n * sizeof(uint32_t), s));
    }
    const int engine = engine_for(ctx, level, bytes);
    ctx.mark("typing+geometry", level);

    // Stage 1: sort the LMS substrings.
    DBuf<uint32_t> sorted;
    PSK_TRY(sorted.init(ctx, n1));
    bool extracted = false;
    if constexpr (sizeof(C) == 1) {
        if (engine == PSACAK_ENGINE_BUCKET) {
            unsigned long long *lmscnt = ctx.d_induced + 1;
            PSK_CUDA(cudaMemsetAsync(lmscnt, 0, sizeof(unsigned long long), s));
            PSK_TRY(induce_bucket8(ctx, text, n, lms, hg, dgeom.get(), INDUCE_LMS_SUBSTRINGS, nullptr, n1, sa, s,
                                   sorted));
            uint32_t h[2];
            PSK_TRY(ctx.read_u32((const uint32_t *)lmscnt, h, 2));
            const unsigned long long got = ((unsigned long long)h[1] << 32) | h[0];
            if (got != n1)
                return set_error(PSACAK_EINTERNAL, "level %u: %llu LMS extracted by the S scan, expected %llu", level,
                                 got, (unsigned long long)n1);
            extracted = true;
        } else {
            PSK_TRY(induce_doubling<C>(ctx, text, n, types, lms, geom, 256, INDUCE_LMS_SUBSTRINGS, nullptr, n1,
                                       cursor, sa, s));
        }
    } else {
        PSK_TRY(induce_doubling<C>(ctx, text, n, types, lms, geom, nbuckets, INDUCE_LMS_SUBSTRINGS, nullptr, n1,
                                   cursor, sa, s));
    }
    cursor.reset();
    ctx.mark("induce lms-substrings", level);

    // Stage 2: name them and build the reduced string.
    DBuf<uint32_t> red, heads, flags, sa1, names1;
    DBuf<uint64_t> sorted_win;  // byte levels, bucket engine: final-mode LMS list with predecessor windows
    DBuf<uint64_t> sorted_sym;  // doubling engine: final-mode LMS list with the positions' symbols
    uint32_t k = 0;
    if (n1 > 0 && !extracted) {
        PSK_TRY(ctx.compact(SortedLmsPred{sa, lms, n, ctx.d_err}, SortedLmsEmit{sa, sorted}, n, ctx.d_scalars + 1,
                            "extract_lms"));
        uint32_t got = 0;
        PSK_TRY(ctx.read_u32(ctx.d_scalars + 1, &got));
        if (got != n1)
            return set_error(PSACAK_EINTERNAL, "level %u: %u LMS after the induced sort, expected %llu", level, got,
                             (unsigned long long)n1);
    }
    if (n1 > 0) {
        PSK_TRY(red.init(ctx, n1));
        PSK_TRY(heads.init(ctx, n1 + 1));
        PSK_TRY(flags.init(ctx, n1));
        DBuf<uint64_t> lmsx;
        PSK_TRY(lmsx.init(ctx, nwords));
        PSK_TRY(name_lms<C>(text, n, lms, pref, sorted, n1, red, heads, flags, lmsx, ctx.d_scalars + 2, env,
                            ctx.scan_ctas, s));
        PSK_TRY(ctx.read_u32(ctx.d_scalars + 2, &k));
    }
    sorted.reset();
    flags.reset();
    ctx.mark("extract+name", level);
    PSK_TRY(sa1.init(ctx, n1));
    if (n1 > 0) {
        if (k < n1) {
            {
                const uint64_t w1 = ceil_div(n1, 32);
                DBuf<uint32_t> t1, l1, c1, sc1;
                PSK_TRY(t1.init(ctx, w1 + 1));
                PSK_TRY(l1.init(ctx, w1 + 1));
                PSK_TRY(c1.init(ctx, w1 + 1));
                PSK_TRY(sc1.init(ctx, 2 * ceil_div(n1, TYPE_TILE) + 1024));
                PSK_TRY(type_text<uint32_t>(red, n1, t1, l1, c1, nullptr, sc1, env, ctx.scan_ctas, s));
                // the names stay as the next level's dense bucket ids
                PSK_TRY(names1.init(ctx, n1));
                PSK_CUDA(cudaMemcpyAsync(names1.get(), red.get(), n1 * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
                PSK_TRY(translate_names(red, n1, t1, heads, ctx.d_err, s));
            }
            if (level == 0 && ctx.debug_red) {
                uint64_t c = n1 < ctx.debug_cap ? n1 : ctx.debug_cap;
                PSK_CUDA(cudaMemcpyAsync(ctx.debug_red, red.get(), c * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
                ctx.debug_n1 = n1;
                ctx.debug_k = k;
                return ctx.sync();
            }
            PSK_TRY(trace_push_hashed(ctx, level, width, n, n1, k, red));
            ctx.mark("translate", level);
            // heads[c] (c <= k) are the next level's bucket boundaries by name
            PSK_TRY(build_level<uint32_t>(ctx, red, names1, heads, k, n1, sa1, level + 1));
            heads.reset();
            ctx.mark("(back from recursion)", level);
        } else {
            heads.reset();
            if (level == 0 && ctx.debug_red) {
                // all names unique: the reduced string is the name string
                uint64_t c = n1 < ctx.debug_cap ? n1 : ctx.debug_cap;
                PSK_CUDA(cudaMemcpyAsync(ctx.debug_red, red.get(), c * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
                ctx.debug_n1 = n1;
                ctx.debug_k = k;
                return ctx.sync();
            }
            trace_push(ctx, level, width, n, n1, k, 0);
            PSK_TRY(direct_inverse(red, n1, sa1, ctx.d_err, s));
        }
        if constexpr (sizeof(C) == 1) {
            if (engine == PSACAK_ENGINE_BUCKET) {
                // the bucket scans take the list with predecessor windows
                red.reset();
                names1.reset();
                DBuf<uint64_t> plist;
                PSK_TRY(sorted_win.init(ctx, n1));
                PSK_TRY(plist.init(ctx, n1));
                PSK_TRY(permute_lms8(sa1, n1, text, lms, pref, n, plist, sorted_win, ctx.d_err, s));
            }
        }
        // the doubling scans take the list with the LMS positions' symbols
        if (!sorted_win.get()) {
            red.reset();
            names1.reset();
            DBuf<uint64_t> plist;
            PSK_TRY(sorted_sym.init(ctx, n1));
            PSK_TRY(plist.init(ctx, n1));
            PSK_TRY(permute_lms_sym<C>(sa1, n1, text, lms, pref, n, plist, sorted_sym, ctx.d_err, s));
        }
    } else {
        if (level == 0 && ctx.debug_red) {
            ctx.debug_n1 = 0;
            ctx.debug_k = 0;
            return ctx.sync();
        }
        trace_push(ctx, level, width, n, 0, 0, 0);
    }
    red.reset();
    names1.reset();
    ctx.mark("permute", level);

    // Stage 3: induce the whole suffix array from the sorted LMS suffixes.
    if constexpr (sizeof(C) == 1) {
        if (engine == PSACAK_ENGINE_BUCKET) {
            sa1.reset();
            return induce_bucket8(ctx, text, n, lms, hg, dgeom.get(), INDUCE_FINAL, sorted_win, n1, sa, s);
        }
        sa1.reset();
        return induce_doubling<C>(ctx, text, n, types, lms, geom, 256, INDUCE_FINAL, sorted_sym, n1, nullptr, sa, s);
    } else {
        sa1.reset();
        return induce_doubling<C>(ctx, text, n, types, lms, geom, nbuckets, INDUCE_FINAL, sorted_sym, n1, nullptr, sa,
                                  s);
    }
}

template status_t build_level<uint8_t>(Ctx &, const uint8_t *, const uint32_t *, const uint32_t *, uint64_t, uint64_t,
                                       uint32_t *, uint32_t);

status_t build_batch(Ctx &ctx, const uint8_t *d_texts, const uint64_t *h_off, uint32_t ntexts, uint32_t *d_sas);

// ---------------------------------------------------------------------------
// translate_sample on the device (src/psacak32.rs:912-943): the distinct
// symbols in order give buckets; an L-type symbol becomes its bucket head
// (count of smaller symbols), an S-type one its bucket tail - 1.
// ---------------------------------------------------------------------------
__global__ void k_iota(uint32_t *v, uint64_t n) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        v[i] = (uint32_t)i;
}
__global__ void k_copy_u32(const uint32_t *a, uint32_t *b, uint64_t n) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        b[i] = a[i];
}
struct HeadLoad {
    const uint32_t *vals;
    __device__ __forceinline__ uint32_t operator()(uint64_t i) const {
        return (i == 0 || vals[i] != vals[i - 1]) ? (uint32_t)(i + 1) : 0u;
    }
};
struct HeadStore {
    uint32_t *head;
    __device__ __forceinline__ void operator()(uint64_t i, uint32_t excl, uint32_t v) const {
        head[i] = (excl > v ? excl : v) - 1;
    }
};
struct TailLoad {  // reversed index r = n - 1 - i; marks the last item of a group
    const uint32_t *vals;
    uint64_t n;
    __device__ __forceinline__ uint32_t operator()(uint64_t r) const {
        uint64_t i = n - 1 - r;
        return (i + 1 == n || vals[i + 1] != vals[i]) ? (uint32_t)(r + 1) : 0u;
    }
};
struct TailStore {
    const uint32_t *vals, *pos, *head, *types;
    uint64_t n;
    uint32_t *out;
    __device__ __forceinline__ void operator()(uint64_t r, uint32_t excl, uint32_t v) const {
        uint32_t inc = excl > v ? excl : v;
        uint64_t i = n - 1 - r;
        uint32_t tail = (uint32_t)(n - inc + 1);  // one past the last index of the group
        uint32_t p = pos[i];
        out[p] = bm_get(types, p) ? tail - 1 : head[i];
    }
};
// index i starts a run of equal sorted symbols (i == n closes the last one)
struct DistinctPred {
    const uint32_t *vals;
    uint64_t n;
    __device__ __forceinline__ bool operator()(uint64_t i) const {
        return i == n || i == 0 || vals[i] != vals[i - 1];
    }
};
struct HeadEmit {
    uint32_t *heads;
    uint64_t n;
    uint32_t distinct;
    __device__ __forceinline__ void operator()(uint64_t i, uint32_t slot) const {
        if (slot <= distinct) heads[slot] = (uint32_t)i;
    }
};
struct DistinctLoad {
    const uint32_t *vals;
    __device__ __forceinline__ uint32_t operator()(uint64_t i) const {
        return (i == 0 || vals[i] != vals[i - 1]) ? 1u : 0u;
    }
};
// names[p] = rank of the symbol at p among the distinct symbols.
struct RankStore {
    const uint32_t *pos;
    uint32_t *names;
    __device__ __forceinline__ void operator()(uint64_t i, uint32_t excl, uint32_t v) const {
        names[pos[i]] = excl + v - 1;
    }
};

status_t build_psacak32(Ctx &ctx, const uint32_t *text, uint64_t n, uint32_t *sa) {
    cudaStream_t s = ctx.stream;
    if (n == 0) return PSACAK_OK;
    PSK_TRY(ctx.checkpoint());
    DBuf<uint32_t> k0, v0, k1, v1;
    PSK_TRY(k0.init(ctx, n));
    PSK_TRY(v0.init(ctx, n));
    PSK_TRY(k1.init(ctx, n));
    PSK_TRY(v1.init(ctx, n));
    k_copy_u32<<<grid_for(n), 256, 0, s>>>(text, k0, n);
    PSK_KCOUNT();
    k_iota<<<grid_for(n), 256, 0, s>>>(v0, n);
    PSK_KCOUNT();
    PSK_LAUNCH_CHECK();
    int in1 = 0;
    PSK_TRY((ctx.radix_sort<uint32_t, uint32_t>(k0, v0, k1, v1, n, 0, 32, &in1)));
    const uint32_t *vals = in1 ? k1.get() : k0.get();
    const uint32_t *pos = in1 ? v1.get() : v0.get();
    DBuf<uint32_t> names;
    PSK_TRY(names.init(ctx, n));
    PSK_TRY((ctx.scan<uint32_t, OpSum<uint32_t>>(DistinctLoad{vals}, RankStore{pos, names}, n, ctx.d_scalars + 3,
                                                 OpSum<uint32_t>(), "scan_ranks")));
    uint32_t distinct = 0;
    PSK_TRY(ctx.read_u32(ctx.d_scalars + 3, &distinct));
    if (distinct >= n) {
        // all symbols distinct: the suffix order is the symbol order.
        k_copy_u32<<<grid_for(n), 256, 0, s>>>(pos, sa, n);
        PSK_KCOUNT();
        PSK_LAUNCH_CHECK();
        trace_push(ctx, 0, 4, n, 0, 0, 0);
        return PSACAK_OK;
    }
    const uint64_t nwords = ceil_div(n, 32);
    DBuf<uint32_t> types, lms, wcnt, tscratch, head, t2;
    PSK_TRY(types.init(ctx, nwords + 1));
    PSK_TRY(lms.init(ctx, nwords + 1));
    PSK_TRY(wcnt.init(ctx, nwords + 1));
    PSK_TRY(tscratch.init(ctx, 2 * ceil_div(n, TYPE_TILE) + 1024));
    PSK_TRY(ctx.ensure_scan(n));
    PSK_TRY(type_text<uint32_t>(text, n, types, lms, wcnt, nullptr, tscratch, ctx.scan_env(), ctx.scan_ctas, s));
    PSK_TRY(head.init(ctx, n));
    PSK_TRY(t2.init(ctx, n));
    PSK_TRY((ctx.scan<uint32_t, OpMax<uint32_t>>(HeadLoad{vals}, HeadStore{head}, n, (uint32_t *)nullptr,
                                                 OpMax<uint32_t>(), "scan_heads")));
    PSK_TRY((ctx.scan<uint32_t, OpMax<uint32_t>>(TailLoad{vals, n}, TailStore{vals, pos, head, types, n, t2}, n,
                                                 (uint32_t *)nullptr, OpMax<uint32_t>(), "scan_tails")));
    types.reset();
    lms.reset();
    wcnt.reset();
    tscratch.reset();
    head.reset();
    k0.reset();
    v0.reset();
    k1.reset();
    v1.reset();
    // bucket boundaries by symbol rank
    DBuf<uint32_t> bheads;
    PSK_TRY(bheads.init(ctx, (uint64_t)distinct + 1));
    PSK_TRY(ctx.compact(DistinctPred{vals, n}, HeadEmit{bheads, n, distinct}, n + 1, ctx.d_scalars + 5, "bucket_heads"));
    return build_level<uint32_t>(ctx, t2, names, bheads, distinct, n, sa, 0);
}

status_t ctx_init(Ctx &c, int device) {
    PSK_CUDA(cudaSetDevice(device));
    c.dev.id = device;
    cudaDeviceProp prop;
    PSK_CUDA(cudaGetDeviceProperties(&prop, device));
    c.dev.num_sms = prop.multiProcessorCount;
    c.dev.smem_optin = prop.sharedMemPerBlockOptin;
    PSK_CUDA(cudaStreamCreateWithFlags(&c.own_stream, cudaStreamNonBlocking));
    c.stream = c.own_stream;
    // A pool of the context's own (the device's default pool, shared with the
    // application, keeps its settings): it keeps freed memory for reuse
    // within a build and is trimmed whenever the arena is regrown.
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    PSK_CUDA(cudaMemPoolCreate(&c.pool, &props));
    uint64_t thresh = UINT64_MAX;
    PSK_CUDA(cudaMemPoolSetAttribute(c.pool, cudaMemPoolAttrReleaseThreshold, &thresh));
    PSK_CUDA(cudaHostAlloc(&c.h_pinned, 4096, cudaHostAllocMapped));
    PSK_CUDA(cudaHostAlloc(&c.h_hist, RADIX_MAX_PASSES * 256 * sizeof(uint32_t), cudaHostAllocMapped));
    PSK_CUDA(cudaHostGetDevicePointer(&c.m_pinned, c.h_pinned, 0));
    PSK_CUDA(cudaHostGetDevicePointer(&c.m_hist, c.h_hist, 0));
    PSK_CUDA(cudaMalloc(&c.os.tickets, 64 * sizeof(uint32_t)));
    PSK_CUDA(cudaMalloc(&c.d_hist, 256 * RADIX_MAX_CTAS * sizeof(uint32_t)));
    PSK_CUDA(cudaMalloc(&c.d_scalars, 64 * sizeof(uint32_t)));
    // error word + wait-limit override (common.cuh)
    PSK_CUDA(cudaMalloc(&c.d_err, 2 * sizeof(uint32_t)));
    PSK_CUDA(cudaMemset(c.d_err, 0, 2 * sizeof(uint32_t)));
    PSK_CUDA(cudaMalloc(&c.d_hashes, Ctx::HASH_SLOTS * sizeof(unsigned long long)));
    PSK_CUDA(cudaMalloc(&c.d_induced, 2 * sizeof(unsigned long long)));
    PSK_CUDA(cudaMemset(c.d_induced, 0, 2 * sizeof(unsigned long long)));
    c.scan_ctas = 4 * (uint32_t)c.dev.num_sms;
    c.radix_ctas = 4 * (uint32_t)c.dev.num_sms;
    if (c.scan_ctas > MAX_CHUNKS) c.scan_ctas = MAX_CHUNKS;
    if (c.radix_ctas > RADIX_MAX_CTAS) c.radix_ctas = RADIX_MAX_CTAS;
    return PSACAK_OK;
}

void ctx_free(Ctx &c) {
    if (c.h_pinned) cudaFreeHost(c.h_pinned);
    if (c.h_hist) cudaFreeHost(c.h_hist);
    if (c.os.tickets) cudaFree(c.os.tickets);
    if (c.os.status) cudaFree(c.os.status);
    c.os.status = nullptr;
    if (c.ss.flags) cudaFree(c.ss.flags);
    c.ss.flags = nullptr;
    c.ss.max_tiles = 0;
    c.os.tickets = nullptr;
    c.h_hist = nullptr;
    c.m_hist = nullptr;
    c.m_pinned = nullptr;
    if (c.d_hist) cudaFree(c.d_hist);
    if (c.d_scalars) cudaFree(c.d_scalars);
    if (c.d_err) cudaFree(c.d_err);
    if (c.d_induced) cudaFree(c.d_induced);
    if (c.d_hashes) cudaFree(c.d_hashes);
    c.d_hashes = nullptr;
    if (c.arena) cudaFree(c.arena);
    c.arena = nullptr;
    if (c.own_stream) cudaStreamSynchronize(c.own_stream);
    if (c.pool) cudaMemPoolDestroy(c.pool);
    c.pool = nullptr;
    if (c.own_stream) cudaStreamDestroy(c.own_stream);
    if (c.copy_stream) {
        cudaStreamSynchronize(c.copy_stream);
        cudaStreamDestroy(c.copy_stream);
    }
    if (c.copy_ev) cudaEventDestroy(c.copy_ev);
    c.copy_stream = nullptr;
    c.copy_ev = nullptr;
    host_stage_free(c);
    c.h_pinned = nullptr;
}

// `width`: symbol width of the input (1 = bytes, 4 = integer symbols), which
// picks the default cut-off of a NULL schedule.
static void apply_schedule(Ctx &c, const psacak_schedule *sched, int width) {
    psacak_schedule d{};
    if (sched) d = *sched;
    else {
        // short texts and reduced strings under 1 Gi symbols by prefix
        // doubling (fewer round trips than recursion), 16-item tiles
        d.finish_below = width == 1 ? PSACAK_DEFAULT_FINISH_BELOW : PSACAK_DEFAULT_FINISH_BELOW32;
        d.inner_finish_below = PSACAK_DEFAULT_INNER_FINISH_BELOW;
        d.tile_items = PSACAK_DEFAULT_TILE_ITEMS;
    }
    c.sched = d;
    uint32_t per = d.scan_ctas_per_sm ? d.scan_ctas_per_sm : 4;
    c.scan_ctas = per * (uint32_t)c.dev.num_sms;
    if (c.scan_ctas > MAX_CHUNKS) c.scan_ctas = MAX_CHUNKS;
    c.radix_ctas = 4 * (uint32_t)c.dev.num_sms;
    if (c.radix_ctas > RADIX_MAX_CTAS) c.radix_ctas = RADIX_MAX_CTAS;
}

// Common body of the device-pointer entry points.
// Sets the thread's profiler hook for the duration of one public call.
struct ProfGuard {
    Ctx &c;
    explicit ProfGuard(Ctx &cc) : c(cc) { t_prof = c.profiling ? &c.prof : nullptr; }
    ~ProfGuard() { t_prof = nullptr; }
};

// The bucket scans count their scattered entries on the device in every
// build; a profiled call starts that count from zero so that it covers its
// own build only.
static status_t profile_begin(Ctx &c) {
    if (c.profiling) PSK_CUDA(cudaMemsetAsync(c.d_induced, 0, sizeof(unsigned long long), c.stream));
    return PSACAK_OK;
}

// Folds the device-side count of entries scattered by the bucket scans into
// the "induce_scatter" class (per entry: the entry and its predecessor
// window written, 8 bytes, and one text byte read in front of it).
static status_t profile_collect(Ctx &c) {
    if (!c.profiling) return PSACAK_OK;
    c.prof.resolve();
    uint32_t h[2];
    PSK_TRY(c.read_u32((const uint32_t *)c.d_induced, h, 2));
    PSK_CUDA(cudaMemsetAsync(c.d_induced, 0, sizeof(unsigned long long), c.stream));
    unsigned long long induced = ((unsigned long long)h[1] << 32) | h[0];
    if (induced) {
        int cls = c.prof.cls_of("induce_scatter");
        c.prof.stats[cls].bytes += 9ull * induced;
    }
    return PSACAK_OK;
}

template <class C>
status_t run_dev(Ctx &c, const C *d_text, uint64_t n, uint32_t *d_sa, cudaStream_t stream,
                 const psacak_schedule *sched) {
    PSK_CUDA(cudaSetDevice(c.dev.id));
    c.stream = stream ? stream : c.own_stream;
    apply_schedule(c, sched, (int)sizeof(C));
    c.trace.clear();
    c.pending_hash.clear();
    PSK_TRY(c.arena_prepare());
    {
        const char *e = getenv("PSACAK_STAGE_TIMES");
        c.stage_timing = e && e[0] == '1';
        c.stage_t0 = 0;
    }
    ProfGuard pg(c);
    PSK_TRY(profile_begin(c));
    status_t st;
    if constexpr (sizeof(C) == 1) st = build_level<uint8_t>(c, d_text, nullptr, nullptr, 256, n, d_sa, 0);
    else st = build_psacak32(c, d_text, n, d_sa);
    if (st != PSACAK_OK) return c.fail(st);
    c.mark("final induce (level 0)", 0);
    PSK_TRY(c.sync());
    PSK_TRY(c.check_device_error());
    PSK_TRY(c.resolve_trace());
    PSK_TRY(profile_collect(c));
    return PSACAK_OK;
}

// Pageable outputs at least this long are drained during the final scans
// (shorter ones are copied after the build, where a host thread would cost
// more than it hides).
constexpr uint64_t PAGEABLE_SINK_MIN = 32ull << 20;

template <class C>
status_t run_host(Ctx &c, const C *text, uint64_t n, uint32_t *sa, const psacak_schedule *sched) {
    PSK_CUDA(cudaSetDevice(c.dev.id));
    c.stream = c.own_stream;
    PSK_TRY(c.arena_prepare());
    DBuf<C> dt;
    DBuf<uint32_t> ds;
    PSK_TRY(dt.init(c, n));
    PSK_TRY(ds.init(c, n));
    if (n) {
        if (host_is_pinned(text))
            PSK_CUDA(cudaMemcpyAsync(dt.get(), text, n * sizeof(C), cudaMemcpyHostToDevice, c.stream));
        else
            PSK_TRY(staged_upload(c, (char *)dt.get(), {HostPiece{(char *)text, 0, n * sizeof(C)}}, c.stream));
    }
    // A pinned output buffer receives the byte-level SA bucket part by bucket
    // part during the final scans (Ctx::sink_part); pageable memory would
    // make each of those copies wait for itself on the host, so it is filled
    // through the staging ring after the build.
    const bool out_pinned = n && host_is_pinned(sa);
    bool sink = false, drain = false;
    if (sizeof(C) == 1 && n && (out_pinned || n >= PAGEABLE_SINK_MIN)) {
        if (!c.copy_stream) PSK_CUDA(cudaStreamCreateWithFlags(&c.copy_stream, cudaStreamNonBlocking));
        if (!c.copy_ev) PSK_CUDA(cudaEventCreateWithFlags(&c.copy_ev, cudaEventDisableTiming));
        if (!out_pinned) {
            // pageable: a host thread drains the parts through the staging ring
            PSK_TRY(drain_begin(c, sa, ds.get()));
            c.sink_pageable = true;
            drain = true;
        }
        c.sink_dev = ds.get();
        c.sink_host = sa;
        sink = true;
    }
    c.sink_done = false;
    const status_t st = run_dev<C>(c, dt.get(), n, ds.get(), c.own_stream, sched);
    c.sink_dev = c.sink_host = nullptr;
    c.sink_pageable = false;
    const status_t dst = drain ? drain_end(c) : PSACAK_OK;
    if (sink) PSK_CUDA(cudaStreamSynchronize(c.copy_stream));  // before ds goes back to the arena
    PSK_TRY(st);
    PSK_TRY(dst);
    if (n && !c.sink_done) {
        if (out_pinned)
            PSK_CUDA(cudaMemcpyAsync(sa, ds.get(), n * sizeof(uint32_t), cudaMemcpyDeviceToHost, c.stream));
        else
            PSK_TRY(staged_download(c, (const char *)ds.get(), {HostPiece{(char *)sa, 0, n * sizeof(uint32_t)}},
                                    c.stream));
    }
    dt.reset();
    ds.reset();
    PSK_TRY(c.sync());
    return PSACAK_OK;
}

}  // namespace psk

using namespace psk;

static thread_local psacak_ctx *t_default_ctx = nullptr;
static thread_local int t_default_device = 0;

static int default_ctx(psacak_ctx **out) {
    if (!t_default_ctx) {
        int rc = psacak_ctx_create(t_default_device, &t_default_ctx);
        if (rc != PSACAK_OK) return rc;
    }
    *out = t_default_ctx;
    return PSACAK_OK;
}

extern "C" {

const char *psacak_version(void) { return "0.1.0"; }

int psacak_init(int device) {
    clear_error();
    if (device < 0) return set_error(PSACAK_EINVAL, "psacak_init: device %d", device);
    int count = 0;
    PSK_CUDA(cudaGetDeviceCount(&count));
    if (device >= count) return set_error(PSACAK_EINVAL, "psacak_init: device %d of %d", device, count);
    if (t_default_ctx && t_default_ctx->c.dev.id != device) {
        psacak_ctx_destroy(t_default_ctx);
        t_default_ctx = nullptr;
    }
    t_default_device = device;
    psacak_ctx *c = nullptr;
    return default_ctx(&c);
}

int psacak_shutdown(void) {
    clear_error();
    if (t_default_ctx) psacak_ctx_destroy(t_default_ctx);
    t_default_ctx = nullptr;
    return PSACAK_OK;
}

const char *psacak_last_error_string(void) { return last_error(); }

int psacak_ctx_create(int device, psacak_ctx **out) {
    clear_error();
    if (!out) return set_error(PSACAK_EINVAL, "psacak_ctx_create: null output pointer");
    std::unique_ptr<psacak_ctx> c(new (std::nothrow) psacak_ctx());
    if (!c) return set_error(PSACAK_ENOMEM, "psacak_ctx_create: out of host memory");
    int rc = ctx_init(c->c, device);
    if (rc != PSACAK_OK) {
        ctx_free(c->c);
        return rc;
    }
    *out = c.release();
    return PSACAK_OK;
}

int psacak_ctx_destroy(psacak_ctx *ctx) {
    if (!ctx) return PSACAK_OK;
    if (t_default_ctx == ctx) t_default_ctx = nullptr;
    {
        std::lock_guard<std::mutex> g(ctx->c.mu);
        cudaSetDevice(ctx->c.dev.id);
        cudaStreamSynchronize(ctx->c.own_stream);
        ctx_free(ctx->c);
    }
    delete ctx;
    return PSACAK_OK;
}

static int check_args8(const void *text, uint64_t n, const void *sa) {
    if (n > 0 && (!text || !sa)) return set_error(PSACAK_EINVAL, "null text or suffix-array pointer");
    if (n >= 0xFFFFFFFFull) return set_error(PSACAK_EINVAL, "text length %llu is not below 2^32-1", (unsigned long long)n);
    return PSACAK_OK;
}
static int check_args32(const void *text, uint64_t n, const void *sa) {
    if (n > 0 && (!text || !sa)) return set_error(PSACAK_EINVAL, "null text or suffix-array pointer");
    if (n > 0x7FFFFFFFull) return set_error(PSACAK_EINVAL, "text length %llu exceeds 2^31-1", (unsigned long long)n);
    return PSACAK_OK;
}

int psacak8_ctx(psacak_ctx *ctx, const uint8_t *text, uint64_t n, uint32_t *sa, const psacak_schedule *sched) {
    clear_error();
    if (!ctx) return set_error(PSACAK_EINVAL, "null context");
    int rc = check_args8(text, n, sa);
    if (rc) return rc;
    std::lock_guard<std::mutex> g(ctx->c.mu);
    return run_host<uint8_t>(ctx->c, text, n, sa, sched);
}

int psacak32_ctx(psacak_ctx *ctx, const uint32_t *text, uint64_t n, uint32_t *sa, const psacak_schedule *sched) {
    clear_error();
    if (!ctx) return set_error(PSACAK_EINVAL, "null context");
    int rc = check_args32(text, n, sa);
    if (rc) return rc;
    std::lock_guard<std::mutex> g(ctx->c.mu);
    return run_host<uint32_t>(ctx->c, text, n, sa, sched);
}

int psacak8(const uint8_t *text, uint64_t n, uint32_t *sa) {
    clear_error();
    int rc = check_args8(text, n, sa);
    if (rc) return rc;
    psacak_ctx *c = nullptr;
    rc = default_ctx(&c);
    if (rc) return rc;
    return psacak8_ctx(c, text, n, sa, nullptr);
}

int psacak32(const uint32_t *text, uint64_t n, uint32_t *sa) {
    clear_error();
    int rc = check_args32(text, n, sa);
    if (rc) return rc;
    psacak_ctx *c = nullptr;
    rc = default_ctx(&c);
    if (rc) return rc;
    return psacak32_ctx(c, text, n, sa, nullptr);
}

int psacak8_dev(psacak_ctx *ctx, const uint8_t *d_text, uint64_t n, uint32_t *d_sa, void *stream,
                const psacak_schedule *sched) {
    clear_error();
    if (!ctx) return set_error(PSACAK_EINVAL, "null context");
    int rc = check_args8(d_text, n, d_sa);
    if (rc) return rc;
    std::lock_guard<std::mutex> g(ctx->c.mu);
    return run_dev<uint8_t>(ctx->c, d_text, n, d_sa, (cudaStream_t)stream, sched);
}

int psacak32_dev(psacak_ctx *ctx, const uint32_t *d_text, uint64_t n, uint32_t *d_sa, void *stream,
                 const psacak_schedule *sched) {
    clear_error();
    if (!ctx) return set_error(PSACAK_EINVAL, "null context");
    int rc = check_args32(d_text, n, d_sa);
    if (rc) return rc;
    std::lock_guard<std::mutex> g(ctx->c.mu);
    return run_dev<uint32_t>(ctx->c, d_text, n, d_sa, (cudaStream_t)stream, sched);
}

int psacak_cancel(psacak_ctx *ctx) {
    if (!ctx) return set_error(PSACAK_EINVAL, "null context");
    ctx->c.cancel_req.store(1);
    return PSACAK_OK;
}

int psacak_get_trace(psacak_ctx *ctx, psacak_level_info *out, uint32_t cap, uint32_t *count) {
    if (!ctx) return set_error(PSACAK_EINVAL, "null context");
    std::lock_guard<std::mutex> g(ctx->c.mu);
    uint32_t n = (uint32_t)ctx->c.trace.size();
    for (uint32_t i = 0; i < n && i < cap && out; i++) out[i] = ctx->c.trace[i];
    if (count) *count = n;
    return PSACAK_OK;
}

}  // extern "C"

template <class C>
static int check_dev(psacak_ctx *ctx, const C *d_text, uint64_t n, const uint32_t *d_sa, int *ok, void *stream) {
    clear_error();
    if (!ctx || !ok) return set_error(PSACAK_EINVAL, "null context or result pointer");
    if (n > 0 && (!d_text || !d_sa)) return set_error(PSACAK_EINVAL, "null text or suffix-array pointer");
    std::lock_guard<std::mutex> g(ctx->c.mu);
    Ctx &c = ctx->c;
    PSK_CUDA(cudaSetDevice(c.dev.id));
    c.stream = stream ? (cudaStream_t)stream : c.own_stream;
    DBuf<uint32_t> isa;
    PSK_TRY(isa.init(c, n));
    PSK_TRY(check_sa<C>(d_text, n, d_sa, isa, c.d_scalars + 40, c.stream));
    uint32_t bad = 0;
    PSK_TRY(c.read_u32(c.d_scalars + 40, &bad));
    *ok = bad == 0;
    return PSACAK_OK;
}

extern "C" {

int psacak_check_sa8_dev(psacak_ctx *ctx, const uint8_t *d_text, uint64_t n, const uint32_t *d_sa, int *ok,
                         void *stream) {
    return check_dev<uint8_t>(ctx, d_text, n, d_sa, ok, stream);
}

int psacak_check_sa32_dev(psacak_ctx *ctx, const uint32_t *d_text, uint64_t n, const uint32_t *d_sa, int *ok,
                          void *stream) {
    return check_dev<uint32_t>(ctx, d_text, n, d_sa, ok, stream);
}

int psacak_profile_enable(psacak_ctx *ctx, int on) {
    if (!ctx) return set_error(PSACAK_EINVAL, "null context");
    std::lock_guard<std::mutex> g(ctx->c.mu);
    ctx->c.profiling = on != 0;
    return PSACAK_OK;
}

int psacak_profile_reset(psacak_ctx *ctx) {
    if (!ctx) return set_error(PSACAK_EINVAL, "null context");
    std::lock_guard<std::mutex> g(ctx->c.mu);
    ctx->c.prof.reset();
    return PSACAK_OK;
}

int psacak_profile_get(psacak_ctx *ctx, psacak_kernel_stat *out, uint32_t cap, uint32_t *count) {
    if (!ctx) return set_error(PSACAK_EINVAL, "null context");
    std::lock_guard<std::mutex> g(ctx->c.mu);
    const auto &st = ctx->c.prof.stats;
    uint32_t n = (uint32_t)st.size();
    for (uint32_t i = 0; i < n && i < cap && out; i++) {
        memset(&out[i], 0, sizeof(out[i]));
        strncpy(out[i].name, st[i].name, sizeof(out[i].name) - 1);
        out[i].launches = st[i].launches;
        out[i].items = st[i].items;
        out[i].bytes = st[i].bytes;
        out[i].ms = st[i].ms;
    }
    if (count) *count = n;
    return PSACAK_OK;
}

uint64_t psacak_kernel_launches(psacak_ctx *ctx) {
    (void)ctx;
    return g_kernel_launches.load();
}

uint64_t psacak_round_trips(psacak_ctx *ctx) {
    (void)ctx;
    return g_round_trips.load();
}

int psacak8_batch_dev(psacak_ctx *ctx, const uint8_t *d_texts, const uint64_t *offsets, uint32_t n_texts,
                      uint32_t *d_sas, void *stream, const psacak_schedule *sched) {
    clear_error();
    if (!ctx) return set_error(PSACAK_EINVAL, "null context");
    if (n_texts > 0 && (!offsets || !d_texts || !d_sas)) return set_error(PSACAK_EINVAL, "null batch pointers");
    for (uint32_t i = 0; i < n_texts; i++)
        if (offsets[i + 1] < offsets[i]) return set_error(PSACAK_EINVAL, "batch offsets decrease at text %u", i);
    std::lock_guard<std::mutex> g(ctx->c.mu);
    Ctx &c = ctx->c;
    PSK_CUDA(cudaSetDevice(c.dev.id));
    c.stream = stream ? (cudaStream_t)stream : c.own_stream;
    apply_schedule(c, sched, 1);
    c.trace.clear();
    c.pending_hash.clear();
    PSK_TRY(c.arena_prepare());
    ProfGuard pg(c);
    PSK_TRY(profile_begin(c));
    status_t st = build_batch(c, d_texts, offsets, n_texts, d_sas);
    if (st != PSACAK_OK) return c.fail(st);
    PSK_TRY(c.sync());
    PSK_TRY(c.check_device_error());
    PSK_TRY(c.resolve_trace());
    PSK_TRY(profile_collect(c));
    return PSACAK_OK;
}

int psacak8_batch(psacak_ctx *ctx, const uint8_t *const *texts, const uint64_t *lens, uint32_t n_texts,
                  uint32_t *const *sas, const psacak_schedule *sched) {
    clear_error();
    if (!ctx) return set_error(PSACAK_EINVAL, "null context");
    if (n_texts > 0 && (!texts || !lens || !sas)) return set_error(PSACAK_EINVAL, "null batch arrays");
    std::vector<uint64_t> off(n_texts + 1, 0);
    for (uint32_t i = 0; i < n_texts; i++) {
        if (lens[i] > 0 && (!texts[i] || !sas[i])) return set_error(PSACAK_EINVAL, "null text or SA %u", i);
        off[i + 1] = off[i] + lens[i];
    }
    if (off[n_texts] == 0) return PSACAK_OK;
    Ctx &c = ctx->c;
    status_t st;
    {
        std::lock_guard<std::mutex> g(c.mu);
        PSK_CUDA(cudaSetDevice(c.dev.id));
        c.stream = c.own_stream;
        PSK_TRY(c.arena_prepare());
    }
    uint8_t *dt = nullptr;
    uint32_t *ds = nullptr;
    PSK_CUDA(cudaMallocFromPoolAsync(&dt, off[n_texts], c.pool, c.own_stream));
    st = cudaMallocFromPoolAsync(&ds, off[n_texts] * sizeof(uint32_t), c.pool, c.own_stream) == cudaSuccess
             ? PSACAK_OK
             : PSACAK_ENOMEM;
    if (st == PSACAK_OK) {
        // pinned buffers are copied directly; any pageable one sends the
        // whole batch through the staging ring (hostio.cuh)
        std::vector<HostPiece> tp, sp;
        bool t_pinned = true, s_pinned = true;
        for (uint32_t i = 0; i < n_texts; i++) {
            if (!lens[i]) continue;
            tp.push_back(HostPiece{(char *)texts[i], off[i], lens[i]});
            sp.push_back(HostPiece{(char *)sas[i], off[i] * sizeof(uint32_t), lens[i] * sizeof(uint32_t)});
            t_pinned = t_pinned && host_is_pinned(texts[i]);
            s_pinned = s_pinned && host_is_pinned(sas[i]);
        }
        {
            std::lock_guard<std::mutex> g(c.mu);
            if (!t_pinned) {
                st = staged_upload(c, (char *)dt, tp, c.own_stream);
            } else {
                for (const HostPiece &p : tp)
                    if (st == PSACAK_OK &&
                        cudaMemcpyAsync(dt + p.dev_off, p.host, p.bytes, cudaMemcpyHostToDevice, c.own_stream) !=
                            cudaSuccess)
                        st = set_error(PSACAK_ECUDA, "batch upload failed");
            }
        }
        if (st == PSACAK_OK) st = psacak8_batch_dev(ctx, dt, off.data(), n_texts, ds, c.own_stream, sched);
        if (st == PSACAK_OK) {
            std::lock_guard<std::mutex> g(c.mu);
            if (!s_pinned) {
                st = staged_download(c, (const char *)ds, sp, c.own_stream);
            } else {
                for (const HostPiece &p : sp)
                    if (st == PSACAK_OK &&
                        cudaMemcpyAsync(p.host, (const char *)ds + p.dev_off, p.bytes, cudaMemcpyDeviceToHost,
                                        c.own_stream) != cudaSuccess)
                        st = set_error(PSACAK_ECUDA, "batch download failed");
            }
        }
    } else {
        set_error(PSACAK_ENOMEM, "batch: device allocation failed");
    }
    cudaStreamSynchronize(c.own_stream);
    if (dt) cudaFreeAsync(dt, c.own_stream);
    if (ds) cudaFreeAsync(ds, c.own_stream);
    cudaStreamSynchronize(c.own_stream);
    return st;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Debug / stage entry points (include/psacak_b200_debug.h).
// ---------------------------------------------------------------------------
__global__ void k_copy_u64(const uint64_t *a, uint64_t *b, uint64_t n) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        b[i] = a[i];
}
struct CopyLoad {
    const uint32_t *in;
    __device__ __forceinline__ uint32_t operator()(uint64_t i) const { return in[i]; }
};
struct CopyStore {
    uint32_t *out;
    __device__ __forceinline__ void operator()(uint64_t i, uint32_t excl, uint32_t) const { out[i] = excl; }
};

template <class K>
static int debug_sort(psacak_ctx *ctx, K *keys, uint32_t *vals, uint64_t n, int b0, int b1) {
    clear_error();
    if (!ctx) return set_error(PSACAK_EINVAL, "null context");
    std::lock_guard<std::mutex> g(ctx->c.mu);
    Ctx &c = ctx->c;
    PSK_CUDA(cudaSetDevice(c.dev.id));
    c.stream = c.own_stream;
    DBuf<K> k1;
    DBuf<uint32_t> v1;
    PSK_TRY(k1.init(c, n));
    PSK_TRY(v1.init(c, n));
    int in1 = 0;
    PSK_TRY((c.radix_sort<K, uint32_t>(keys, vals, k1, v1, n, b0, b1, &in1)));
    if (in1) {
        PSK_CUDA(cudaMemcpyAsync(keys, k1.get(), n * sizeof(K), cudaMemcpyDeviceToDevice, c.stream));
        PSK_CUDA(cudaMemcpyAsync(vals, v1.get(), n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, c.stream));
    }
    k1.reset();
    v1.reset();
    PSK_TRY(c.sync());
    return c.check_device_error();
}

extern "C" {

int psacak_debug_radix_sort_u64(psacak_ctx *ctx, uint64_t *d_keys, uint32_t *d_vals, uint64_t n, int begin_bit,
                                int end_bit) {
    return debug_sort<uint64_t>(ctx, d_keys, d_vals, n, begin_bit, end_bit);
}

int psacak_debug_radix_sort_u32(psacak_ctx *ctx, uint32_t *d_keys, uint32_t *d_vals, uint64_t n, int begin_bit,
                                int end_bit) {
    return debug_sort<uint32_t>(ctx, d_keys, d_vals, n, begin_bit, end_bit);
}

int psacak_debug_exclusive_sum(psacak_ctx *ctx, const uint32_t *d_in, uint32_t *d_out, uint64_t n) {
    clear_error();
    if (!ctx) return set_error(PSACAK_EINVAL, "null context");
    std::lock_guard<std::mutex> g(ctx->c.mu);
    Ctx &c = ctx->c;
    PSK_CUDA(cudaSetDevice(c.dev.id));
    c.stream = c.own_stream;
    PSK_TRY((c.scan<uint32_t, OpSum<uint32_t>>(CopyLoad{d_in}, CopyStore{d_out}, n, (uint32_t *)nullptr,
                                               OpSum<uint32_t>(), "scan")));
    return c.sync();
}

int psacak_debug_set_limits(psacak_ctx *ctx, uint32_t spin_limit, uint64_t workspace_cap) {
    clear_error();
    if (!ctx) return set_error(PSACAK_EINVAL, "null context");
    if (spin_limit > 0x80000000u) return set_error(PSACAK_EINVAL, "spin limit %u above 2^31", spin_limit);
    std::lock_guard<std::mutex> g(ctx->c.mu);
    Ctx &c = ctx->c;
    PSK_CUDA(cudaSetDevice(c.dev.id));
    c.ws_cap = workspace_cap;
    PSK_CUDA(cudaMemcpyAsync(c.d_err + 1, &spin_limit, sizeof(uint32_t), cudaMemcpyHostToDevice, c.own_stream));
    PSK_CUDA(cudaStreamSynchronize(c.own_stream));
    return PSACAK_OK;
}

int psacak_debug_stalled_scan(psacak_ctx *ctx, const uint32_t *d_in, uint32_t *d_out, uint64_t n) {
    clear_error();
    if (!ctx || !d_in || !d_out) return set_error(PSACAK_EINVAL, "null argument");
    constexpr uint64_t TILE = (uint64_t)LS_BLOCK * scan_ipt<uint32_t, CopyLoad>();
    const uint64_t ntiles = ceil_div(n, TILE);
    if (ntiles < 2 || ntiles > 0xFFFFFFFFull)
        return set_error(PSACAK_EINVAL, "stalled scan: n = %llu must span 2 tiles of %llu", (unsigned long long)n,
                         (unsigned long long)TILE);
    std::lock_guard<std::mutex> g(ctx->c.mu);
    Ctx &c = ctx->c;
    PSK_CUDA(cudaSetDevice(c.dev.id));
    c.stream = c.own_stream;
    PSK_TRY(c.ensure_scan(n));
    c.os.epoch = (c.os.epoch + 1) & ((1u << 30) - 1);
    if (c.os.epoch == 0) c.os.epoch = 1;
    uint32_t *ticket = c.os.tickets + (c.os.epoch & 63);
    // the ticket starts at 1: tiles 1 .. ntiles-1 are claimed by the
    // ntiles-1 CTAs (all in range), tile 0 by none
    const uint32_t one = 1;
    PSK_CUDA(cudaMemcpyAsync(ticket, &one, sizeof(uint32_t), cudaMemcpyHostToDevice, c.stream));
    k_lbscan<uint32_t, OpSum<uint32_t>, CopyLoad, CopyStore><<<(uint32_t)(ntiles - 1), LS_BLOCK, 0, c.stream>>>(
        CopyLoad{d_in}, CopyStore{d_out}, n, OpSum<uint32_t>(), c.ss.flags, ticket, c.os.epoch, (uint32_t)ntiles,
        (uint32_t *)nullptr, c.d_err, (const uint32_t *)nullptr);
    PSK_KCOUNT();
    PSK_LAUNCH_CHECK();
    PSK_TRY(c.sync());
    return c.check_device_error();
}

int psacak_debug_types(psacak_ctx *ctx, const void *d_text, uint64_t n, int width, uint32_t *d_types,
                       uint32_t *d_lms) {
    clear_error();
    if (!ctx || (width != 1 && width != 4)) return set_error(PSACAK_EINVAL, "bad context or width");
    std::lock_guard<std::mutex> g(ctx->c.mu);
    Ctx &c = ctx->c;
    PSK_CUDA(cudaSetDevice(c.dev.id));
    c.stream = c.own_stream;
    DBuf<uint32_t> wcnt, scr;
    DBuf<ByteHist> hist;
    PSK_TRY(wcnt.init(c, ceil_div(n, 32) + 1));
    PSK_TRY(scr.init(c, 2 * ceil_div(n, TYPE_TILE) + 1024));
    PSK_TRY(hist.init(c, 1));
    PSK_TRY(c.ensure_scan(n));
    if (width == 1)
        PSK_TRY(type_text<uint8_t>((const uint8_t *)d_text, n, d_types, d_lms, wcnt, hist, scr, c.scan_env(),
                                   c.scan_ctas, c.stream));
    else
        PSK_TRY(type_text<uint32_t>((const uint32_t *)d_text, n, d_types, d_lms, wcnt, nullptr, scr, c.scan_env(),
                                    c.scan_ctas, c.stream));
    return c.sync();
}

int psacak_debug_reduced8(psacak_ctx *ctx, const uint8_t *d_text, uint64_t n, uint32_t *d_red, uint64_t cap,
                          uint64_t *n_lms, uint64_t *k, const psacak_schedule *sched) {
    clear_error();
    if (!ctx || !n_lms || !k) return set_error(PSACAK_EINVAL, "null argument");
    std::lock_guard<std::mutex> g(ctx->c.mu);
    Ctx &c = ctx->c;
    PSK_CUDA(cudaSetDevice(c.dev.id));
    c.stream = c.own_stream;
    apply_schedule(c, sched, 1);
    c.trace.clear();
    c.pending_hash.clear();
    c.debug_red = d_red;
    c.debug_cap = cap;
    c.debug_n1 = c.debug_k = 0;
    status_t st = PSACAK_OK;
    if (n > 3) {
        DBuf<uint32_t> sa;
        st = sa.init(c, n);
        if (st == PSACAK_OK) st = build_level<uint8_t>(c, d_text, nullptr, nullptr, 256, n, sa, 0);
    }
    c.debug_red = nullptr;
    if (st != PSACAK_OK) return st;
    *n_lms = c.debug_n1;
    *k = c.debug_k;
    PSK_TRY(c.sync());
    return c.check_device_error();
}

}  // extern "C"
