// batch.cu -- many independent byte texts in one build.
//
// The texts are packed as t_0 $ t_1 $ ... t_{k-1} $ with a separator byte
// smaller than every byte of every text.  A suffix of text i then reads
// t_i[p..] $ ..., and two suffixes of the same text differ inside t_i or one
// of them meets its $ first -- exactly the order of the text alone with its
// implicit smallest sentinel (src/lib.rs:30-43).  One suffix-array build of
// the concatenation therefore sorts the suffixes of every text at once;
// a stable partition of that array by text id (separators dropped) leaves
// each text's suffix array in place at the text's packed offset.
//
// When byte 0 occurs in the batch, the bytes below the smallest unused value
// v are shifted up by one (order-preserving) so that 0 is free; a batch that
// uses all 256 byte values is built text by text.  Batches larger than the
// chunk limit (schedule batch_chunk_mib, and always below 2^32 - 1 bytes)
// are built chunk by chunk.
#include <algorithm>
#include <vector>

#include "ctx.cuh"
#include "induce.cuh"
#include "small.cuh"

namespace psk {

const char *last_error();
void clear_error();

template <class C>
status_t build_level(Ctx &ctx, const C *text, const uint32_t *names, const uint32_t *bheads, uint64_t nbuckets,
                     uint64_t n, uint32_t *sa, uint32_t level);

// 256-bit presence mask of the bytes of [0, n).
__global__ void k_byte_mask(const uint8_t *__restrict__ t, uint64_t n, uint32_t *mask) {
    __shared__ uint32_t sm[8];
    if (threadIdx.x < 8) sm[threadIdx.x] = 0;
    __syncthreads();
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t c = t[i];
        atomicOr(&sm[c >> 5], 1u << (c & 31));
    }
    __syncthreads();
    if (threadIdx.x < 8 && sm[threadIdx.x]) atomicOr(&mask[threadIdx.x], sm[threadIdx.x]);
}

// Index of the text whose packed range [off[i], off[i+1]) holds position p.
__device__ __forceinline__ uint32_t text_of(const uint64_t *__restrict__ off, uint32_t k, uint64_t p) {
    uint32_t lo = 0, hi = k - 1;
    while (lo < hi) {
        uint32_t mid = (lo + hi + 1) >> 1;
        if (off[mid] <= p) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// cat[q] for q in [0, N): text byte (shifted below v) or the separator 0.
// The i-th text of the chunk occupies [coff[i], coff[i+1] - 1) of the
// concatenation, its separator the slot right after; its bytes start at
// src[soff[i]].
__global__ void k_batch_pack(const uint8_t *__restrict__ src, const uint64_t *__restrict__ coff,
                             const uint64_t *__restrict__ soff, uint32_t k, uint64_t N, uint32_t v, uint8_t *cat) {
    for (uint64_t q = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; q < N; q += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t i = text_of(coff, k, q);
        uint64_t p = q - coff[i];
        uint64_t len = coff[i + 1] - coff[i] - 1;
        uint8_t c = 0;
        if (p < len) {
            c = src[soff[i] + p];
            if (c < v) c = (uint8_t)(c + 1);
        }
        cat[q] = c;
    }
}

// The chunk's suffix arrays, back to back in `sorted` (the i-th text's at
// [coff[i] - i, coff[i+1] - i - 1)), to each text's own offset soff[i].
__global__ void k_batch_unpack(const uint32_t *__restrict__ sorted, const uint64_t *__restrict__ xoff,
                               const uint64_t *__restrict__ soff, uint32_t k, uint64_t total, uint32_t *sas) {
    for (uint64_t q = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; q < total;
         q += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t i = text_of(xoff, k, q);
        sas[soff[i] + (q - xoff[i])] = sorted[q];
    }
}

struct SepPred {
    const uint32_t *sa;
    const uint64_t *coff;
    uint32_t k;
    __device__ __forceinline__ bool operator()(uint64_t q) const {
        uint64_t P = sa[q];
        uint32_t i = text_of(coff, k, P);
        return P - coff[i] < coff[i + 1] - coff[i] - 1;
    }
};
struct SepEmit {
    const uint32_t *sa;
    const uint64_t *coff;
    uint32_t k;
    uint32_t *keys, *vals;
    __device__ __forceinline__ void operator()(uint64_t q, uint32_t slot) const {
        uint64_t P = sa[q];
        uint32_t i = text_of(coff, k, P);
        keys[slot] = i;
        vals[slot] = (uint32_t)(P - coff[i]);
    }
};

// One chunk: the texts ids[0 .. k) of the packed device input (text t at
// [h_off[t], h_off[t+1])), SAs to the same packed offsets of d_sas.
static status_t batch_chunk(Ctx &ctx, const uint8_t *d_src, const uint64_t *h_off, const uint32_t *ids, uint32_t k,
                            uint32_t *d_sas, uint32_t v) {
    cudaStream_t s = ctx.stream;
    // host tables: coff (with separators), xoff (without), soff (source offsets)
    std::vector<uint64_t> tab(3 * (size_t)k + 2);
    uint64_t *coff = tab.data(), *xoff = coff + k + 1, *soff = xoff + k + 1;
    bool contiguous = true;
    coff[0] = xoff[0] = 0;
    for (uint32_t i = 0; i < k; i++) {
        const uint64_t len = h_off[ids[i] + 1] - h_off[ids[i]];
        coff[i + 1] = coff[i] + len + 1;
        xoff[i + 1] = xoff[i] + len;
        soff[i] = h_off[ids[i]];
        if (i > 0 && ids[i] != ids[i - 1] + 1) contiguous = false;
    }
    const uint64_t total = xoff[k];
    const uint64_t N = coff[k];
    DBuf<uint64_t> dtab;
    DBuf<uint8_t> cat;
    DBuf<uint32_t> sa, k0, v0, k1, v1;
    PSK_TRY(dtab.init(ctx, tab.size()));
    PSK_CUDA(cudaMemcpyAsync(dtab.get(), tab.data(), tab.size() * sizeof(uint64_t), cudaMemcpyHostToDevice, s));
    const uint64_t *dcoff = dtab.get(), *dxoff = dcoff + k + 1, *dsoff = dxoff + k + 1;
    PSK_TRY(cat.init(ctx, N));
    uint64_t g = ceil_div(N, 256);
    PSK_PROF_LAUNCH(s, "batch_pack", N, 2 * N,
                    (k_batch_pack<<<(uint32_t)(g < 16384 ? g : 16384), 256, 0, s>>>(d_src, dcoff, dsoff, k, N, v,
                                                                                   cat)));
    PSK_TRY(sa.init(ctx, N));
    PSK_TRY(build_level<uint8_t>(ctx, cat.get(), nullptr, nullptr, 256, N, sa, 0));
    // drop the separators, key every suffix by its text
    PSK_TRY(k0.init(ctx, total));
    PSK_TRY(v0.init(ctx, total));
    PSK_TRY(k1.init(ctx, total));
    PSK_TRY(ctx.compact(SepPred{sa, dcoff, k}, SepEmit{sa, dcoff, k, k0, v0}, N, ctx.d_scalars + 12, "batch_split"));
    uint32_t got = 0;
    PSK_TRY(ctx.read_u32(ctx.d_scalars + 12, &got));
    if (got != total) return set_error(PSACAK_EINTERNAL, "batch: %u suffixes after dropping separators, expected %llu",
                                       got, (unsigned long long)total);
    // stable sort by text id: the values become every text's SA in order
    // (written in place when the chunk's texts are adjacent in d_sas)
    int in1 = 0;
    uint32_t *out = d_sas + soff[0];
    if (!contiguous) {
        PSK_TRY(v1.init(ctx, total));
        out = v1.get();
    }
    PSK_TRY((ctx.radix_sort<uint32_t, uint32_t>(k0, v0, k1, out, total, 0, bitlen(k > 1 ? k - 1 : 1), &in1)));
    if (!in1) PSK_CUDA(cudaMemcpyAsync(out, v0.get(), total * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
    if (!contiguous) {
        g = ceil_div(total, 256);
        PSK_PROF_LAUNCH(s, "batch_unpack", total, 8 * total,
                        (k_batch_unpack<<<(uint32_t)(g < 16384 ? g : 16384), 256, 0, s>>>(out, dxoff, dsoff, k, total,
                                                                                        d_sas)));
        PSK_LAUNCH_CHECK();
    }
    return PSACAK_OK;
}

// Device form: texts packed back to back in d_texts (text i in
// [h_off[i], h_off[i+1])), SAs written at the same offsets of d_sas.
// Texts short enough for the direct prefix-doubling finisher (shorter than
// the schedule's finish_below and at most SMALL_MAX bytes) are sorted one
// CTA each in shared memory; the others by one build of their
// concatenation (chunked).
status_t build_batch(Ctx &ctx, const uint8_t *d_texts, const uint64_t *h_off, uint32_t ntexts, uint32_t *d_sas) {
    cudaStream_t s = ctx.stream;
    const uint64_t total = h_off[ntexts] - h_off[0];
    if (total == 0) return PSACAK_OK;
    PSK_TRY(ctx.checkpoint());
    std::vector<uint32_t> small, big;
    for (uint32_t i = 0; i < ntexts; i++) {
        const uint64_t len = h_off[i + 1] - h_off[i];
        if (len == 0) continue;
        if (len <= SMALL_MAX && ctx.sched.finish_below && len < ctx.sched.finish_below) small.push_back(i);
        else big.push_back(i);
    }
    DBuf<uint64_t> d_off;
    DBuf<uint32_t> d_ids;
    if (!small.empty()) {
        std::stable_sort(small.begin(), small.end(), [&](uint32_t a, uint32_t b) {
            return h_off[a + 1] - h_off[a] > h_off[b + 1] - h_off[b];
        });
        PSK_TRY(d_off.init(ctx, (size_t)ntexts + 1));
        PSK_TRY(d_ids.init(ctx, small.size()));
        PSK_CUDA(cudaMemcpyAsync(d_off.get(), h_off, ((size_t)ntexts + 1) * sizeof(uint64_t), cudaMemcpyHostToDevice, s));
        PSK_CUDA(cudaMemcpyAsync(d_ids.get(), small.data(), small.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, s));
        uint64_t symbols = 0;
        for (uint32_t i : small) symbols += h_off[i + 1] - h_off[i];
        PSK_TRY(small_sa<uint8_t>(ctx, d_texts, SmallJobs{d_off.get(), d_ids.get(), (uint32_t)small.size(), 0, symbols}, 256,
                                  d_sas, s));
        // the host tables must outlive the copies
        PSK_CUDA(cudaStreamSynchronize(s));
    }
    if (big.empty()) return PSACAK_OK;
    // which byte values occur?
    uint32_t *mask = ctx.d_scalars + 16;
    PSK_CUDA(cudaMemsetAsync(mask, 0, 8 * sizeof(uint32_t), s));
    uint64_t g = ceil_div(total, 256);
    PSK_PROF_LAUNCH(s, "batch_mask", total, total,
                    (k_byte_mask<<<(uint32_t)(g < 4096 ? g : 4096), 256, 0, s>>>(d_texts + h_off[0], total, mask)));
    uint32_t hm[8];
    PSK_TRY(ctx.read_u32(mask, hm, 8));
    uint32_t v = 256;
    for (uint32_t c = 0; c < 256; c++)
        if (!((hm[c >> 5] >> (c & 31)) & 1u)) {
            v = c;
            break;
        }
    uint64_t chunk = ctx.sched.batch_chunk_mib ? (uint64_t)ctx.sched.batch_chunk_mib << 20 : (3ull << 30);
    const uint64_t limit = 0xFFFFFFF0ull;
    if (chunk > limit) chunk = limit;
    if (v == 256) {
        // all byte values in use: build every text on its own
        for (uint32_t i : big) {
            PSK_TRY(ctx.checkpoint());
            uint64_t len = h_off[i + 1] - h_off[i];
            PSK_TRY(build_level<uint8_t>(ctx, d_texts + h_off[i], nullptr, nullptr, 256, len, d_sas + h_off[i], 0));
        }
        return PSACAK_OK;
    }
    size_t t0 = 0;
    while (t0 < big.size()) {
        PSK_TRY(ctx.checkpoint());
        size_t t1 = t0;
        uint64_t acc = 0;
        while (t1 < big.size()) {
            uint64_t len = h_off[big[t1] + 1] - h_off[big[t1]];
            if (t1 > t0 && acc + len + 1 > chunk) break;
            acc += len + 1;
            t1++;
        }
        if (acc > limit) return set_error(PSACAK_EINVAL, "batch text %u is too long (%llu bytes)", big[t0],
                                          (unsigned long long)(h_off[big[t0] + 1] - h_off[big[t0]]));
        PSK_TRY(batch_chunk(ctx, d_texts, h_off, big.data() + t0, (uint32_t)(t1 - t0), d_sas, v));
        t0 = t1;
    }
    return PSACAK_OK;
}

}  // namespace psk
