// small.cu -- suffix arrays of short strings, one CTA per string, entirely
// in shared memory.
//
// A string of at most SMALL_MAX symbols fits in one SM's shared memory with
// its keys, positions and ranks, so it is sorted there by prefix doubling:
// rank[i] starts as the symbol (+1; 0 stands for "past the end", smaller
// than every symbol, which is the reference's sentinel, src/lib.rs:30-43),
// and each round sorts the positions by (rank[i], rank[i + h]) with a
// block-wide LSD radix sort (8-bit digits, stable ranks from warp ballots),
// then gives every position the dense rank of its key.  After the round
// with 2h >= n all ranks differ and the sorted positions are the suffix
// array.  No global memory is touched between loading the string and
// writing its suffix array, and no host round trip happens per round.
//
// The kernel is persistent: each CTA takes the next string from a queue
// (longest first) until the queue is empty, so a batch of many short
// strings keeps every SM busy with one launch.
#include "ctx.cuh"
#include "small.cuh"

namespace psk {

namespace {

constexpr int SMALL_THREADS = 1024;
constexpr int SMALL_WARPS = SMALL_THREADS / 32;
constexpr int SMALL_IPT = SMALL_MAX / SMALL_THREADS;  // items per thread
static_assert(SMALL_MAX % SMALL_THREADS == 0, "tile shape");
static_assert(SMALL_MAX < 65536, "positions and ranks are 16-bit");
constexpr size_t SMALL_SMEM =
    (size_t)SMALL_MAX * (2 * sizeof(uint32_t) + 2 * sizeof(uint16_t) + sizeof(uint16_t)) +
    (size_t)SMALL_WARPS * 256 * sizeof(uint16_t);

struct SmallSmem {
    uint32_t *key[2];
    uint16_t *idx[2];
    uint16_t *rank;
    uint16_t (*wcnt)[256];
};

// One stable pass on the digit (key >> shift) & 255: items kin/iin[0, n)
// to kout/iout.  Item j belongs to warp j / (32 * SMALL_IPT), step
// (j / 32) % SMALL_IPT, lane j % 32, so warp order, then step, then lane is
// index order and the ranks are stable.
__device__ __forceinline__ void small_pass(const SmallSmem &m, const uint32_t *kin, const uint16_t *iin,
                                           uint32_t *kout, uint16_t *iout, uint32_t n, int shift, uint32_t *s_scan) {
    const int w = threadIdx.x >> 5;
    const uint32_t lane = threadIdx.x & 31, lt = lanemask_lt();
    for (int k = lane; k < 256; k += 32) m.wcnt[w][k] = 0;
    __syncwarp();
    uint32_t dg[SMALL_IPT], rk[SMALL_IPT];
#pragma unroll
    for (int r = 0; r < SMALL_IPT; r++) {
        const uint32_t j = (uint32_t)w * 32 * SMALL_IPT + (uint32_t)r * 32 + lane;
        const bool valid = j < n;
        const uint32_t d = valid ? (kin[j] >> shift) & 255u : 256u;
        // lanes with the same digit: intersection of eight bit ballots
        uint32_t peers = __ballot_sync(FULL_MASK, valid);
#pragma unroll
        for (int b = 0; b < 8; b++) {
            const uint32_t bit = (d >> b) & 1u;
            const uint32_t bb = __ballot_sync(FULL_MASK, bit);
            peers &= bit ? bb : ~bb;
        }
        const uint32_t prior = valid ? m.wcnt[w][d] : 0u;
        rk[r] = prior + __popc(peers & lt);
        dg[r] = d;
        __syncwarp();
        if (valid && (int)lane == __ffs(peers) - 1) m.wcnt[w][d] = (uint16_t)(prior + __popc(peers));
        __syncwarp();
    }
    __syncthreads();
    // bases in digit-major, warp-minor order
    uint32_t cnt = 0;
    if (threadIdx.x < 256)
        for (int ww = 0; ww < SMALL_WARPS; ww++) cnt += m.wcnt[ww][threadIdx.x];
    uint32_t ex = 0;
    block_scan<uint32_t, OpSum<uint32_t>, SMALL_THREADS>(cnt, OpSum<uint32_t>(), s_scan, &ex, (uint32_t *)nullptr);
    if (threadIdx.x < 256) {
        uint32_t run = ex;
        for (int ww = 0; ww < SMALL_WARPS; ww++) {
            const uint32_t c = m.wcnt[ww][threadIdx.x];
            m.wcnt[ww][threadIdx.x] = (uint16_t)run;
            run += c;
        }
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < SMALL_IPT; r++) {
        if (dg[r] < 256) {
            const uint32_t j = (uint32_t)w * 32 * SMALL_IPT + (uint32_t)r * 32 + lane;
            const uint32_t dst = m.wcnt[w][dg[r]] + rk[r];
            kout[dst] = kin[j];
            iout[dst] = iin[j];
        }
    }
    __syncthreads();
}

// Suffix array of t[0, n) (2 <= n <= SMALL_MAX) into out; symbol values
// must be below `sigma` (sigma <= 65535).  Returns false when a bound was
// broken (recorded in err).
template <class C>
__device__ bool small_build(const SmallSmem &m, const C *__restrict__ t, uint32_t n, uint32_t sigma, uint32_t *out,
                            uint32_t *s_scan, uint32_t *err) {
    bool ok = true;
    for (uint32_t i = threadIdx.x; i < n; i += SMALL_THREADS) {
        const uint32_t v = (uint32_t)t[i];
        if (v >= sigma) ok = false;
        m.rank[i] = (uint16_t)(v + 1);
    }
    if (__syncthreads_or(!ok)) {
        if (threadIdx.x == 0) dev_fail(err, DEVERR_RANGE);
        return false;
    }
    uint32_t maxrank = sigma;  // ranks lie in [1, maxrank]
    for (uint32_t h = 1;; h <<= 1) {
        if (h >= 2 * SMALL_MAX) {  // cannot happen: all ranks differ once 2h >= n
            if (threadIdx.x == 0) dev_fail(err, DEVERR_RANGE);
            return false;
        }
        {
            const int w = threadIdx.x >> 5;
            const uint32_t lane = threadIdx.x & 31;
#pragma unroll
            for (int r = 0; r < SMALL_IPT; r++) {
                const uint32_t j = (uint32_t)w * 32 * SMALL_IPT + (uint32_t)r * 32 + lane;
                if (j < n) {
                    m.key[0][j] = (uint32_t)m.rank[j] << 16 | (j + h < n ? (uint32_t)m.rank[j + h] : 0u);
                    m.idx[0][j] = (uint16_t)j;
                }
            }
        }
        __syncthreads();
        // an even number of passes: the sorted pairs end in key[0] / idx[0]
        const bool wide = maxrank >= 256;
        small_pass(m, m.key[0], m.idx[0], m.key[1], m.idx[1], n, 0, s_scan);
        if (wide) {
            small_pass(m, m.key[1], m.idx[1], m.key[0], m.idx[0], n, 8, s_scan);
            small_pass(m, m.key[0], m.idx[0], m.key[1], m.idx[1], n, 16, s_scan);
            small_pass(m, m.key[1], m.idx[1], m.key[0], m.idx[0], n, 24, s_scan);
        } else {
            small_pass(m, m.key[1], m.idx[1], m.key[0], m.idx[0], n, 16, s_scan);
        }
        // dense ranks of the sorted keys (thread-contiguous chunks)
        const uint32_t base = threadIdx.x * SMALL_IPT;
        uint32_t f[SMALL_IPT], c = 0;
#pragma unroll
        for (int r = 0; r < SMALL_IPT; r++) {
            const uint32_t j = base + r;
            f[r] = (j < n && (j == 0 || m.key[0][j] != m.key[0][j - 1])) ? 1u : 0u;
            c += f[r];
        }
        uint32_t ex = 0, distinct = 0;
        block_scan<uint32_t, OpSum<uint32_t>, SMALL_THREADS>(c, OpSum<uint32_t>(), s_scan, &ex, &distinct);
        uint32_t run = ex;
#pragma unroll
        for (int r = 0; r < SMALL_IPT; r++) {
            const uint32_t j = base + r;
            if (j < n) {
                run += f[r];
                m.rank[m.idx[0][j]] = (uint16_t)run;
            }
        }
        __syncthreads();
        if (distinct == n) break;
        maxrank = distinct;
    }
    for (uint32_t j = threadIdx.x; j < n; j += SMALL_THREADS) out[j] = m.idx[0][j];
    __syncthreads();
    return true;
}

template <class C>
__global__ void __launch_bounds__(SMALL_THREADS, 1) k_small_sa(const C *__restrict__ text, SmallJobs jobs,
                                                               uint32_t sigma, uint32_t *queue, uint32_t *sas,
                                                               uint32_t *err) {
    extern __shared__ __align__(16) unsigned char small_smem[];
    __shared__ uint32_t s_scan[33];
    __shared__ uint32_t s_job;
    SmallSmem m;
    m.key[0] = (uint32_t *)small_smem;
    m.key[1] = m.key[0] + SMALL_MAX;
    m.idx[0] = (uint16_t *)(m.key[1] + SMALL_MAX);
    m.idx[1] = m.idx[0] + SMALL_MAX;
    m.rank = m.idx[1] + SMALL_MAX;
    m.wcnt = (uint16_t(*)[256])(m.rank + SMALL_MAX);
    for (;;) {
        if (threadIdx.x == 0) s_job = atomicAdd(queue, 1u);
        __syncthreads();
        const uint32_t job = s_job;
        __syncthreads();
        if (job >= jobs.count) return;
        uint64_t off = 0, n = jobs.n;
        if (jobs.offs) {
            const uint32_t id = jobs.ids[job];
            off = jobs.offs[id];
            n = jobs.offs[id + 1] - off;
        }
        if (n > SMALL_MAX) {
            if (threadIdx.x == 0) dev_fail(err, DEVERR_RANGE);
            continue;
        }
        if (n <= 1) {
            if (n == 1 && threadIdx.x == 0) sas[off] = 0;
            continue;
        }
        small_build<C>(m, text + off, (uint32_t)n, sigma, sas + off, s_scan, err);
    }
}

}  // namespace

template <class C>
status_t small_sa(Ctx &ctx, const C *text, SmallJobs jobs, uint32_t sigma, uint32_t *sas, cudaStream_t s) {
    if (jobs.count == 0) return PSACAK_OK;
    if (sigma == 0 || sigma > 65535) return set_error(PSACAK_EINTERNAL, "small strings: alphabet of %u", sigma);
    static_assert(SMALL_SMEM + 40 * 4 <= 227 * 1024, "shared memory");
    PSK_CUDA(cudaFuncSetAttribute(k_small_sa<C>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMALL_SMEM));
    uint32_t *queue = ctx.d_scalars + 40;
    PSK_CUDA(cudaMemsetAsync(queue, 0, sizeof(uint32_t), s));
    const uint32_t grid = jobs.count < (uint32_t)ctx.dev.num_sms ? jobs.count : (uint32_t)ctx.dev.num_sms;
    // algorithmic bytes: every string read once and its suffix array written once
    PSK_PROF_LAUNCH(s, "small_strings", jobs.symbols, jobs.symbols * (sizeof(C) + sizeof(uint32_t)),
                    (k_small_sa<C><<<grid, SMALL_THREADS, SMALL_SMEM, s>>>(text, jobs, sigma, queue, sas, ctx.d_err)));
    PSK_LAUNCH_CHECK();
    return PSACAK_OK;
}

template status_t small_sa<uint8_t>(Ctx &, const uint8_t *, SmallJobs, uint32_t, uint32_t *, cudaStream_t);
template status_t small_sa<uint32_t>(Ctx &, const uint32_t *, SmallJobs, uint32_t, uint32_t *, cudaStream_t);

}  // namespace psk
