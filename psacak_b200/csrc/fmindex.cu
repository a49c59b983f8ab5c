// fmindex.cu -- FM-index over the Burrows-Wheeler transform produced by
// psacak_bwt8_dev, and backward search on the device.  hucsmn/psacak has no
// counterpart; the index is a consumer of its suffix array (the sentinel
// convention of src/lib.rs:30-43 fixes the rows).
//
// Rows.  The suffixes of text + sentinel, sorted, are rows 0..n; row 0 is
// the sentinel suffix and row r >= 1 is suffix SA[r-1].  Column L (the BWT
// with the sentinel) has L[0] = text[n-1] and L[r] = text[SA[r-1]-1], with
// the sentinel at row `primary` (SA[primary-1] = 0).  psacak_bwt8_dev
// returns L without that row: B[r] = L[r] below primary, B[r-1] = L[r]
// above it.  C[c] = 1 + the number of text bytes smaller than c (row 0 is
// the smallest).  Occ(c, r) = occurrences of c in L[0, r) = occurrences in
// B[0, r - (r > primary)).
//
// Backward search of P: [sp, ep) = [0, n + 1), then for k = |P|-1 .. 0:
// sp = C[P[k]] + Occ(P[k], sp), ep = C[P[k]] + Occ(P[k], ep).  The rows
// [sp, ep) hold the suffixes that start with P; in suffix-array indices
// (no sentinel row) that is [sp - 1, ep - 1).
//
// Layout (one device buffer, psacak_fm_bytes(n)):
//   header   n, primary, super rows, block rows (4 x u64), then C[0..256]
//            (u32), padded to FM_HEADER bytes;
//   super    (nsuper + 1) rows of 256 u32: occurrences in B[0, s * 2^16);
//   blocks   (nblocks + 1) rows of 256 u16: occurrences in B from the
//            start of the block's superblock up to b * 256.
// Occ in B[0, i) = super[i >> 16][c] + blocks[i >> 8][c] + the count of c
// in B[(i >> 8) * 256, i), which one half-warp reads as 16 x 16 bytes.
// 2 + 4/256 bytes per text byte.
#include "ctx.cuh"
#include "../../include/psacak_b200.h"

namespace psk {

void clear_error();

constexpr uint64_t FM_SUPER = 1ull << 16;
constexpr uint64_t FM_BLOCK = 256;
constexpr uint64_t FM_HEADER = 2048;

struct FmLayout {
    uint64_t n, primary, nsuper, nblocks;
    uint64_t super_off, block_off, bytes;
};

__host__ __device__ inline FmLayout fm_layout(uint64_t n) {
    FmLayout L;
    L.n = n;
    L.primary = 0;
    L.nsuper = (n + FM_SUPER - 1) / FM_SUPER;
    L.nblocks = (n + FM_BLOCK - 1) / FM_BLOCK;
    L.super_off = FM_HEADER;
    L.block_off = L.super_off + (L.nsuper + 1) * 256 * sizeof(uint32_t);
    L.bytes = L.block_off + (L.nblocks + 1) * 256 * sizeof(uint16_t);
    L.bytes = (L.bytes + 255) & ~255ull;
    return L;
}

// One CTA per superblock s (rows s * 256 .. s * 256 + 255 of the block
// table, those <= nblocks): per-block histograms in shared memory (two u16
// counters per u32 word, a block has at most 256 bytes), then thread c
// turns them into the running counts of byte c.  tot[s][c] = occurrences of
// c in the superblock.
__global__ void __launch_bounds__(256) k_fm_blocks(const uint8_t *__restrict__ B, uint64_t n, uint64_t nblocks,
                                                   uint16_t *__restrict__ blocks, uint32_t *__restrict__ tot) {
    extern __shared__ uint32_t s_h[];  // [256 blocks][128 words]
    const uint64_t s = blockIdx.x;
    const uint32_t lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint64_t base = s * FM_SUPER;
    for (uint32_t b = w; b < 256; b += 8) {
        uint32_t *h = s_h + b * 128;
        for (uint32_t k = lane; k < 128; k += 32) h[k] = 0;
        __syncwarp();
        const uint64_t p0 = base + (uint64_t)b * FM_BLOCK + lane * 8;
#pragma unroll
        for (int k = 0; k < 8; k++) {
            const uint64_t p = p0 + k;
            if (p < n) {
                const uint32_t c = B[p];
                atomicAdd(&h[c >> 1], 1u << ((c & 1) * 16));
            }
        }
        __syncwarp();
    }
    __syncthreads();
    const uint32_t c = threadIdx.x;
    uint32_t run = 0;
    for (uint32_t b = 0; b < 256; b++) {
        const uint64_t row = s * 256 + b;
        if (row <= nblocks) blocks[row * 256 + c] = (uint16_t)run;
        run += (s_h[b * 128 + (c >> 1)] >> ((c & 1) * 16)) & 0xFFFFu;
    }
    tot[s * 256 + c] = run;
}

// super[s][c] = occurrences of c before superblock s (exclusive prefix over
// the superblock totals), C[c] = 1 + bytes smaller than c.  One CTA; thread
// c walks the rows, loads of 16 rows in flight at a time.
__global__ void __launch_bounds__(256) k_fm_super(const uint32_t *__restrict__ tot, uint64_t rows,
                                                  uint32_t *__restrict__ super, uint32_t *C, uint64_t n) {
    __shared__ uint32_t s_scan[33];
    const uint32_t c = threadIdx.x;
    uint32_t run = 0;
    for (uint64_t s0 = 0; s0 < rows; s0 += 16) {
        uint32_t v[16];
#pragma unroll
        for (int k = 0; k < 16; k++) v[k] = s0 + k < rows ? tot[(s0 + k) * 256 + c] : 0u;
#pragma unroll
        for (int k = 0; k < 16; k++)
            if (s0 + k < rows) {
                super[(s0 + k) * 256 + c] = run;
                run += v[k];
            }
    }
    super[rows * 256 + c] = run;  // row nsuper: every occurrence
    uint32_t total = 0;
    const uint32_t ex = block_exclusive_sum<uint32_t, 256>(run, s_scan, &total);
    C[c] = 1u + ex;
    if (c == 0) C[256] = (uint32_t)n + 1u;
}

struct FmView {
    uint64_t n, primary;
    const uint32_t *C, *super;
    const uint16_t *blocks;
};

__device__ __forceinline__ FmView fm_view(const unsigned char *fm) {
    const uint64_t *hd = (const uint64_t *)fm;
    FmLayout L = fm_layout(hd[0]);
    FmView v;
    v.n = hd[0];
    v.primary = hd[1];
    v.C = (const uint32_t *)(fm + 32);
    v.super = (const uint32_t *)(fm + L.super_off);
    v.blocks = (const uint16_t *)(fm + L.block_off);
    return v;
}

// Occurrences of c in B[0, i), by one half-warp (`h` = lane within the
// half, `hmask` = the half's lanes): every lane counts c in its 16 bytes of
// the block that holds i, the half adds them up, and the checkpoints add
// the rest.
__device__ __forceinline__ uint32_t fm_occ_half(const FmView &F, const uint8_t *__restrict__ B, bool aligned,
                                                uint32_t c, uint64_t i, uint32_t h, uint32_t hmask) {
    const uint64_t b0 = i & ~(FM_BLOCK - 1);
    const uint64_t q = b0 + h * 16;
    uint32_t cnt = 0;
    if (q < i) {
        const uint32_t lim = (uint32_t)(i - q < 16 ? i - q : 16);  // bytes of this lane below i
        if (aligned && q + 16 <= F.n) {
            const uint4 x = *reinterpret_cast<const uint4 *>(B + q);
            const uint32_t cc = c * 0x01010101u;
            const uint32_t wv[4] = {x.x, x.y, x.z, x.w};
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const uint32_t eq = __vcmpeq4(wv[k], cc);  // 0xFF in every equal byte
                const int lo = k * 4;
                uint32_t keep = lim >= (uint32_t)lo + 4 ? 0xFFFFFFFFu
                                : lim <= (uint32_t)lo   ? 0u
                                                        : (0xFFFFFFFFu >> (32 - 8 * (lim - lo)));
                cnt += __popc(eq & keep) >> 3;
            }
        } else {
            for (uint32_t k = 0; k < lim; k++) cnt += B[q + k] == c;
        }
    }
    cnt = __reduce_add_sync(hmask, cnt);
    return cnt + F.super[(i >> 16) * 256 + c] + F.blocks[(i >> 8) * 256 + c];
}

// One warp per pattern: lanes 0-15 keep sp, lanes 16-31 keep ep.
__global__ void __launch_bounds__(256) k_fm_count(const unsigned char *__restrict__ fm, const uint8_t *__restrict__ B,
                                                  const uint8_t *__restrict__ pat, const uint64_t *__restrict__ off,
                                                  uint32_t npat, uint32_t *__restrict__ ranges, uint32_t *err) {
    const FmView F = fm_view(fm);
    const bool aligned = (((uintptr_t)B) & 15u) == 0;
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t half = lane >> 4, h = lane & 15;
    const uint32_t hmask = half ? 0xFFFF0000u : 0x0000FFFFu;
    const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x >> 5);
    for (uint64_t p = (uint64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); p < npat; p += warps) {
        const uint64_t a = off[p], e = off[p + 1];
        if (e < a) {
            dev_fail(err, DEVERR_RANGE);
            continue;
        }
        uint64_t sp = 0, ep = F.n + 1;  // rows
        for (uint64_t k = e; k-- > a && sp < ep;) {
            const uint32_t c = pat[k];
            uint64_t r = half ? ep : sp;
            r -= r > F.primary ? 1 : 0;  // row -> index into B (the sentinel row has no byte)
            const uint64_t v = (uint64_t)F.C[c] + fm_occ_half(F, B, aligned, c, r, h, hmask);
            const uint64_t sp2 = __shfl_sync(FULL_MASK, v, 0);
            const uint64_t ep2 = __shfl_sync(FULL_MASK, v, 16);
            sp = sp2;
            ep = ep2;
        }
        if (lane == 0) {
            // rows -> suffix-array indices (row 0, the sentinel, has none)
            uint64_t lo = sp > 0 ? sp - 1 : 0, hi = ep > 0 ? ep - 1 : 0;
            if (ep <= sp) lo = hi = (sp > 0 ? sp - 1 : 0);
            if (e == a) {
                lo = 0;
                hi = F.n;
            }
            ranges[2 * p] = (uint32_t)lo;
            ranges[2 * p + 1] = (uint32_t)(hi > lo ? hi : lo);
        }
    }
}

}  // namespace psk

using namespace psk;

extern "C" {

uint64_t psacak_fm_bytes(uint64_t n) { return fm_layout(n).bytes; }

int psacak_fm_build_dev(psacak_ctx *ctx, const uint8_t *d_bwt, uint64_t n, uint64_t primary, void *d_fm,
                        void *stream) {
    clear_error();
    if (!ctx || !d_fm) return set_error(PSACAK_EINVAL, "null context or index pointer");
    if (n >= 0xFFFFFFFFull) return set_error(PSACAK_EINVAL, "n = %llu is not below 2^32 - 1", (unsigned long long)n);
    if (n > 0 && !d_bwt) return set_error(PSACAK_EINVAL, "null BWT pointer");
    if (n > 0 && (primary < 1 || primary > n))
        return set_error(PSACAK_EINVAL, "primary index %llu outside 1..%llu", (unsigned long long)primary,
                         (unsigned long long)n);
    if (((uintptr_t)d_fm) & 15u) return set_error(PSACAK_EINVAL, "the index buffer must be 16-byte aligned");
    std::lock_guard<std::mutex> g(ctx->c.mu);
    Ctx &c = ctx->c;
    PSK_CUDA(cudaSetDevice(c.dev.id));
    c.stream = stream ? (cudaStream_t)stream : c.own_stream;
    cudaStream_t s = c.stream;
    FmLayout L = fm_layout(n);
    L.primary = n ? primary : 0;
    const uint64_t hd[4] = {L.n, L.primary, L.nsuper, L.nblocks};
    unsigned char *fm = (unsigned char *)d_fm;
    PSK_CUDA(cudaMemcpyAsync(fm, hd, sizeof(hd), cudaMemcpyHostToDevice, s));
    DBuf<uint32_t> tot;
    PSK_TRY(tot.init(c, (L.nsuper + 1) * 256));
    const size_t smem = 256 * 128 * sizeof(uint32_t);
    PSK_CUDA(cudaFuncSetAttribute(k_fm_blocks, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    PSK_PROF_LAUNCH(s, "fm_blocks", n, n + 2 * n + 4 * L.nsuper * 256,
                    (k_fm_blocks<<<(uint32_t)(L.nsuper + 1), 256, smem, s>>>(
                        d_bwt, n, L.nblocks, (uint16_t *)(fm + L.block_off), tot.get())));
    PSK_PROF_LAUNCH(s, "fm_super", L.nsuper, 8 * L.nsuper * 256,
                    (k_fm_super<<<1, 256, 0, s>>>(tot.get(), L.nsuper, (uint32_t *)(fm + L.super_off),
                                                  (uint32_t *)(fm + 32), n)));
    PSK_LAUNCH_CHECK();
    tot.reset();
    PSK_TRY(c.sync());  // the header copy reads a stack array
    return c.check_device_error();
}

int psacak_fm_count_dev(psacak_ctx *ctx, const void *d_fm, const uint8_t *d_bwt, const uint8_t *d_patterns,
                        const uint64_t *d_offsets, uint32_t n_patterns, uint32_t *d_ranges, void *stream) {
    clear_error();
    if (!ctx || !d_fm) return set_error(PSACAK_EINVAL, "null context or index pointer");
    if (n_patterns > 0 && (!d_offsets || !d_ranges)) return set_error(PSACAK_EINVAL, "null pattern arrays");
    std::lock_guard<std::mutex> g(ctx->c.mu);
    Ctx &c = ctx->c;
    PSK_CUDA(cudaSetDevice(c.dev.id));
    c.stream = stream ? (cudaStream_t)stream : c.own_stream;
    cudaStream_t s = c.stream;
    if (n_patterns == 0) return PSACAK_OK;
    uint64_t hd[2] = {0, 0};
    PSK_CUDA(cudaMemcpyAsync(hd, d_fm, sizeof(hd), cudaMemcpyDeviceToHost, s));
    PSK_CUDA(cudaStreamSynchronize(s));
    if (hd[0] > 0 && !d_bwt) return set_error(PSACAK_EINVAL, "null BWT pointer");
    const uint64_t warps_per_cta = 8;
    const uint64_t ctas = (n_patterns + warps_per_cta - 1) / warps_per_cta;
    const uint32_t cap = 64 * (uint32_t)c.dev.num_sms;
    PSK_PROF_LAUNCH(s, "fm_count", n_patterns, 0,
                    (k_fm_count<<<(uint32_t)(ctas < cap ? ctas : cap), 256, 0, s>>>(
                        (const unsigned char *)d_fm, d_bwt, d_patterns, d_offsets, n_patterns, d_ranges, c.d_err)));
    PSK_LAUNCH_CHECK();
    PSK_TRY(c.sync());
    return c.check_device_error();
}

}  // extern "C"
