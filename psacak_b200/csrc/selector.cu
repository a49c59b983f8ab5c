// selector.cu -- text statistics and the schedule-selector MLP (fp32).
//
// The selector predicts, from 16 cheap statistics of a text, the log build
// time of every candidate schedule; the schedule with the smallest
// prediction is used.  Every schedule produces the same suffix array, so a
// wrong prediction costs time, never correctness.  Network: 16 -> 64 -> 64
// -> K (ReLU), trained with a masked mean-squared error on measured
// log2(ms), Adam updates; all of it in the kernels below.
#include <math.h>

#include "ctx.cuh"
#include "../../include/psacak_b200_select.h"

namespace psk {

const char *last_error();
void clear_error();

constexpr int F = PSACAK_SEL_FEATURES;  // 16
constexpr int H = PSACAK_SEL_HIDDEN;    // 64
constexpr int KMAX = PSACAK_SEL_MAX_OUT;

__host__ __device__ inline size_t off_w1() { return 0; }
__host__ __device__ inline size_t off_b1() { return (size_t)F * H; }
__host__ __device__ inline size_t off_w2() { return off_b1() + H; }
__host__ __device__ inline size_t off_b2() { return off_w2() + (size_t)H * H; }
__host__ __device__ inline size_t off_w3() { return off_b2() + H; }
__host__ __device__ inline size_t off_b3(uint32_t K) { return off_w3() + (size_t)H * K; }

__device__ __forceinline__ uint32_t hmix(uint64_t z) {
    z += 0x9e3779b97f4a7c15ull;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return (uint32_t)(z ^ (z >> 31));
}

// ---------------------------------------------------------------------------
// Statistics of a text from a sample of <= 65536 evenly spaced positions and
// 2048 windows of 16 symbols at hashed offsets.  One CTA of 1024 threads.
// ---------------------------------------------------------------------------
template <class C>
__device__ __forceinline__ int type_at(const C *t, uint64_t n, uint64_t p) {  // 1 = S, 0 = L
    for (uint64_t q = p; q + 1 < n && q < p + 64; q++) {
        if (t[q] != t[q + 1]) return t[q] < t[q + 1] ? 1 : 0;
    }
    return 0;
}

template <class C>
__global__ void __launch_bounds__(1024) k_text_stats(const C *__restrict__ t, uint64_t n, float *out) {
    __shared__ uint32_t s_bits[512];  // 16384-bit distinct sketch
    __shared__ uint32_t s_hist[256];
    __shared__ uint32_t s_win[2048];
    __shared__ unsigned long long s_acc[6];  // lms, stype, runs, dups, maxsym, samples
    for (int i = threadIdx.x; i < 512; i += 1024) s_bits[i] = 0;
    for (int i = threadIdx.x; i < 256; i += 1024) s_hist[i] = 0;
    if (threadIdx.x < 6) s_acc[threadIdx.x] = 0;
    __syncthreads();
    const uint64_t S = n < 65536 ? n : 65536;
    unsigned long long lms = 0, st = 0, runs = 0, mx = 0;
    for (uint64_t i = threadIdx.x; i < S; i += 1024) {
        uint64_t p = (i * n) / S;
        uint64_t v = (uint64_t)t[p];
        uint32_t h = hmix(v);
        atomicOr(&s_bits[(h >> 5) & 511], 1u << (h & 31));
        atomicAdd(&s_hist[(h >> 16) & 255], 1u);
        int ty = type_at(t, n, p);
        st += ty;
        if (p > 0) {
            C a = t[p - 1], b = t[p];
            int tp = a < b ? 1 : (a > b ? 0 : ty);
            if (ty == 1 && tp == 0) lms++;
            if (a == b) runs++;
        }
        mx = v > mx ? v : mx;
    }
    atomicAdd(&s_acc[0], lms);
    atomicAdd(&s_acc[1], st);
    atomicAdd(&s_acc[2], runs);
    atomicMax(&s_acc[4], mx);
    // windows of 16 symbols
    const uint64_t W = 16;
    for (int i = threadIdx.x; i < 2048; i += 1024) {
        uint32_t h = 0;
        if (n > W) {
            uint64_t p = hmix(0x1234567ull + i) % (n - W);
            uint64_t acc = 0;
            for (uint64_t q = 0; q < W; q++) acc = acc * 0x100000001b3ull + (uint64_t)t[p + q] + 1;
            h = hmix(acc) | 1u;
        } else {
            h = (uint32_t)i + 1;  // no windows: all distinct
        }
        s_win[i] = h;
    }
    __syncthreads();
    // bitonic sort of the 2048 window hashes
    for (int k = 2; k <= 2048; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = threadIdx.x; i < 2048; i += 1024) {
                int l = i ^ j;
                if (l > i) {
                    uint32_t a = s_win[i], b = s_win[l];
                    bool up = (i & k) == 0;
                    if ((a > b) == up) {
                        s_win[i] = b;
                        s_win[l] = a;
                    }
                }
            }
            __syncthreads();
        }
    }
    unsigned long long dups = 0;
    for (int i = threadIdx.x; i < 2048; i += 1024)
        if ((i > 0 && s_win[i] == s_win[i - 1]) || (i + 1 < 2048 && s_win[i] == s_win[i + 1])) dups++;
    atomicAdd(&s_acc[3], dups);
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t zeros = 0;
        for (int i = 0; i < 512; i++) zeros += 32 - __popc(s_bits[i]);
        double m = 16384.0;
        double distinct = zeros > 0 ? -m * log((double)zeros / m) : m * 8;
        double ent = 0;
        for (int i = 0; i < 256; i++)
            if (s_hist[i]) {
                double pr = (double)s_hist[i] / (double)S;
                ent -= pr * log2(pr);
            }
        double Sd = S > 0 ? (double)S : 1.0;
        double f0 = log2((double)n + 1) / 32.0;
        double f1 = (double)sizeof(C) / 4.0;
        double f2 = log2(distinct + 1) / 32.0;
        double f3 = (double)s_acc[0] / Sd;
        double f4 = (double)s_acc[1] / Sd;
        double f5 = (double)s_acc[2] / Sd;
        double f6 = (double)s_acc[3] / 2048.0;
        double f7 = ent / 8.0;
        double f8 = log2((double)s_acc[4] + 1) / 32.0;
        out[0] = (float)f0;
        out[1] = (float)f1;
        out[2] = (float)f2;
        out[3] = (float)f3;
        out[4] = (float)f4;
        out[5] = (float)f5;
        out[6] = (float)f6;
        out[7] = (float)f7;
        out[8] = (float)f8;
        out[9] = (float)(f0 * f0);
        out[10] = (float)(f0 * f1);
        out[11] = (float)(f2 - f0);
        out[12] = (float)(f3 * f0);
        out[13] = (float)(f6 * f0);
        out[14] = (float)(f5 * f0);
        out[15] = 1.0f;
    }
}

// ---------------------------------------------------------------------------
// MLP.  One CTA of H threads per sample.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(H) k_mlp_forward(const float *__restrict__ P, const float *__restrict__ X,
                                                   float *__restrict__ Y, float *__restrict__ H1,
                                                   float *__restrict__ H2, uint32_t K) {
    __shared__ float sx[F], s1[H], s2[H];
    const uint32_t b = blockIdx.x, j = threadIdx.x;
    if (j < F) sx[j] = X[(size_t)b * F + j];
    __syncthreads();
    float a = P[off_b1() + j];
    for (int i = 0; i < F; i++) a = fmaf(sx[i], P[off_w1() + (size_t)i * H + j], a);
    a = fmaxf(a, 0.f);
    s1[j] = a;
    if (H1) H1[(size_t)b * H + j] = a;
    __syncthreads();
    float c = P[off_b2() + j];
    for (int i = 0; i < H; i++) c = fmaf(s1[i], P[off_w2() + (size_t)i * H + j], c);
    c = fmaxf(c, 0.f);
    s2[j] = c;
    if (H2) H2[(size_t)b * H + j] = c;
    __syncthreads();
    if (j < K) {
        float y = P[off_b3(K) + j];
        for (int i = 0; i < H; i++) y = fmaf(s2[i], P[off_w3() + (size_t)i * K + j], y);
        Y[(size_t)b * K + j] = y;
    }
}

// Gradients of L = sum(M * (Y - T)^2) / sum(M), accumulated into G
// (zeroed by the caller); one CTA of H threads per sample.
__global__ void __launch_bounds__(H) k_mlp_backward(const float *__restrict__ P, const float *__restrict__ X,
                                                    const float *__restrict__ H1, const float *__restrict__ H2,
                                                    const float *__restrict__ Y, const float *__restrict__ T,
                                                    const float *__restrict__ M, float inv_count, uint32_t K,
                                                    float *__restrict__ G, float *loss) {
    __shared__ float sx[F], s1[H], s2[H], dy[KMAX], d2[H], d1[H];
    const uint32_t b = blockIdx.x, j = threadIdx.x;
    if (j < F) sx[j] = X[(size_t)b * F + j];
    s1[j] = H1[(size_t)b * H + j];
    s2[j] = H2[(size_t)b * H + j];
    if (j < K) {
        float m = M[(size_t)b * K + j];
        float e = Y[(size_t)b * K + j] - T[(size_t)b * K + j];
        dy[j] = 2.f * m * e * inv_count;
        if (m != 0.f) atomicAdd(loss, m * e * e * inv_count);
    }
    __syncthreads();
    // layer 3
    {
        float acc = 0.f;
        for (uint32_t o = 0; o < K; o++) {
            atomicAdd(&G[off_w3() + (size_t)j * K + o], s2[j] * dy[o]);
            acc = fmaf(dy[o], P[off_w3() + (size_t)j * K + o], acc);
        }
        if (j < K) atomicAdd(&G[off_b3(K) + j], dy[j]);
        d2[j] = s2[j] > 0.f ? acc : 0.f;
    }
    __syncthreads();
    // layer 2
    {
        float acc = 0.f;
        for (int o = 0; o < H; o++) {
            atomicAdd(&G[off_w2() + (size_t)j * H + o], s1[j] * d2[o]);
            acc = fmaf(d2[o], P[off_w2() + (size_t)j * H + o], acc);
        }
        atomicAdd(&G[off_b2() + j], d2[j]);
        d1[j] = s1[j] > 0.f ? acc : 0.f;
    }
    __syncthreads();
    // layer 1
    for (int i = 0; i < F; i++) atomicAdd(&G[off_w1() + (size_t)i * H + j], sx[i] * d1[j]);
    atomicAdd(&G[off_b1() + j], d1[j]);
}

__global__ void k_adam(float *P, const float *G, float *m1, float *m2, uint64_t n, float lr, float b1, float b2,
                       float eps, float c1, float c2) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        float g = G[i];
        float a = b1 * m1[i] + (1.f - b1) * g;
        float v = b2 * m2[i] + (1.f - b2) * g * g;
        m1[i] = a;
        m2[i] = v;
        P[i] -= lr * (a / c1) / (sqrtf(v / c2) + eps);
    }
}

// Inference for one feature vector: forward pass and argmin over the K
// predictions (ties: lowest index).
__global__ void __launch_bounds__(H) k_select(const float *__restrict__ P, const float *__restrict__ X, uint32_t K,
                                              uint32_t *out, float *pred) {
    __shared__ float sx[F], s1[H], s2[H], sy[KMAX];
    const uint32_t j = threadIdx.x;
    if (j < F) sx[j] = X[j];
    __syncthreads();
    float a = P[off_b1() + j];
    for (int i = 0; i < F; i++) a = fmaf(sx[i], P[off_w1() + (size_t)i * H + j], a);
    s1[j] = fmaxf(a, 0.f);
    __syncthreads();
    float c = P[off_b2() + j];
    for (int i = 0; i < H; i++) c = fmaf(s1[i], P[off_w2() + (size_t)i * H + j], c);
    s2[j] = fmaxf(c, 0.f);
    __syncthreads();
    if (j < K) {
        float y = P[off_b3(K) + j];
        for (int i = 0; i < H; i++) y = fmaf(s2[i], P[off_w3() + (size_t)i * K + j], y);
        sy[j] = y;
        if (pred) pred[j] = y;
    }
    __syncthreads();
    if (j == 0) {
        uint32_t best = 0;
        for (uint32_t o = 1; o < K; o++)
            if (sy[o] < sy[best]) best = o;
        *out = best;
    }
}

}  // namespace psk

using namespace psk;

static int sel_guard(psacak_ctx *ctx, uint32_t K) {
    if (!ctx) return set_error(PSACAK_EINVAL, "null context");
    if (K == 0 || K > KMAX) return set_error(PSACAK_EINVAL, "selector outputs must be in 1..%d", KMAX);
    return PSACAK_OK;
}

extern "C" {

uint64_t psacak_sel_param_count(uint32_t nout) { return off_b3(nout) + nout; }

int psacak_text_stats(psacak_ctx *ctx, const void *d_text, uint64_t n, int width, float *features) {
    clear_error();
    if (!ctx || !features || (width != 1 && width != 4)) return set_error(PSACAK_EINVAL, "bad stats arguments");
    if (n > 0 && !d_text) return set_error(PSACAK_EINVAL, "null text");
    std::lock_guard<std::mutex> g(ctx->c.mu);
    Ctx &c = ctx->c;
    PSK_CUDA(cudaSetDevice(c.dev.id));
    c.stream = c.own_stream;
    float *d_out = (float *)(c.d_scalars + 44);  // 16 floats
    if (n == 0) {
        for (int i = 0; i < F; i++) features[i] = 0.f;
        features[F - 1] = 1.f;
        return PSACAK_OK;
    }
    if (width == 1) k_text_stats<uint8_t><<<1, 1024, 0, c.stream>>>((const uint8_t *)d_text, n, d_out);
    else k_text_stats<uint32_t><<<1, 1024, 0, c.stream>>>((const uint32_t *)d_text, n, d_out);
    PSK_KCOUNT();
    PSK_LAUNCH_CHECK();
    PSK_CUDA(cudaMemcpyAsync(features, d_out, F * sizeof(float), cudaMemcpyDeviceToHost, c.stream));
    PSK_CUDA(cudaStreamSynchronize(c.stream));
    return PSACAK_OK;
}

int psacak_mlp_forward(psacak_ctx *ctx, const float *d_params, const float *d_x, float *d_y, float *d_h1,
                       float *d_h2, uint32_t batch, uint32_t nout) {
    clear_error();
    PSK_TRY(sel_guard(ctx, nout));
    std::lock_guard<std::mutex> g(ctx->c.mu);
    Ctx &c = ctx->c;
    PSK_CUDA(cudaSetDevice(c.dev.id));
    if (batch == 0) return PSACAK_OK;
    k_mlp_forward<<<batch, H, 0, c.own_stream>>>(d_params, d_x, d_y, d_h1, d_h2, nout);
    PSK_KCOUNT();
    PSK_LAUNCH_CHECK();
    PSK_CUDA(cudaStreamSynchronize(c.own_stream));
    return PSACAK_OK;
}

int psacak_mlp_backward(psacak_ctx *ctx, const float *d_params, const float *d_x, const float *d_h1,
                        const float *d_h2, const float *d_y, const float *d_t, const float *d_m, float *d_grads,
                        uint32_t batch, uint32_t nout, float mask_sum, float *loss) {
    clear_error();
    PSK_TRY(sel_guard(ctx, nout));
    if (!(mask_sum > 0.f)) return set_error(PSACAK_EINVAL, "mask sum must be positive");
    std::lock_guard<std::mutex> g(ctx->c.mu);
    Ctx &c = ctx->c;
    PSK_CUDA(cudaSetDevice(c.dev.id));
    cudaStream_t s = c.own_stream;
    float *d_loss = (float *)(c.d_scalars + 60);
    PSK_CUDA(cudaMemsetAsync(d_grads, 0, psacak_sel_param_count(nout) * sizeof(float), s));
    PSK_CUDA(cudaMemsetAsync(d_loss, 0, sizeof(float), s));
    if (batch > 0) {
        k_mlp_backward<<<batch, H, 0, s>>>(d_params, d_x, d_h1, d_h2, d_y, d_t, d_m, 1.f / mask_sum, nout, d_grads,
                                           d_loss);
        PSK_KCOUNT();
        PSK_LAUNCH_CHECK();
    }
    float hl = 0.f;
    PSK_CUDA(cudaMemcpyAsync(&hl, d_loss, sizeof(float), cudaMemcpyDeviceToHost, s));
    PSK_CUDA(cudaStreamSynchronize(s));
    if (loss) *loss = hl;
    return PSACAK_OK;
}

int psacak_mlp_adam(psacak_ctx *ctx, float *d_params, const float *d_grads, float *d_m1, float *d_m2,
                    uint64_t n_params, float lr, float beta1, float beta2, float eps, uint32_t step) {
    clear_error();
    if (!ctx || step == 0) return set_error(PSACAK_EINVAL, "bad adam arguments");
    std::lock_guard<std::mutex> g(ctx->c.mu);
    Ctx &c = ctx->c;
    PSK_CUDA(cudaSetDevice(c.dev.id));
    float c1 = 1.f - powf(beta1, (float)step), c2 = 1.f - powf(beta2, (float)step);
    uint64_t gsz = ceil_div(n_params, 256);
    k_adam<<<(uint32_t)(gsz < 1024 ? gsz : 1024), 256, 0, c.own_stream>>>(d_params, d_grads, d_m1, d_m2, n_params, lr,
                                                                         beta1, beta2, eps, c1, c2);
    PSK_KCOUNT();
    PSK_LAUNCH_CHECK();
    PSK_CUDA(cudaStreamSynchronize(c.own_stream));
    return PSACAK_OK;
}

int psacak_select_schedule(psacak_ctx *ctx, const float *d_params, uint32_t nout, const float *features,
                           uint32_t *choice, float *predictions) {
    clear_error();
    PSK_TRY(sel_guard(ctx, nout));
    if (!features || !choice) return set_error(PSACAK_EINVAL, "null features or choice");
    std::lock_guard<std::mutex> g(ctx->c.mu);
    Ctx &c = ctx->c;
    PSK_CUDA(cudaSetDevice(c.dev.id));
    cudaStream_t s = c.own_stream;
    float *d_x = (float *)(c.d_scalars + 44);
    uint32_t *d_out = c.d_scalars + 62;
    float *d_pred = (float *)(c.d_hist + 4096);  // KMAX floats of scratch
    PSK_CUDA(cudaMemcpyAsync(d_x, features, F * sizeof(float), cudaMemcpyHostToDevice, s));
    k_select<<<1, H, 0, s>>>(d_params, d_x, nout, d_out, d_pred);
    PSK_KCOUNT();
    PSK_LAUNCH_CHECK();
    uint32_t h = 0;
    PSK_CUDA(cudaMemcpyAsync(&h, d_out, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    if (predictions) PSK_CUDA(cudaMemcpyAsync(predictions, d_pred, nout * sizeof(float), cudaMemcpyDeviceToHost, s));
    PSK_CUDA(cudaStreamSynchronize(s));
    *choice = h;
    return PSACAK_OK;
}

}  // extern "C"
