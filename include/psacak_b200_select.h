/*
 * psacak_b200_select.h -- learned schedule selection.
 *
 * A small fp32 MLP (16 -> 64 -> 64 -> K, ReLU) reads 16 cheap statistics of
 * a text and predicts log2(build milliseconds) of each of K candidate
 * schedules (psacak_schedule values); the smallest prediction wins.  Every
 * schedule builds the same suffix array, so the selector only changes speed.
 * None of this has a counterpart in hucsmn/psacak, which has compile-time
 * constants only (src/psacak8.rs:11-15, src/psacak32.rs:14-18).
 *
 * Parameters are one fp32 array of psacak_sel_param_count(K) values:
 * W1[16][64], b1[64], W2[64][64], b2[64], W3[64][K], b3[K].  All array
 * arguments are device pointers unless named `features` / `loss` /
 * `choice` / `predictions` (host).
 */
#ifndef PSACAK_B200_SELECT_H
#define PSACAK_B200_SELECT_H

#include "psacak_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

#define PSACAK_SEL_FEATURES 16
#define PSACAK_SEL_HIDDEN 64
#define PSACAK_SEL_MAX_OUT 32

/* Number of fp32 parameters of the network with `nout` outputs. */
PSACAK_API uint64_t psacak_sel_param_count(uint32_t nout);

/*
 * 16 statistics of a text (width 1 = bytes, 4 = u32 symbols) from a sample of
 * <= 65536 evenly spaced positions and 2048 windows of 16 symbols: log length,
 * width, distinct-symbol sketch, LMS density, S-type share, equal-neighbour
 * share, sampled repeat rate (duplicate windows), symbol entropy, largest
 * symbol, and products of these; the last value is 1.
 */
PSACAK_API int psacak_text_stats(psacak_ctx *ctx, const void *d_text, uint64_t n, int width, float *features);

/* Forward pass of `batch` feature rows d_x[batch][16] into d_y[batch][nout];
 * d_h1 / d_h2 (nullable) keep the hidden activations for the backward pass. */
PSACAK_API int psacak_mlp_forward(psacak_ctx *ctx, const float *d_params, const float *d_x, float *d_y, float *d_h1,
                                  float *d_h2, uint32_t batch, uint32_t nout);

/* Gradients of sum(M * (Y - T)^2) / mask_sum into d_grads (overwritten);
 * *loss receives the loss. */
PSACAK_API int psacak_mlp_backward(psacak_ctx *ctx, const float *d_params, const float *d_x, const float *d_h1,
                                   const float *d_h2, const float *d_y, const float *d_t, const float *d_m,
                                   float *d_grads, uint32_t batch, uint32_t nout, float mask_sum, float *loss);

/* One Adam step (step counts from 1). */
PSACAK_API int psacak_mlp_adam(psacak_ctx *ctx, float *d_params, const float *d_grads, float *d_m1, float *d_m2,
                               uint64_t n_params, float lr, float beta1, float beta2, float eps, uint32_t step);

/* Inference: the index of the schedule with the smallest predicted time. */
PSACAK_API int psacak_select_schedule(psacak_ctx *ctx, const float *d_params, uint32_t nout, const float *features,
                                      uint32_t *choice, float *predictions);

/*
 * i.i.d. text on the device for load generation: symbol i drawn from
 * splitmix64(seed, i); width 1 draws from the `alphabet_size` listed bytes,
 * width 4 draws u32 symbols uniform on [0, alphabet_size).  Asynchronous on
 * `stream` (NULL = the context's stream).
 */
PSACAK_API int psacak_gen_iid_dev(psacak_ctx *ctx, void *d_out, uint64_t n, int width, const uint8_t *alphabet,
                                  uint32_t alphabet_size, uint64_t seed, void *stream);

#ifdef __cplusplus
}
#endif
#endif
