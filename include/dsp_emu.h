/*
 * dsp_emu.h — C ABI of libdsp_emu.so: the learned flux emulator of the B200
 * DISORT engine (no counterpart in the reference, which has no learned part).
 *
 * An MLP maps per-column features to log-normalised flux profiles:
 *   n_in features -> n_hidden_layers x (hidden, GELU) -> n_heads heads of n_out,
 * BF16 weights and activations, FP32 accumulation on the tcgen05 tensor cores,
 * FP32 master weights updated by a fused Adam kernel.  Widths are padded
 * internally to multiples of 64; padded weights stay zero.
 *
 * All array arguments are device pointers on the emulator's device and all
 * work is queued on its stream.  Features are BF16 stored as uint16_t bit
 * patterns, row-major [rows][in_pad] with in_pad = dsp_emu_input_stride().
 * Predictions are FP32 [rows][n_heads * n_out] (head-major within a row).
 */
#ifndef DSP_EMU_H
#define DSP_EMU_H

#include <stdint.h>

#include "dsp.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct dsp_emu_s* dsp_emu;

typedef struct dsp_emu_config {
  int32_t n_in;            /* input features (e.g. 247) */
  int32_t hidden;          /* hidden width, a multiple of 128 (e.g. 512) */
  int32_t n_hidden_layers; /* hidden layers (e.g. 4) */
  int32_t n_out;           /* outputs per head (e.g. 82) */
  int32_t n_heads;         /* ensemble heads (e.g. 2) */
  int32_t batch;           /* training batch (multiple of 128) */
  uint64_t seed;           /* weight initialisation */
} dsp_emu_config;

dsp_status dsp_emu_create(int32_t device, void* stream, const dsp_emu_config* cfg, dsp_emu* out);
dsp_status dsp_emu_destroy(dsp_emu emu);
const char* dsp_emu_last_error(dsp_emu emu);
int32_t dsp_emu_input_stride(dsp_emu emu);

/* Training set: feats [n][in_pad] BF16, targets [n][n_out] FP32, optional
 * per-(row, head) loss weights [n][n_heads] (NULL: all 1).  Copied into the
 * emulator (shuffled copies are made per epoch). */
dsp_status dsp_emu_set_data(dsp_emu emu, const uint16_t* feats, const float* targets, const float* head_weights,
                            int64_t n);

/* Adam (beta 0.9 / 0.999, eps 1e-8), cosine learning-rate decay from lr to
 * lr_min over all steps of all epochs; one pass over shuffled batches per epoch.
 * epoch_loss (host, [epochs] or NULL) receives the epoch's training loss per row: the
 * squared errors of the n_out outputs summed (not averaged), weighted and summed over
 * the heads, averaged over the rows. */
dsp_status dsp_emu_train(dsp_emu emu, int32_t epochs, float lr, float lr_min, uint64_t shuffle_seed,
                         float* epoch_loss);

/* Forward pass (inference): preds [rows][n_heads * n_out] FP32. */
dsp_status dsp_emu_forward(dsp_emu emu, const uint16_t* feats, int64_t rows, float* preds);

/* One forward + backward pass on the first `batch` rows of the training set,
 * without an update: gradients of the training loss w.r.t. every parameter,
 * written to `grads` (device, dsp_emu_param_count() floats, parameter order). */
dsp_status dsp_emu_gradients(dsp_emu emu, float* grads, float* loss);

/* Parameters in order W_1, b_1, ..., W_L, b_L with W_i [out_pad][in_pad]
 * row-major and the padded widths of dsp_emu_layer_dims; host FP32 arrays. */
int64_t dsp_emu_param_count(dsp_emu emu);
dsp_status dsp_emu_layer_dims(dsp_emu emu, int32_t layer, int32_t* in_pad, int32_t* out_pad);
dsp_status dsp_emu_get_params(dsp_emu emu, float* host);
dsp_status dsp_emu_set_params(dsp_emu emu, const float* host);

/* Kernel-level entry for tests and profiling: C[M][N] = A[M][K] * B[N][K]^T,
 * BF16 in, FP32 out, on the emulator's GEMM (K a multiple of 8). */
dsp_status dsp_emu_gemm_bf16(dsp_emu emu, const uint16_t* A, const uint16_t* B, float* C, int32_t M, int32_t N,
                             int32_t K);

/* Self-test of the device-side bounded waits: a kernel waits `cycles` clock
 * cycles (at most 2^31) on an mbarrier that nothing arrives on, with no copy or
 * MMA in flight, gives up and sets the error flag the GEMMs use; the call
 * returns DSP_ERR_TIMEOUT read from that flag, then clears the flag so that the
 * emulator stays usable. */
dsp_status dsp_emu_wait_selftest(dsp_emu emu, int64_t cycles);

/* Gate: a row falls back to the FP64 solver when any raw feature lies outside
 * [lo, hi] (per feature, n_in values each) or when its heads disagree on the
 * reconstructed fluxes F_h,k = scale_r * (exp(pred_h,k * sd_k + mu_k) - eps) + add_r,k
 * (scale [rows] and add [rows][n_out] optional: NULL means 1 and 0):
 * max_k |F_0k - F_1k| > rel_tol * max(|F_k|, floor_frac * max_k |F_k|), F = head mean.
 * Writes F to flux [rows][n_out], the fallback flag to fallback[rows] and the
 * fallback rows to idx (count in *n_fallback, device int32). */
dsp_status dsp_emu_gate(dsp_emu emu, const float* raw_feats, int32_t raw_stride, const float* lo, const float* hi,
                        const float* preds, const float* mu, const float* sd, const float* scale, const float* add,
                        float eps, float rel_tol, float floor_frac, int64_t rows, float* flux, int32_t* fallback,
                        int32_t* idx, int32_t* n_fallback);

#ifdef __cplusplus
}
#endif

#endif /* DSP_EMU_H */
