/* silt_closure.h -- C ABI of the learned sub-grid flux closure.
 *
 * The closure stands in for the nested 2 cm tire sheets of `FluidCore::step`
 * (src/fluid_core.rs:6034-6128: refine -> fine pair -> restrict) on the
 * coarse window: a 3-layer 3 x 3 convolutional network (BF16 weights and
 * activations, FP32 accumulation on the tcgen05 tensor cores) reads the
 * coarse state around the vehicle and predicts, per coarse face, depth moved
 * across it, and per wet cell a velocity change, so that the window after the
 * coarse step (which then applies no tire shove) matches what the nested
 * sheets would have left. The correction moves depth between neighbouring
 * cells only, so the window's volume is conserved to the ledger. The nested sheets remain the fallback:
 * a window whose closure residual estimate exceeds the threshold steps nested
 * on one of its next steps.
 *
 * Network (one crop of CROP x CROP coarse cells centred on the vehicle):
 *   in  : 6 channels (water depth, slurry depth, water u, water v, bed,
 *         tire shove field), normalised, zero-padded to 16 channels;
 *   L1  : 3x3 conv 16 -> 32, ReLU;  L2 : 3x3 conv 32 -> 32, ReLU;
 *   L3  : 3x3 conv 32 -> 16 (8 used: water x-face, water z-face, slurry
 *         x-face, slurry z-face depth transfer; water u, water v, slurry u,
 *         slurry v change; normalised).
 * Activations are NHWC BF16 ([image][row][col][channel]); weights for the
 * forward pass are [cout][tap][cin] BF16, tap = 3 * (dy + 1) + (dx + 1).
 * The FP32 parameter vector (silt_closure_create, the training entry points)
 * holds, in order: W1 [9][16][32], b1 [32], W2 [9][32][32], b2 [32],
 * W3 [9][32][16], b3 [16] (weights as [tap][cin][cout]).
 *
 * Every device pointer below is CUDA device memory; `stream` is a
 * cudaStream_t (NULL = the legacy default stream). Calls are asynchronous.
 */
#ifndef SILT_CLOSURE_H
#define SILT_CLOSURE_H

#include <stdint.h>

#include "silt_sheet.h"

#ifdef __cplusplus
extern "C" {
#endif

#define SILT_CLOSURE_CROP 32
#define SILT_CLOSURE_CIN 16
#define SILT_CLOSURE_HIDDEN 32
#define SILT_CLOSURE_COUT 16
#define SILT_CLOSURE_IN_USED 6
#define SILT_CLOSURE_OUT_USED 8
/* FP32 parameters: 9*16*32 + 32 + 9*32*32 + 32 + 9*32*16 + 16. */
#define SILT_CLOSURE_NPARAM 18512
/* Normalisation block: 6 input means, 6 input inverse deviations, 8 output
 * scales (m of depth, then m/s, per unit of network output). */
#define SILT_CLOSURE_NNORM 20

/* Coupling of the tire sheets into the window (silt_set_coupling). */
#define SILT_COUPLING_NESTED 0  /* the reference: nested 2 cm sheets */
#define SILT_COUPLING_NONE 1    /* tires shove the coarse cells directly, no sheets */
#define SILT_COUPLING_CLOSURE 2 /* no sheets and no coarse shove: the learned face-flux
                                 * correction carries the tires' effect */

/* ---- Tensor-core kernels (inference and training) ---------------------- */

/* y = act(conv3x3(x, w) + bias) over n_img images of h x w pixels, zero
 * padding. (cin, cout) is one of (16, 32), (32, 32), (32, 16). `bias` may be
 * NULL. relu != 0 applies max(0, .). `gate` (NULL or NHWC BF16 with cout
 * channels) multiplies each output by (gate > 0): the ReLU derivative when
 * the call computes an input gradient. Writes `y_bf16` (NHWC, cout channels)
 * and/or `y_f32` (NHWC FP32). Any pointer output may be NULL. */
int silt_conv3x3_forward(const void* x_bf16, const void* w_bf16, const float* bias, const void* gate_bf16,
                         void* y_bf16, float* y_f32, int32_t n_img, int32_t h, int32_t w, int32_t cin,
                         int32_t cout, int32_t relu, void* stream);

/* Weight and bias gradients of y = conv3x3(x, w): dw[tap][cin][cout] +=
 * sum over pixels of x[p + tap][cin] * dy[p][cout], db[cout] += sum of dy.
 * Accumulates (FP32 atomics): zero dw and db first. (cin, cout) as above. */
int silt_conv3x3_wgrad(const void* x_bf16, const void* dy_bf16, float* dw, float* db, int32_t n_img, int32_t h,
                       int32_t w, int32_t cin, int32_t cout, void* stream);

/* Mean squared error of y[:, :n_out] against target (n_pix x n_out FP32),
 * weighted per pixel (NULL = 1): loss += sum w (y - t)^2 * scale (FP64), and
 * dy = 2 w (y - t) * scale as BF16 (channels >= n_out zero). */
int silt_closure_loss_grad(const float* y, const float* target, const float* pixel_weight, void* dy_bf16,
                           double* loss, int32_t n_pix, int32_t cout_pad, int32_t n_out, float scale, void* stream);

/* Loss of one closure step's correction, per crop of SILT_CLOSURE_CROP^2
 * cells. y: n_img crops x CROP^2 x SILT_CLOSURE_COUT FP32 network output
 * (channels 0..7 as above, in units of scale[c]; faces across the crop's
 * edge count as 0). t: n_img x CROP^2 x 8 FP32 targets: water and slurry
 * depth change (m), water u, v and slurry u, v change (m/s), and the water
 * and slurry weights of the velocity terms (1 where the cell is wet). loss +=
 * norm * sum over cells of [inv_var[l] (div_l - dh_l)^2 over the two layers +
 * inv_var[2 + k] w (y[4 + k] scale[4 + k] - dv_k)^2 over the four velocity
 * channels + lambda * sum of y[0..7]^2], with div the cell's inflow minus
 * outflow; dy = d loss / d y as BF16 (channels >= 8 zero). */
int silt_closure_step_loss_grad(const float* y, const float* t, const float* scale, const float* inv_var, float lambda,
                                void* dy_bf16, double* loss, int32_t n_img, float norm, void* stream);

/* One Adam step (bias-corrected) on n FP32 parameters. */
int silt_closure_adam(float* param, float* m, float* v, const float* grad, int32_t n, float lr, float beta1,
                      float beta2, float eps, int32_t step, void* stream);

/* FP32 [tap][cin][cout] weights -> BF16 forward [cout][tap][cin] and BF16
 * input-gradient [cin][8 - tap][cout] (the flipped, transposed kernel). */
int silt_closure_pack(const float* w, void* w_fwd_bf16, void* w_bwd_bf16, int32_t cin, int32_t cout, void* stream);

/* Whether a tensor-core kernel of this library gave up a bounded wait (its
 * mbarrier phase did not complete within the poll limit; the kernel then
 * skips its epilogue, frees its tensor memory and returns) since the last
 * call: *gave_up = 1 if so. Reads and clears the flag; synchronises stream.
 * No counterpart in the reference (it has no GPU kernels). */
int silt_closure_wait_status(int32_t* gave_up, void* stream);
/* Diagnostic of that path without a fault: one CTA waits, `polls` polls at
 * most (1..2^20), on an mbarrier phase nothing completes, gives up and sets
 * the flag silt_closure_wait_status reads. */
int silt_closure_wait_probe(int32_t polls, void* stream);

/* ---- The closure in the step -------------------------------------------- */

typedef struct silt_closure silt_closure;

/* Uploads a trained network: SILT_CLOSURE_NPARAM parameters and the
 * SILT_CLOSURE_NNORM normalisation block (host arrays), on `device`. */
int silt_closure_create(const float* params, int32_t n_params, const float* norm, int32_t device,
                        silt_closure** out);
int silt_closure_destroy(silt_closure* c);

/* Chooses how the sheet couples its tires (SILT_COUPLING_*). CLOSURE needs a
 * network; `threshold` is the residual estimate above which the next step
 * falls back to the nested sheets. The network must outlive the sheet's use
 * of it. */
int silt_set_coupling(silt_sheet* s, int32_t mode, silt_closure* net, float threshold);

/* The network input of the sheet's current state for this step's queued
 * tires (silt_push_tire): one crop, NHWC BF16 with SILT_CLOSURE_CIN
 * channels, written to the device buffer `x_bf16`; the crop's first coarse
 * cell (i, j) to `origin` (host, 2 ints). Does not consume the tires. */
int silt_closure_features(silt_sheet* s, silt_closure* net, void* x_bf16, int32_t* origin);

/* Closure statistics since the sheet was created. */
typedef struct {
    int64_t closure_steps;   /* steps corrected by the network */
    int64_t fallback_steps;  /* steps the residual estimate sent to the nested sheets */
    float last_residual;     /* residual estimate of the last corrected step (read one step late) */
    double moved_m3;         /* volume the corrections moved between cells (FP64) */
} silt_closure_stats;
int silt_get_closure_stats(silt_sheet* s, silt_closure_stats* out);

#ifdef __cplusplus
}
#endif

#endif
