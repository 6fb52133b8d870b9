/* diva_cnn.h -- the learned warm start of the DIVA solve: a small encoder-decoder
 * network that predicts the state the viscosity iteration carries from one iteration
 * to the next -- the depth-averaged velocities u_vav_cx / v_vav_cy, the basal shear
 * stress taub_cx / taub_cy and the 3D effective viscosity visc_eff_3D_a -- from the
 * fields the solve reads, so that solve_DIVA starts close to its fixed point.  The
 * Picard loop always runs to its own tolerance, so the network only changes where the
 * iteration starts, never what it converges to.
 *
 * The reference has no counterpart: solve_DIVA (src/ice_velocity_module.f90:249-374)
 * starts from whatever those fields hold (zero at initialisation, the previous
 * solution during a run).  The velocities alone are not enough: the first iteration's
 * vertical shear (calc_vertical_shear_strain_rates, :664-721) is computed from the
 * previous viscosity and basal stress, so a context given the converged velocities
 * but a cold viscosity and stress iterates as long as a cold start.  diva_cnn_predict
 * writes the predicted velocities and completes the rest of the state from them
 * (diva_complete_state), or writes all five fields; a caller places it before
 * diva_solve_diva.
 *
 * Network (one instance per grid size; all sizes in cells of the a-grid):
 *   input  16 channels on the a-grid padded to multiples of 4 (8 used, see below)
 *   e1a 3x3 16->32, e1b 3x3 32->32                       full resolution
 *   avg-pool 2x2; e2a 3x3 32->64, e2b 3x3 64->64           1/2
 *   avg-pool 2x2; ba 3x3 64->128, bb 3x3 128->64           1/4
 *   nearest x2, concat e2b; d2a 3x3 128->64, d2b 3x3 64->32 1/2
 *   nearest x2, concat e1b; d1a 3x3 64->32, d1b 3x3 32->32  full
 *   head 1x1 32->20 (no activation); every 3x3 layer has a bias and a ReLU
 * Input channels: Hi/1000, Hb/1000, 100 dHs/dx, 100 dHs/dy, log10(A_flow_vav)+17,
 * log10(beta_sq)-4, mask_sheet, mask_shelf (cells outside the grid: zero).
 * Output channels at a-grid cell (j,i): 0 asinh(u_vav_cx(j,i) / 10 m/yr) and
 * 2 asinh(taub_cx(j,i) / 1000 Pa) for i < nx-1; 1 asinh(v_vav_cy(j,i) / 10 m/yr) and
 * 3 asinh(taub_cy(j,i) / 1000 Pa) for j < ny-1; 4+k log10(visc_eff_3D_a(k,j,i)) - 8 for
 * the nz <= 16 layers; the remaining channels are unused.  The training loss is the
 * weighted sum of squared errors over the valid entries divided by their number.
 *
 * Arithmetic: BF16 activations and weights, FP32 accumulation in tensor memory
 * (tcgen05.mma, kind::f16), FP32 master weights and Adam moments.
 *
 * Flat weight vector (diva_cnn_weights): for each 3x3 layer in the order above its
 * weights as [tap][cout][cin] (tap = 3*(dy+1) + (dx+1); the output at (y,x) reads the
 * input at (y+dy, x+dx)), then its bias [cout]; then the head [20][32] and its bias [20].
 */
#ifndef DIVA_CNN_H
#define DIVA_CNN_H

#include <stdint.h>
#include "diva.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct diva_cnn diva_cnn_t;

/* A network for contexts of ny x nx a-grid cells and nz layers (nz <= 16, else
 * DIVA_UNSUPPORTED): minibatches of up to `batch` samples, a device-resident training
 * set of up to `capacity` samples, weights initialised from `seed` (He-normal, zero
 * biases).  Runs on its own stream. */
int32_t diva_cnn_create(diva_cnn_t** net, int32_t ny, int32_t nx, int32_t nz, int32_t batch, int32_t capacity,
                        uint64_t seed);
int32_t diva_cnn_destroy(diva_cnn_t* net);

/* Number of floats of the flat weight vector. */
int32_t diva_cnn_num_weights(const diva_cnn_t* net, int64_t* n);

/* direction 0: copy the FP32 master weights to host[n]; 1: set them from host[n]
 * (and reset the Adam moments).  n must equal diva_cnn_num_weights. */
int32_t diva_cnn_weights(diva_cnn_t* net, float* host, int64_t n, int32_t direction);

/* Append the context's current state as a training sample: the input channels from
 * its fields and the targets from its u_vav_cx, v_vav_cy, taub_cx, taub_cy and
 * visc_eff_3D_a (call after a converged solve).  The context must have the network's
 * grid size. */
int32_t diva_cnn_add_sample(diva_cnn_t* net, diva_ctx_t* ctx);
int32_t diva_cnn_num_samples(const diva_cnn_t* net, int32_t* n);

/* Weights of the 20 output channels in the training loss (default 1 each; >= 0).  The
 * default predict mode uses only channels 0 and 1 (the velocities, the rest of the
 * state completed from them), so weights {1, 1, 0, ...} spend the network's capacity
 * on those. */
int32_t diva_cnn_set_loss_weights(diva_cnn_t* net, const float* w, int32_t n);

/* `epochs` passes of Adam (lr, beta1 0.9, beta2 0.999, eps 1e-8) over the training
 * set in minibatches, the order shuffled from `seed`; *loss = mean masked squared
 * error of the last epoch.  DIVA_NAN_DETECTED if an epoch's loss is not finite
 * (training diverged; reset the weights with diva_cnn_weights before using them). */
int32_t diva_cnn_train(diva_cnn_t* net, int32_t epochs, float lr, uint64_t seed, float* loss);

/* Warm-start the context from the network's prediction for its current fields.
 * complete_sweeps > 0: set u_vav_cx and v_vav_cy from the prediction, then derive the
 * viscosity and basal stress that belong to them with diva_complete_state(ctx,
 * complete_sweeps) (the more robust choice: measured on 20 km ice caps with the
 * oracle, 10 sweeps after a predicted velocity field cut the viscosity iterations by
 * a fifth and lengthened one case of twenty; 30 or 60 sweeps gained one iteration
 * more, because the guess's own error dominates).  complete_sweeps = 0: set all five
 * state fields from the prediction.  On the context's stream, synchronised before
 * return. */
int32_t diva_cnn_predict(diva_cnn_t* net, diva_ctx_t* ctx, int32_t complete_sweeps);

/* Device-buffer forms for tests and callers with their own data (pointers are device
 * memory; n <= batch).  feat: [n][Hp][Wp][16] BF16 with Hp, Wp = ny, nx rounded up to
 * multiples of 4; out: [n][Hp][Wp][20] FP32; tgt like out. */
int32_t diva_cnn_padded_shape(const diva_cnn_t* net, int32_t* Hp, int32_t* Wp);
int32_t diva_cnn_forward(diva_cnn_t* net, const void* feat, float* out, int32_t n);

/* One Adam step on a device batch; *loss is the batch's masked mean squared error
 * before the step.  The gradient of that loss stays readable through diva_cnn_grads
 * (same layout as the weight vector) until the next step. */
int32_t diva_cnn_train_step(diva_cnn_t* net, const void* feat, const float* tgt, int32_t n, float lr,
                            float* loss);
int32_t diva_cnn_grads(diva_cnn_t* net, float* host, int64_t n);

#ifdef __cplusplus
}
#endif
#endif
