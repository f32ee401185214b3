/*
 * aeolus_b200_unet.h -- C ABI of the learned preconditioner: a 3-level
 * convolutional U-Net (16 / 32 / 32 channels, BF16 weights and activations,
 * FP32 accumulation and FP32 master weights) whose 3x3x3 convolutions and
 * weight gradients run as tcgen05 implicit GEMMs, trained on the GPU with
 * Adam on residual -> error pairs of the plain solver.  It serves as the
 * preconditioner of flexible CG in aeolus_b200_mgpcg.h (AEO_PC_LEARNED).
 *
 * This part has no counterpart in the reference, whose pressure solvers are
 * FFT, multigrid and CG (src/Multigrid.jl, src/Backends.jl:1511-1589); the
 * learned preconditioner is new here and never changes the converged
 * answer: the CG it sits in still stops at ||r|| <= tol ||b||.
 *
 * Grids: nx, ny, nz multiples of 4 (two 2x2x2 poolings); at every level nx
 * a multiple or a divisor of 128 (tiles of 128 cells) and ny a multiple of
 * the rows such a tile spans.  Fields are interior-only FP64 arrays, x
 * fastest, as in aeolus_b200_mgpcg.h.  Parameters are one flat FP32 array:
 * per layer (e1a, e1, e2a, e2, e3a, e3, d2, d1, out) the weights
 * W[27][c_out][c_in] (tap (dz+1)*9 + (dy+1)*3 + (dx+1)) then the biases.
 */
#ifndef AEOLUS_B200_UNET_H
#define AEOLUS_B200_UNET_H

#include <stdint.h>

#include "aeolus_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct aeo_unet aeo_unet;

/* number of FP32 parameters */
int64_t aeo_unet_param_count(void);
/* He-normal initial weights from `seed`, zero biases */
aeo_status aeo_unet_create(int32_t nx, int32_t ny, int32_t nz, uint64_t seed, int32_t device, aeo_unet** out);
aeo_status aeo_unet_destroy(aeo_unet* h);
aeo_status aeo_unet_set_params(aeo_unet* h, const float* params);
/* params and/or grads (accumulated by aeo_unet_gradients) may be NULL */
aeo_status aeo_unet_get_params(aeo_unet* h, float* params, float* grads);
/* fluid mask (1 fluid, 0 solid): a network input and the output mask */
aeo_status aeo_unet_set_mask(aeo_unet* h, const float* fluid);
/* the error scale: z = out_scale / s * network output, s = the input scale
 * that gives r unit RMS over the fluid */
aeo_status aeo_unet_set_out_scale(aeo_unet* h, double out_scale);
/* z = M r (host arrays) */
aeo_status aeo_unet_apply(aeo_unet* h, const double* r, double* z);
/* forward and backward on one pair (r, e = A^-1 r), gradients replaced (not
 * accumulated across calls); loss = mean over fluid cells of the squared
 * difference of the mean-free network output and the mean-free error scaled
 * to unit RMS on the fluid (flexible CG is invariant to the scale of each
 * preconditioner application, so only the error's shape is learned) */
aeo_status aeo_unet_gradients(aeo_unet* h, const double* r, const double* e, double* loss);
/* aeo_unet_gradients then one Adam step (beta 0.9 / 0.999, eps 1e-8) */
aeo_status aeo_unet_train_step(aeo_unet* h, const double* r, const double* e, double lr, double* loss);
/* an activation of the last forward pass as FP32, channels last: 0 x,
 * 1 e1a, 2 e1, 3 p1, 4 e2a, 5 e2, 6 p2, 7 e3a, 8 e3, 9 u2, 10 d2, 11 u1,
 * 12 d1, 13 z (one channel) */
aeo_status aeo_unet_activation(aeo_unet* h, int32_t which, float* out);
/* mean device ms of: 0 a forward pass, 1 forward + backward, 2 one
 * full-resolution 16->16 convolution, 3 its weight gradient */
aeo_status aeo_unet_profile(aeo_unet* h, int32_t what, int32_t reps, double* ms);
const char* aeo_unet_last_error(const aeo_unet* h);

#ifdef __cplusplus
}
#endif
#endif
