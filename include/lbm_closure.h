/* Learned subgrid closure and on-device post-processing for 2D D2Q9 runs (sm_100a).
 *
 * No counterpart in the reference: it has no closure, and its post-processing
 * (python/boltzmann/utils/postproc.py:12-83) is numpy on the host.
 *
 * The closure is a 3-layer CNN on the coarse lattice: 3x3 convolutions with 4 -> 32 -> 32 -> 1
 * channels, GELU (tanh form) after the first two, zero padding at the domain edges. Inputs per
 * cell are (rho - 1, u_x, u_y, curl u), normalised and stored as BF16; weights are BF16 copies of an FP32
 * master vector; every product sum accumulates in FP32 (tensor cores for the 32 -> 32 layer, in
 * both directions). Its output, times a gain, is a per-cell relaxation-time correction that
 * lbm_set_omega_field() hands to the stencil.
 *
 * Layouts. Fields are row-major [batch][nx][ny] (y fastest), as the reference's numpy views;
 * `flags` is the reference's int32 cell-flag array [nx][ny], shared by every batch entry (walls
 * get zero features; walls and fixed cells are left out of the loss). Activations are
 * channels-last [batch][nx][ny][C]. BF16 arrays are raw 16-bit words (uint16_t).
 *
 * Parameter vector (floats, LBM_CLOSURE_PARAMS of them), in this order:
 *   w1 [32][9][4]   (out channel, tap, in channel; tap = 3 (dx + 1) + (dy + 1))
 *   b1 [32]
 *   w2 [32][9][32]
 *   b2 [32]
 *   w3 [9][32]
 *   b3 [1]
 * A gradient vector has the same layout. The BF16 mirror (`params_bf16`) is the same vector
 * rounded to nearest even; kernels read weights from it and biases from the FP32 vector.
 *
 * All calls are asynchronous on `stream` (a cudaStream_t; NULL = the legacy default stream) and
 * return an lbm_status; lbm_last_error() has the message.
 */
#ifndef LBM_CLOSURE_H
#define LBM_CLOSURE_H

#include <stddef.h>
#include <stdint.h>

#include "lbm_cuda.h"

#ifdef __cplusplus
extern "C" {
#endif

#define LBM_CLOSURE_CHANNELS 32
#define LBM_CLOSURE_PARAMS 10721
#define LBM_CLOSURE_OFF_W1 0
#define LBM_CLOSURE_OFF_B1 1152
#define LBM_CLOSURE_OFF_W2 1184
#define LBM_CLOSURE_OFF_B2 10400
#define LBM_CLOSURE_OFF_W3 10432
#define LBM_CLOSURE_OFF_B3 10720

/* curl of a 2D velocity field [nx][ny][2] into out [nx][ny], exactly as
 * postproc.calc_curl (python/boltzmann/utils/postproc.py:33-82) computes it with np.gradient:
 * d(u_x)/dy - d(u_y)/dx, central differences inside, one-sided first differences at the edges
 * (no periodic wrap). nx, ny >= 2. */
LBM_API int lbm_postproc_curl2d(const float* vel, int64_t nx, int64_t ny, float* out, void* stream);

/* curl of a 3D velocity field [nx][ny][nz][3] into out [nx][ny][nz][3] (postproc.py:69-77). */
LBM_API int lbm_postproc_curl3d(const float* vel, int64_t nx, int64_t ny, int64_t nz, float* out,
                                void* stream);

/* |u| of an [n][dim] vector field (postproc.calc_vmag, postproc.py:12-30). */
LBM_API int lbm_postproc_vmag(const float* vel, int64_t n, int dim, float* out, void* stream);

/* Features of `batch` coarse states: x [batch][nx][ny][4] BF16 with
 * x_c = (v_c - norm[c]) * norm[4 + c] for v = (rho - 1, u_x, u_y, curl u), and 0 on walls.
 * `norm` is a host array of 8 floats. */
LBM_API int lbm_closure_features(const float* rho, const float* vel, const int32_t* flags,
                                 int64_t nx, int64_t ny, int64_t batch, const float* norm,
                                 uint16_t* x, void* stream);

/* Forward pass. z1, a1, z2, a2 ([batch][nx][ny][32]; z FP32 pre-activations, a BF16 GELU outputs)
 * receive the activations a backward pass needs; z1 and z2 may be NULL (inference). y gets the
 * output [batch][nx][ny] (FP32). */
LBM_API int lbm_closure_forward(const float* params, const uint16_t* params_bf16, const uint16_t* x,
                                int64_t nx, int64_t ny, int64_t batch, float* z1, uint16_t* a1,
                                float* z2, uint16_t* a2, float* y, void* stream);

/* Bytes of device workspace lbm_closure_loss and lbm_closure_backward need for this shape. */
LBM_API int64_t lbm_closure_workspace_bytes(int64_t nx, int64_t ny, int64_t batch);

/* Masked mean-squared error over the cells that are neither walls nor fixed:
 * loss = sum m (y - t)^2 / count, dy = 2 m (y - t) / count (FP32, [batch][nx][ny]), with
 * count = batch x (number of such cells). `loss` is a device double. */
LBM_API int lbm_closure_loss(const float* y, const float* target, const int32_t* flags, int64_t nx,
                             int64_t ny, int64_t batch, float* dy, double* loss, void* workspace,
                             void* stream);

/* Backward pass: the gradient of the loss with respect to every parameter into `grad`
 * (LBM_CLOSURE_PARAMS floats, overwritten), from the forward's activations and dy. The
 * gradients of the pre-activations are rounded to BF16 before they enter any product sum;
 * sums run in FP32 per tile and are added across tiles in a fixed order (deterministic). */
LBM_API int lbm_closure_backward(const float* params, const uint16_t* params_bf16,
                                 const uint16_t* x, const float* z1, const uint16_t* a1,
                                 const float* z2, const uint16_t* a2, const float* dy, int64_t nx,
                                 int64_t ny, int64_t batch, float* grad, void* workspace,
                                 void* stream);

/* One Adam step (bias-corrected, step >= 1) on the FP32 parameters, then refreshes the BF16
 * mirror. m and v are FP32 moment vectors of LBM_CLOSURE_PARAMS floats. */
LBM_API int lbm_closure_adam(float* params, uint16_t* params_bf16, const float* grad, float* m,
                             float* v, float lr, float beta1, float beta2, float eps, int64_t step,
                             void* stream);

/* Rounds the FP32 parameters into the BF16 mirror. */
LBM_API int lbm_closure_sync_bf16(const float* params, uint16_t* params_bf16, void* stream);

/* Relaxation field from the network output y [nx][ny]:
 * omega = 1 / (tau0 + min(max_dtau, gain * max(y, 0))) on cells that are neither walls nor fixed,
 * 1 / tau0 elsewhere (the stencil relaxes fixed cells with 1 regardless). */
LBM_API int lbm_closure_omega(const float* y, const int32_t* flags, int64_t nx, int64_t ny,
                              float tau0, float gain, float max_dtau, float* omega, void* stream);

/* Inference in one kernel: the relaxation field omega [nx][ny] of lbm_closure_omega, computed
 * from the coarse state (rho [nx][ny], vel [nx][ny][2], flags) through the features and the three
 * layers without any intermediate array in global memory (each tile recomputes its halo in shared
 * memory; all three layers on tensor cores, the 32 -> 32 layer as tcgen05 MMAs with TMEM
 * accumulators). Equal to lbm_closure_features + lbm_closure_forward +
 * lbm_closure_omega up to the FP32 summation order of layers 1 and 3. `norm` is a host array of
 * 8 floats. */
LBM_API int lbm_closure_relaxation(const float* params, const uint16_t* params_bf16,
                                   const float* rho, const float* vel, const int32_t* flags,
                                   int64_t nx, int64_t ny, const float* norm, float tau0,
                                   float gain, float max_dtau, float* omega, void* stream);

/* Which kernel runs layer 2 (32 -> 32 channels) of lbm_closure_forward and the transposed conv of
 * lbm_closure_backward, process-wide: LBM_CLOSURE_LAYER2_TCGEN05 (default; fifth-generation tensor
 * cores, accumulators in tensor memory) or LBM_CLOSURE_LAYER2_WARP_MMA (warp-level mma.sync). Both
 * take BF16 operands and accumulate in FP32; they differ only in summation order. No reference
 * counterpart. */
#define LBM_CLOSURE_LAYER2_TCGEN05 0
#define LBM_CLOSURE_LAYER2_WARP_MMA 1
LBM_API int lbm_closure_set_layer2_kernel(int kind);

/* Polls that the lbm_closure_relaxation kernel makes, on the current device, while waiting for
 * its tensor-core products before it gives up (polls < 0: the default, 2^22). A kernel that gives
 * up records it for lbm_closure_status, still waits (with the default bound) for the products in
 * flight, frees its tensor memory and returns; 0 makes the wait give up at once, a way to exercise
 * that path. Synchronous. No reference counterpart. */
LBM_API int lbm_closure_set_spin_limit(int64_t polls);

/* LBM_OK, or LBM_ERR_STATE when a lbm_closure_relaxation kernel on the current device gave up
 * waiting for its tensor-core products (bounded wait) since the last call; its omega is then
 * incomplete. Synchronous; clears the condition. */
LBM_API int lbm_closure_status(void);

/* Box filter of a fine state onto the coarse lattice (factor f, nx and ny multiples of f):
 * rho_c, vel_c ([nx/f][ny/f], [..][2]) and c_c (if c != NULL) are block means; sgs gets the
 * square root of the subgrid kinetic energy, sqrt(max(0, (mean(|u|^2) - |mean u|^2) / 2)). */
LBM_API int lbm_closure_coarsen(const float* rho, const float* vel, const float* c, int64_t nx,
                                int64_t ny, int factor, float* rho_c, float* vel_c, float* c_c,
                                float* sgs, void* stream);

#ifdef __cplusplus
}
#endif

#endif
