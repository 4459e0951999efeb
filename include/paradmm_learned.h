/*
 * paradmm_learned.h -- learned warm start for batched circle packing
 * (libparadmm_b200.so).  No counterpart in the reference, which always starts
 * from a user-provided or random state (core/paradmm.c:188-375).
 *
 * A permutation-equivariant set MLP (3 layers, width 128, BF16 weights, FP32
 * accumulation) maps per-circle features of an instance's plain start (its
 * own position and radius, nearest-neighbour and wall distances, a
 * neighbour-repulsion vector, density counts, N and box aspect) to a guess of
 * the packing plain ADMM converges to.  The guess warm-starts the engine
 * (paradmm_gpu_warm_start); the ADMM residual decides, and instances that
 * do not converge within their budget are re-solved from the plain start.
 * Training (forward, backward, Adam) runs on the GPU with this library's own
 * kernels on packings the plain solver produced.
 */
#ifndef PARADMM_B200_PARADMM_LEARNED_H
#define PARADMM_B200_PARADMM_LEARNED_H

#include <stdint.h>
#include "paradmm_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct paradmm_setmlp paradmm_setmlp; /* opaque network + data set */

/* Number of FP32 parameters (W1 128x32, b1, W2 128x256, b2, W3 4x128, b3). */
int64_t paradmm_setmlp_num_params(void);

/* New network on `device`, weights drawn from a splitmix64 stream. */
int paradmm_setmlp_create(int device, uint64_t seed, paradmm_setmlp **out);
void paradmm_setmlp_destroy(paradmm_setmlp *net);
int paradmm_setmlp_get_params(paradmm_setmlp *net, float *params);
int paradmm_setmlp_set_params(paradmm_setmlp *net, const float *params);

/* Data set of n_inst instances: n_circles[b], box[2b], box[2b+1] = (W, H),
 * plain starts `init` and (for training) converged packings `target`, both
 * [cx, cy, r] per circle, instances consecutive.  Features are computed on
 * the device; rmax is the plain start's radius bound. */
int paradmm_setmlp_set_data(paradmm_setmlp *net, int n_inst, const int *n_circles, const double *box,
                            const double *init, const double *target, double rmax);

/* Adam on the data set's mean squared error (targets in units of the mean
 * spacing), `epochs` passes in mini-batches of batch_inst instances, learning
 * rate decaying linearly from lr to lr_end; per-epoch mean losses out. */
int paradmm_setmlp_train(paradmm_setmlp *net, int epochs, int batch_inst, float lr, float lr_end, double *losses);

/* Mean loss over the data set (no update). */
int paradmm_setmlp_eval(paradmm_setmlp *net, double *loss);

/* Gradients (FP32, paradmm_setmlp_num_params values) of the loss over
 * instances [b0, b0 + nb) of the data set, without an update. */
int paradmm_setmlp_gradients(paradmm_setmlp *net, int b0, int nb, float *grads, double *loss);

/* The features of every row of the data set (32 floats per circle). */
int paradmm_setmlp_features(paradmm_setmlp *net, float *out);

/* The proposal for every circle of the data set, [cx, cy, r] (host). */
int paradmm_setmlp_predict(paradmm_setmlp *net, const double *init, double *out);

/* Warm-starts every instance of a packing handle from `circles`
 * ([cx, cy, r] per circle, instances consecutive): Z = circles, X_e = Z_v(e),
 * pair and wall duals 0; with radius_duals = 1 the radius-factor duals are
 * set to the value the radius prox has at a fixed point with that radius
 * (a r^(a-1) / rho for exponent a), else 0. */
int paradmm_gpu_warm_start_all(paradmm_gpu *h, const double *circles, int radius_duals);

/* The same, then `dual_iters` rounds of the reference's optimal-initialisation
 * map on every factor's duals (paradmm_gpu_warm_start_duals with Uinit = the
 * duals above): X~ = prox_f(Z - U), U <- X~ - (Z - U)
 * (core/paradmm.c:349-357).  dual_iters = 0 is paradmm_gpu_warm_start_all. */
int paradmm_gpu_warm_start_all_duals(paradmm_gpu *h, const double *circles, int radius_duals, int dual_iters);

#ifdef __cplusplus
}
#endif

#endif
