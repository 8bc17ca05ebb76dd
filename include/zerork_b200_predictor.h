/*
 * zerork_b200_predictor.h -- the learned BDF predictor network.
 *
 * No counterpart in the reference (its integrator is CVODE's BDF, whose
 * predictor is the polynomial extrapolation of the step history).  A
 * multilayer perceptron with SiLU hidden layers, BF16 weights and
 * activations, FP32 accumulation, FP32 master weights and Adam moments,
 * trained and evaluated by the library's own tensor-core kernels.  Inputs
 * and targets are FP32 device arrays, row-major [n][n_in] and [n][n_out].
 * Parameter arrays for get/set are FP32 host arrays laid out layer by layer
 * with every dimension padded to a multiple of 16 (zrk_mlp_sizes gives the
 * totals).  Errors as in zerork_b200.h.
 */
#ifndef ZERORK_B200_PREDICTOR_H
#define ZERORK_B200_PREDICTOR_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct zrk_mlp_impl *zrk_mlp_t;

/* n_in -> layers x hidden (SiLU) -> n_out; seeded Kaiming-uniform weights. */
int zrk_mlp_create(int n_in, int hidden, int layers, int n_out, unsigned long long seed, zrk_mlp_t *out);
int zrk_mlp_free(zrk_mlp_t m);
int zrk_mlp_sizes(zrk_mlp_t m, long *n_weights, long *n_biases);
int zrk_mlp_get_params(zrk_mlp_t m, float *weights, float *biases);
int zrk_mlp_set_params(zrk_mlp_t m, const float *weights, const float *biases);
/* Gradients of the last zrk_mlp_gradients call (synchronizes the device). */
int zrk_mlp_get_grads(zrk_mlp_t m, float *weights, float *biases);
/* y[n][n_out] = net(x[n][n_in]); asynchronous on stream. */
int zrk_mlp_forward(zrk_mlp_t m, int n, const float *x, float *y, void *stream);
/* Forward + backward of the mean squared error over a batch of n rows (n a
 * multiple of 16): gradients stay on the device for zrk_mlp_adam; the sum of
 * squared errors is written to the device float *loss_sum_dev. */
int zrk_mlp_gradients(zrk_mlp_t m, int n, const float *x, const float *t, float *loss_sum_dev, void *stream);
/* One Adam step (Kingma and Ba, 2015) with the last gradients. */
int zrk_mlp_adam(zrk_mlp_t m, float lr, float beta1, float beta2, float eps, void *stream);

/* Attach a trained network to a cfd_plugin handle (struct
 * zerork_handle_impl *, include/zerork_cfd_plugin.h) as the learned BDF
 * predictor of its dense-block integrator: at the start of every step the
 * network's estimate of the state at t + h (inputs: log10 mass fractions
 * clamped at 1e-30, (T - 1500 K) / 1000 K, log10(P / 1 bar), log10(h);
 * targets: change of log10 mass fraction and (T' - T) / 100 K; both
 * standardised with the given per-column mean and standard deviation) is
 * the Newton starting iterate; after any rejection the step continues from
 * the polynomial predictor, and the error test is unchanged.  The network
 * must have nsp + 3 inputs, nsp + 1 outputs and layers no wider than 256,
 * and must outlive the handle's solves; net = NULL detaches it.  No
 * counterpart in the reference. */
struct zerork_handle_impl;
int zrk_plugin_set_predictor(struct zerork_handle_impl *h, zrk_mlp_t net, const float *x_mu,
                             const float *x_sd, const float *t_mu, const float *t_sd);

#ifdef __cplusplus
}
#endif
#endif
