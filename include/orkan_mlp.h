/*
 * orkan_mlp.h - FP32 multilayer perceptron used as a surrogate of the batched simulator's
 * expectation values (no counterpart in the reference's API).
 *
 *     y = W3 . gelu(W2 . gelu(W1 . x + b1) + b2) + b3        (x: n_in, hidden: h, y: scalar)
 *
 * with gelu(z) = z Phi(z) (exact, erf form).  Training minimises the mean squared error
 * with Adam (beta1 0.9, beta2 0.999, eps 1e-8).  Every kernel is hand-written FP32 CUDA
 * (tiled GEMMs with fused bias/GELU epilogues, deterministic reductions); parameters and
 * optimiser state live in device memory.  Pointers marked _dev are device pointers; all
 * calls are asynchronous on `stream` unless stated.  Functions return 0 or a cudaError_t.
 *
 * Parameter vector layout (orkan_mlp_params): W1 [n_in][h], b1 [h], W2 [h][h], b2 [h],
 * W3 [h], b3 [1]  (row-major, W[i][j] multiplies input i into output j).
 */
#ifndef ORKAN_MLP_H
#define ORKAN_MLP_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orkan_mlp orkan_mlp_t;

/* Create on the current device with deterministic initial weights (uniform in
 * +-sqrt(6 / fan_in) for W, zero biases) from `seed`; max_batch bounds every batch. */
int orkan_mlp_create(orkan_mlp_t **out, unsigned n_in, unsigned hidden, unsigned max_batch, unsigned long long seed);
void orkan_mlp_destroy(orkan_mlp_t *m);

/* Number of parameters, and host copies of the parameter vector (synchronous). */
size_t orkan_mlp_param_count(const orkan_mlp_t *m);
int orkan_mlp_get_params(const orkan_mlp_t *m, float *host);
int orkan_mlp_set_params(orkan_mlp_t *m, const float *host);      /* also resets Adam */

/* y_dev[b] = f(x_dev[b][:]) for b < batch. */
int orkan_mlp_forward(orkan_mlp_t *m, const float *x_dev, unsigned batch, float *y_dev, void *stream);

/* Loss L = mean_b (f(x_b) - t_b)^2 and its gradients: grad_dev (param_count floats, the
 * parameter-vector layout) and, when gx_dev is not NULL, dL/dx [batch][n_in].  loss_dev
 * receives L (one float).  No parameter changes. */
int orkan_mlp_gradients(orkan_mlp_t *m, const float *x_dev, const float *t_dev, unsigned batch, float *loss_dev,
                        float *grad_dev, float *gx_dev, void *stream);

/* Train on count samples (x_dev [count][n_in], t_dev [count]) for `epochs` epochs of
 * minibatches of `batch` samples (the last partial batch of an epoch is dropped) with
 * learning rate lr; each epoch visits the samples in the order i -> (a_e i + c_e) mod
 * count for a per-epoch a_e coprime to count, drawn from `seed`.  The step sequence is
 * one captured CUDA graph replayed per step.  loss_dev (may be NULL) receives the mean
 * training loss of the last epoch.  Adam's state carries over between calls. */
int orkan_mlp_train(orkan_mlp_t *m, const float *x_dev, const float *t_dev, unsigned count, unsigned epochs,
                    unsigned batch, float lr, unsigned long long seed, float *loss_dev, void *stream);

/* Proposals: `steps` steps of Adam ascent (lr) on the inputs x_dev [count][n_in] (in
 * place) to maximise f, each coordinate clamped to [lo, hi]; y_dev (may be NULL) receives
 * f at the final inputs. */
int orkan_mlp_ascend(orkan_mlp_t *m, float *x_dev, unsigned count, unsigned steps, float lr, float lo, float hi,
                     float *y_dev, void *stream);

/* Kernel launches issued by this module since load (all MLP entry points). */
unsigned long long orkan_mlp_launch_count(void);

#ifdef __cplusplus
}
#endif

#endif /* ORKAN_MLP_H */
