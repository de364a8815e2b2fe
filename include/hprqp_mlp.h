/*
 * hprqp_mlp.h — the warm-start network of libhprqp: a 3-layer MLP
 * (n_in -> width -> width -> n_out, ReLU) with BF16 weights and activations,
 * FP32 accumulation, FP32 master weights and Adam, trained and evaluated by
 * the library's own CUDA kernels.
 *
 * It proposes a starting point (and log sigma) for a new instance of a
 * problem family; hprqp_solve then starts from that proposal and certifies
 * the result with the unmodified HPR iteration, so a poor proposal costs
 * iterations, never correctness.  No counterpart in the reference (its warm
 * start is the user-supplied initial_x / initial_y, src/algorithm.jl:1783).
 *
 * Host arrays are row-major float32: X is rows x n_in, T and Y rows x n_out.
 * Parameter vectors are [W1, b1, W2, b2, W3, b3] with W row-major (out x in).
 */
#ifndef HPRQP_MLP_H
#define HPRQP_MLP_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct hprqp_mlp* hprqp_mlp_handle;

/* Create a network on `device`; weights He-uniform from `seed`, biases 0.
 * `batch` is the largest number of rows per train/gradient call. */
int hprqp_mlp_create(hprqp_mlp_handle* h, int32_t device, int32_t n_in, int32_t width, int32_t n_out,
                     int32_t batch, uint64_t seed);

/* One Adam step (lr; beta 0.9/0.999) on the mean-squared-error loss
 * 0.5/rows * sum ||f(X_r) - T_r||^2; returns that loss before the step. */
int hprqp_mlp_train_batch(hprqp_mlp_handle h, const float* X, const float* T, int32_t rows, float lr,
                          double* loss_out);

/* Loss and its gradient with respect to every parameter (same layout as the
 * parameter vector), without updating; for gradient checks. */
int hprqp_mlp_gradients(hprqp_mlp_handle h, const float* X, const float* T, int32_t rows, float* grads,
                        double* loss_out);

/* Y = f(X) for any number of rows. */
int hprqp_mlp_predict(hprqp_mlp_handle h, const float* X, int64_t rows, float* Y);

/* Read / write the FP32 master parameters (params may be NULL to query count). */
int hprqp_mlp_get_params(hprqp_mlp_handle h, float* params, int64_t* count);
int hprqp_mlp_set_params(hprqp_mlp_handle h, const float* params);

const char* hprqp_mlp_last_error(hprqp_mlp_handle h);
int hprqp_mlp_destroy(hprqp_mlp_handle h);

#ifdef __cplusplus
}
#endif
#endif /* HPRQP_MLP_H */
