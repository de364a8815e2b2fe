/*
 * hprqp_batch.h — batched HPR solves in one launch sequence (libhprqp), for
 * two families:
 *  - LASSO problems as built by the reference's build_from_Ab_lambda
 *    (src/utils.jl:1222-1267): Q = A_k' A_k, c_k = -A_k' b_k, no
 *    constraints (m = 0), lambda_k;
 *  - QAP relaxations as built by build_from_ABST (src/utils.jl:1133-1180):
 *    x = vec(X_k), doubly-stochastic rows, X_k >= 0,
 *    Q_k(X) = 2 (A_k X B_k - S_k X - X T_k), instances of uneven size.
 * The instances are concatenated block-diagonally and each HPR pass is one
 * kernel over all of them; converged instances drop out through a
 * per-instance mask.  Each instance follows the reference's control logic
 * on its own (restarts, sigma, stopping), so its result is the one
 * hprqp_solve would return up to rounding.  No counterpart in the reference
 * (which solves one model per call).
 */
#ifndef HPRQP_BATCH_H
#define HPRQP_BATCH_H

#include <stdint.h>

#include "hprqp.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct hprqp_batch* hprqp_batch_handle;

int hprqp_batch_create(hprqp_batch_handle* h, int32_t device);

/* Copy `count` LASSO problems (Q_kind = HPRQP_Q_LASSO, m = 0). */
int hprqp_batch_load_lasso(hprqp_batch_handle h, int32_t count, const hprqp_problem* problems);

/* Copy `count` QAP relaxations (Q_kind = HPRQP_Q_QAP, m = 2 qap_n); replaces
 * whatever the handle held.  hprqp_batch_solve then solves this family. */
int hprqp_batch_load_qap(hprqp_batch_handle h, int32_t count, const hprqp_problem* problems);

/* Solve all instances.  initial_x: NULL or `count` pointers (entries may be
 * NULL) to length-n_k warm starts; sigma0: NULL or `count` initial sigmas
 * (<= 0: the parameter rule).  results: `count` records; x_out: NULL or
 * `count` pointers to length-n_k outputs (entries may be NULL).  params has
 * the meaning of hprqp_solve's, including precision (FP32 + FP64 polish
 * switches per instance). */
int hprqp_batch_solve(hprqp_batch_handle h, const hprqp_params* params, const double* const* initial_x,
                      const double* sigma0, hprqp_result* results, double* const* x_out);

/* Test and measurement hook (no reference counterpart): Y = Q_k(X_k) for
 * every instance of the loaded QAP family (Qmap!, src/Q_operators/
 * QAP_operator.jl:52-75), X and Y concatenated in instance order (sum of
 * n_k^2 values, each block column-major), computed by the batch engine of
 * `precision`: HPRQP_PRECISION_FP64 runs the CUDA-core FP64 GEMMs,
 * HPRQP_PRECISION_FP32_POLISH the FP32 phase's operator (the fused 3xTF32
 * tensor-core kernel when every n_k <= 128).  *tensor_cores (may be NULL)
 * tells which ran. */
int hprqp_batch_qap_apply(hprqp_batch_handle h, int32_t precision, const double* X, double* Y,
                          int32_t* tensor_cores);

const char* hprqp_batch_last_error(hprqp_batch_handle h);
int hprqp_batch_destroy(hprqp_batch_handle h);

#ifdef __cplusplus
}
#endif
#endif /* HPRQP_BATCH_H */
