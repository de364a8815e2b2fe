// batch_qp.h — batched HPR solves of QAP relaxations (batch_qp.cu), driven
// by the hprqp_batch_* entry points (batch.cu).
#pragma once

#include <cuda_runtime.h>

#include "../../include/hprqp.h"

namespace hprqp {
namespace bqp {

struct QpBatch;  // family + engines, opaque to batch.cu

QpBatch* create(cudaStream_t st);
void destroy(QpBatch* q);
// Every problem must be a QAP relaxation (Q_kind QAP, m > 0), as
// build_from_ABST makes it.
void load(QpBatch* q, int count, const hprqp_problem* problems);
int count(const QpBatch* q);
void solve(QpBatch* q, const hprqp_params& p, const double* const* x0s, const double* sig0, hprqp_result* res,
           double* const* xs);
// Y = Q_k(X_k) for every instance (X, Y concatenated, sum n_k^2 values) in
// the engine of `precision`; returns 1 when the FP32 engine ran the fused
// tensor-core operator, 0 for the CUDA-core GEMMs.
int apply_q(QpBatch* q, int precision, const double* X, double* Y);

}  // namespace bqp
}  // namespace hprqp
