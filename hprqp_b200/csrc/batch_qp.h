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

}  // namespace bqp
}  // namespace hprqp
