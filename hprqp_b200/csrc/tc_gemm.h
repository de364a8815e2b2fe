// tc_gemm.h — 3xTF32 tensor-core GEMM (tc_gemm.cu) for the QAP operator.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace hprqp {

// C = alpha * A * B + beta * C, N x N column-major FP32, on `st`: the
// operands are pre-split into TF32 hi/lo images in `ws`
// (gemm_3xtf32_ws_floats(N) floats, caller-owned), then bulk-copied tiles.
int64_t gemm_3xtf32_ws_floats(int N);
void gemm_3xtf32_ws(int N, float alpha, const float* A, const float* B, float beta, float* C, float* ws,
                    cudaStream_t st);

// True (and the flag cleared) when a launch since the last call gave up a
// bounded wait; synchronises `st`.
bool gemm_3xtf32_failed(cudaStream_t st);

}  // namespace hprqp
