// common.cuh — shared device helpers for the HPR-QP iteration engine.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cmath>
#include <cstdio>
#include <stdexcept>
#include <string>

namespace hprqp {

// Error carrying an ABI return code; caught at the C boundary.
struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define HPRQP_CUDA(call)                                                                  \
  do {                                                                                    \
    cudaError_t e_ = (call);                                                              \
    if (e_ != cudaSuccess)                                                                \
      throw ::hprqp::Error(e_ == cudaErrorMemoryAllocation ? -3 : -2,                     \
                           std::string(#call) + ": " + cudaGetErrorString(e_) + " (" +   \
                               __FILE__ + ":" + std::to_string(__LINE__) + ")");         \
  } while (0)

#define HPRQP_LAUNCH_CHECK() HPRQP_CUDA(cudaGetLastError())

#ifdef __CUDACC__
constexpr int kBlock = 256;  // threads per CTA for every row/element kernel

// Device view of a sparse matrix: CSR (0-based, int32 indices), plus
// optional ELL and SELL-32 copies (slices of 32 consecutive rows stored column-major,
// entry k of row r at sptr[r/32] + 32k + r%32) used when the row-schedule
// autotuner finds it faster.  Row lengths come from the CSR ptr, so the
// padding of a slice is never read.
template <typename V>
struct DCsr {
  int rows = 0, cols = 0;
  int64_t nnz = 0;
  const int* ptr = nullptr;
  const int* col = nullptr;
  const V* val = nullptr;
  int tpr = 4;  // threads cooperating on one row (1,2,4,8,16,32)
  bool sell = false;
  const int* sptr = nullptr;
  const int* scol = nullptr;
  const V* sval = nullptr;
  int64_t sell_len = 0;
  // ELL copy for short, even rows: width ell_w, entry k of row r at
  // k * rows + r (column-major), padding = (column 0, value 0), so a row's
  // product needs neither row pointers nor lengths
  bool ell = false;
  int ell_w = 0;
  const int* ecol = nullptr;
  const V* evalv = nullptr;
  // Row-split schedule for a heavy tail of long rows: `npieces` pieces
  // {row, begin, end, split index or -1}, heaviest first, one warp each; a
  // row longer than split_T is cut into pieces of split_T entries whose
  // partial sums go to spart[srow[s].x + j] (j = piece index in the row) and
  // are folded in order by the row's last piece (counter scnt[s])
  bool split = false;
  int npieces = 0, split_T = 0;
  const int4* pieces = nullptr;
  const int2* srow = nullptr;
  double* spart = nullptr;
  unsigned* scnt = nullptr;
};

// Programmatic dependent launch: wait until the previous kernel in the
// stream has completed and flushed, then let the next kernel start its CTAs
// (they wait in turn), so kernel boundaries overlap launch and tail.
__device__ __forceinline__ void pdl_enter() {
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 900
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
#endif
}

// Reduce `v` over the TPR lanes of a row group (lanes of a group are
// consecutive and the group is aligned inside its warp).
template <int TPR, typename T>
__device__ __forceinline__ T group_sum(T v) {
  if constexpr (TPR > 1) {
    const unsigned lane = threadIdx.x & 31u;
    const unsigned mask = (TPR == 32) ? 0xffffffffu
                                      : (((1u << TPR) - 1u) << (lane & ~(unsigned)(TPR - 1)));
#pragma unroll
    for (int off = TPR / 2; off > 0; off >>= 1) v += __shfl_xor_sync(mask, v, off, TPR);
  }
  return v;
}

#endif  // __CUDACC__

}  // namespace hprqp
