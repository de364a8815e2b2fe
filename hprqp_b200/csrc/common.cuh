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
constexpr int kStageSmem = 200 * 1024;     // its shared-memory budget for one column block
constexpr int kStageSlots = 2048;          // and the row-sum slots of one tile (FP64 at most: 16 KiB)

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
  // Column-blocked staged schedule (k_stage_pass), for products whose input
  // gathers dominate: the columns are cut into st_nblk blocks of st_bw
  // columns, each small enough for one CTA's shared memory.  Block b's part
  // of every row is a run of 8-entry chunks (zero-padded, at least one per
  // row) holding 16-bit block-local columns and the values; chunk offsets
  // st_cptr[b * (rows + 1) + r].  Tiles {first warp tile, chunks, first row,
  // end row} are runs of whole rows with at most kStageSlots row-sum slots,
  // starting at a whole warp tile (32 chunks; the values of a warp tile are
  // stored lane-interleaved in 16-byte slices); each warp tile has a
  // descriptor {first slot, segment-head mask}, and a row has one slot per
  // warp tile it touches (first slot st_srow[b * (rows + 1) + r]).  CTA i
  // of the one-wave grid takes block st_item[i].x and tiles [st_item[i].y,
  // st_item[i].z).  With several blocks a row's block sums go to
  // st_part[b * rows + r] and the last block to arrive (counter st_cnt[r])
  // folds them in block order.
  bool stage = false;
  int st_nblk = 0, st_bw = 0, st_grid = 0, st_ntile = 0;
  int64_t st_chunks = 0, st_nwt = 0;
  const int* st_cptr = nullptr;
  const int* st_srow = nullptr;
  const uint16_t* st_col = nullptr;
  const V* st_val = nullptr;
  const int2* st_wt = nullptr;
  const int4* st_tile = nullptr;
  const int4* st_item = nullptr;
  double* st_part = nullptr;
  unsigned* st_cnt = nullptr;
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
