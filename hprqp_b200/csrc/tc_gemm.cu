// tc_gemm.cu — 3xTF32 split-precision GEMM on the sm_100a tensor cores
// (tcgen05.mma kind::tf32, accumulator in TMEM), for the dense products of
// the QAP operator (src/Q_operators/QAP_operator.jl:52-61) in the FP32
// phase:  C = alpha * A * B + beta * C, all N x N column-major FP32.
//
// Each operand value a is split as a = hi + lo with hi = tf32(a) and
// lo = tf32(a - hi); A*B is accumulated as Alo*Bhi + Ahi*Blo + Ahi*Bhi in
// FP32, which recovers FP32-level accuracy from TF32 tensor-core products
// (the Alo*Blo term is below FP32 resolution).
//
// Two kernels.  k_split_img writes each operand once as TF32 hi/lo
// "images": for every 128-row block and 32-k chunk, 16 KiB of hi followed by
// 16 KiB of lo, each already in the canonical K-major no-swizzle layout of
// the UMMA descriptors (8-row x 16-byte core matrices).  k_gemm_tc then
// computes one 128 x 128 tile of C per CTA: one thread runs a 3-stage ring
// of shared-memory buffers, filling each with two 32 KiB bulk copies
// (cp.async.bulk, completion counted on the stage's "full" mbarrier),
// issuing 4 k-steps x 3 MMAs (M = N = 128, K = 8) per chunk, committing them
// to the stage's "empty" mbarrier and refilling a stage as soon as its MMAs
// have completed, so the copies of later chunks run under the MMAs of
// earlier ones.  The epilogue reads the tile from TMEM (warp w owns lanes
// 32w..32w+31, i.e. rows of C) and writes alpha * acc + beta * C.
//
// Every mbarrier wait is bounded; on a timeout the kernel raises the
// device flag g_tc_err, drains what it issued (bounded), frees its TMEM and
// returns; gemm_3xtf32_failed() reads and clears the flag.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <mutex>

#include "pool.h"
#include "common.cuh"
#include "tc_gemm.h"
#include "tcgen05.cuh"

namespace hprqp {
namespace tc {

__device__ int g_tc_err = 0;


constexpr int kStages = 3;
constexpr int kImgFloats = 2 * kTile * kChunk;        // hi + lo of one (block, chunk): 8192 floats
constexpr int kStageBytes = 2 * kImgFloats * 4;       // A image + B image: 64 KiB
constexpr int kSmemPipe = kStages * kStageBytes + 1024;

// image of an N x N operand: rows = the M (A) or N (B) index, k contiguous
// within 4-element core-matrix rows.  trans = 0: element (row, k) = M[row +
// k N] (A, column-major); trans = 1: element (row, k) = M[k + row N] (B).
__global__ void __launch_bounds__(256) k_split_img(int N, int nkc, const float* __restrict__ M, int trans,
                                                   float* __restrict__ img) {
  const int rows_p = ((N + kTile - 1) / kTile) * kTile, k_p = nkc * kChunk;
  const int64_t t = (int64_t)blockIdx.x * 256 + threadIdx.x;
  if (t >= (int64_t)rows_p * k_p) return;
  int row, k;
  if (trans) {  // consecutive threads: consecutive k (contiguous in B)
    k = (int)(t % k_p);
    row = (int)(t / k_p);
  } else {  // consecutive threads: consecutive rows (contiguous in A)
    row = (int)(t % rows_p);
    k = (int)(t / rows_p);
  }
  const float a = (row < N && k < N) ? (trans ? M[k + (int64_t)row * N] : M[row + (int64_t)k * N]) : 0.0f;
  const uint32_t h = to_tf32(a);
  const uint32_t l = to_tf32(a - __uint_as_float(h));
  const int64_t base = ((int64_t)(row / kTile) * nkc + k / kChunk) * kImgFloats;
  const uint32_t off = kmaj_off(row % kTile, k % kChunk) / 4;
  img[base + off] = __uint_as_float(h);
  img[base + kTile * kChunk + off] = __uint_as_float(l);
}

__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__global__ void __launch_bounds__(kThreads) k_gemm_tc(int N, int nkc, float alpha, const float* __restrict__ Aimg,
                                                      const float* __restrict__ Bimg, float beta, float* C) {
  extern __shared__ unsigned char smem_raw[];
  __shared__ __align__(8) uint64_t full[kStages], empty[kStages], done;
  __shared__ uint32_t tmem_base;
  __shared__ int s_fail;
  unsigned char* sm = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  const int tid = threadIdx.x, warp = tid >> 5;
  const int bi = blockIdx.x, bj = blockIdx.y;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                 "r"((uint32_t)kTile));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    for (int q = 0; q < kStages; ++q) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&full[q])), "r"(1u));
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&empty[q])), "r"(1u));
    }
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&done)), "r"(1u));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    s_fail = 0;
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tm = tmem_base;
  if (tid == 0) {
    const float* arow = Aimg + (int64_t)bi * nkc * kImgFloats;
    const float* brow = Bimg + (int64_t)bj * nkc * kImgFloats;
    auto stage_a = [&](int q) { return smem_u32(sm + q * kStageBytes); };
    auto stage_b = [&](int q) { return smem_u32(sm + q * kStageBytes + kStageBytes / 2); };
    auto issue = [&](int q, int kc) {
      expect_tx(&full[q], kStageBytes);
      bulk_g2s(stage_a(q), arow + (int64_t)kc * kImgFloats, kStageBytes / 2, &full[q]);
      bulk_g2s(stage_b(q), brow + (int64_t)kc * kImgFloats, kStageBytes / 2, &full[q]);
    };
    uint32_t fuse[kStages] = {0, 0, 0}, euse[kStages] = {0, 0, 0}, issued[kStages] = {0, 0, 0};
    for (int q = 0; q < kStages && q < nkc; ++q) {
      issue(q, q);
      ++issued[q];
    }
    bool ok = true;
    for (int kc = 0; kc < nkc && ok; ++kc) {
      const int q = kc % kStages;
      if (!mbar_wait(&full[q], fuse[q] & 1u)) { ok = false; break; }
      ++fuse[q];
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t a = stage_a(q), b = stage_b(q);
      mma_chunk_3x(tm, a, a + kOpBytes, b, b + kOpBytes, kc == 0);
      mma_commit(&empty[q]);
      // refill the stage of the previous chunk once its MMAs have completed
      const int pk = kc - 1;
      if (pk >= 0 && pk + kStages < nkc) {
        const int pq = pk % kStages;
        if (!mbar_wait(&empty[pq], euse[pq] & 1u)) { ok = false; break; }
        ++euse[pq];
        issue(pq, pk + kStages);
        ++issued[pq];
      }
    }
    mma_commit(&done);  // completes when every MMA issued above has
    if (!mbar_wait(&done, 0) || !ok) {
      s_fail = 1;
      for (int q = 0; q < kStages; ++q)  // let copies still in flight land (bounded)
        while (fuse[q] < issued[q] && mbar_wait(&full[q], fuse[q] & 1u)) ++fuse[q];
    }
  }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (!s_fail) {
    const int row = bi * kTile + warp * 32 + (tid & 31);
    const uint32_t lane_base = tm + ((uint32_t)(warp * 32) << 16);
#pragma unroll 1
    for (int c0 = 0; c0 < kTile; c0 += 32) {
      uint32_t v[32];
      tmem_ld32(lane_base + (uint32_t)c0, v);
      if (row < N) {
#pragma unroll
        for (int q = 0; q < 32; ++q) {
          const int col = bj * kTile + c0 + q;
          if (col < N) {
            float* p = C + (size_t)col * N + row;
            const float acc = __uint_as_float(v[q]);
            *p = beta == 0.0f ? alpha * acc : fmaf(alpha, acc, beta * *p);
          }
        }
      }
    }
  } else if (tid == 0) {
    atomicExch(&g_tc_err, 1);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tm), "r"((uint32_t)kTile));
  }
}

}  // namespace tc

int64_t gemm_3xtf32_ws_floats(int N) {
  const int64_t nb = (N + tc::kTile - 1) / tc::kTile, nkc = (N + tc::kChunk - 1) / tc::kChunk;
  return 2 * nb * nkc * tc::kImgFloats;  // A and B images
}

void gemm_3xtf32_ws(int N, float alpha, const float* A, const float* B, float beta, float* C, float* ws,
                    cudaStream_t st) {
  static std::mutex mu;
  static bool ready[64] = {};
  int dev = 0;
  HPRQP_CUDA(cudaGetDevice(&dev));
  {
    std::lock_guard<std::mutex> lk(mu);
    if (dev < 0 || dev >= 64) throw Error(-2, "device ordinal out of range");
    if (!ready[dev]) {
      HPRQP_CUDA(cudaFuncSetAttribute(tc::k_gemm_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, tc::kSmemPipe));
      ready[dev] = true;
    }
  }
  if (N <= 0) return;
  const int nb = (N + tc::kTile - 1) / tc::kTile, nkc = (N + tc::kChunk - 1) / tc::kChunk;
  float* aimg = ws;
  float* bimg = ws + (int64_t)nb * nkc * tc::kImgFloats;
  const int64_t elems = (int64_t)nb * tc::kTile * nkc * tc::kChunk;
  const int g = (int)((elems + 255) / 256);
  tc::k_split_img<<<g, 256, 0, st>>>(N, nkc, A, 0, aimg);
  tc::k_split_img<<<g, 256, 0, st>>>(N, nkc, B, 1, bimg);
  tc::k_gemm_tc<<<dim3(nb, nb), tc::kThreads, tc::kSmemPipe, st>>>(N, nkc, alpha, aimg, bimg, beta, C);
  HPRQP_LAUNCH_CHECK();
}


bool gemm_3xtf32_failed(cudaStream_t st) {
  int v = 0;
  const int zero = 0;
  HPRQP_CUDA(cudaMemcpyFromSymbolAsync(&v, tc::g_tc_err, sizeof(int), 0, cudaMemcpyDeviceToHost, st));
  HPRQP_CUDA(cudaStreamSynchronize(st));
  if (v) {
    HPRQP_CUDA(cudaMemcpyToSymbolAsync(tc::g_tc_err, &zero, sizeof(int), 0, cudaMemcpyHostToDevice, st));
    HPRQP_CUDA(cudaStreamSynchronize(st));
  }
  return v != 0;
}

}  // namespace hprqp

// ---------------------------------------------------------------------------
// C ABI (include/hprqp.h)
// ---------------------------------------------------------------------------
extern "C" int64_t hprqp_gemm_3xtf32_ws_floats(int32_t n) { return n > 0 ? hprqp::gemm_3xtf32_ws_floats(n) : 0; }

extern "C" int hprqp_gemm_3xtf32_ws(int32_t n, float alpha, const float* A, const float* B, float beta, float* C,
                                    float* ws, void* stream) {
  try {
    if (n < 0 || (n > 0 && (!A || !B || !C || !ws))) return -1;
    const cudaStream_t st = (cudaStream_t)stream;
    hprqp::gemm_3xtf32_ws(n, alpha, A, B, beta, C, ws, st);
    return 0;
  } catch (const hprqp::Error& e) {
    std::fprintf(stderr, "hprqp_gemm_3xtf32_ws: %s\n", e.what());
    return e.code;
  } catch (...) {
    return -2;
  }
}

extern "C" int hprqp_gemm_3xtf32(int32_t n, float alpha, const float* A, const float* B, float beta, float* C,
                                 void* stream) {
  try {
    if (n < 0 || (n > 0 && (!A || !B || !C))) return -1;
    const cudaStream_t st = (cudaStream_t)stream;
    const int64_t wf = hprqp::gemm_3xtf32_ws_floats(n);
    hprqp::PoolBlocks tmp;  // the TF32 operand images, returned to the pool on exit
    float* ws = (float*)tmp.get(sizeof(float) * (size_t)std::max<int64_t>(wf, 1));
    hprqp::gemm_3xtf32_ws(n, alpha, A, B, beta, C, ws, st);
    const bool failed = hprqp::gemm_3xtf32_failed(st);  // synchronises the stream
    return failed ? -2 : 0;
  } catch (const hprqp::Error& e) {
    std::fprintf(stderr, "hprqp_gemm_3xtf32: %s\n", e.what());
    return e.code;
  } catch (...) {
    return -2;
  }
}
