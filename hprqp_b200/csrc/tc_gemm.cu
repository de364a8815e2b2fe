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
// One CTA computes one 128 x 128 tile of C.  K is walked in chunks of 32:
// the 128 threads load the A and B chunk from global memory, split it, and
// store it into shared memory in the canonical K-major no-swizzle layout of
// the UMMA descriptors (8-row x 16-byte core matrices); one thread issues
// 4 k-steps x 3 MMAs (M = 128, N = 128, K = 8) and commits them to an
// mbarrier that the CTA waits on before reusing the buffers.  The epilogue
// reads the accumulator tile from TMEM (warp w owns lanes 32w..32w+31, i.e.
// rows of C) and writes alpha * acc + beta * C.
//
// Every mbarrier wait is bounded; on a timeout the kernel raises the
// device flag g_tc_err, skips the rest of its work, frees its TMEM and
// returns; gemm_3xtf32_failed() reads and clears the flag.
#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>

#include "common.cuh"
#include "tc_gemm.h"
#include "tcgen05.cuh"

namespace hprqp {
namespace tc {

constexpr int kSmemBytes = 4 * kOpBytes + 1024;   // A hi/lo, B hi/lo, + alignment slack

__device__ int g_tc_err = 0;

__global__ void __launch_bounds__(kThreads) k_gemm_3xtf32(int N, float alpha, const float* __restrict__ A,
                                                           const float* __restrict__ B, float beta, float* C) {
  extern __shared__ unsigned char smem_raw[];
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint32_t tmem_base;
  __shared__ int s_fail;
  unsigned char* sm = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  unsigned char* sAh = sm;
  unsigned char* sAl = sm + kOpBytes;
  unsigned char* sBh = sm + 2 * kOpBytes;
  unsigned char* sBl = sm + 3 * kOpBytes;
  const int tid = threadIdx.x, warp = tid >> 5;
  const int i0 = blockIdx.x * kTile, j0 = blockIdx.y * kTile;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                 "r"((uint32_t)kTile));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&bar)), "r"(1u));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    s_fail = 0;
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tm = tmem_base;

  uint32_t parity = 0;
  bool first = true;
  for (int k0 = 0; k0 < N; k0 += kChunk) {
    // stage A[i0 + r, k0 + k] and B[k0 + k, j0 + c] (zero outside the matrix)
    // A is column-major: consecutive threads take consecutive rows, 4 k each
    for (int e = tid; e < kTile * kChunk / 4; e += kThreads) {
      const int r = e & (kTile - 1), k = (e >> 7) * 4;
      const int gi = i0 + r, gk = k0 + k;
      float a[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) a[q] = (gi < N && gk + q < N) ? __ldg(A + (size_t)(gk + q) * N + gi) : 0.0f;
      put_split4(sAh, sAl, kmaj_off(r, k), a[0], a[1], a[2], a[3]);
    }
    // B[k, j] with k contiguous in memory: 4 consecutive k of one column each
    for (int e = tid; e < kTile * kChunk / 4; e += kThreads) {
      const int k = (e & (kChunk / 4 - 1)) * 4, c = e >> 3;
      const int gk = k0 + k, gj = j0 + c;
      float b[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) b[q] = (gk + q < N && gj < N) ? __ldg(B + (size_t)gj * N + gk + q) : 0.0f;
      put_split4(sBh, sBl, kmaj_off(c, k), b[0], b[1], b[2], b[3]);
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t ah = smem_u32(sAh), al = smem_u32(sAl), bh = smem_u32(sBh), bl = smem_u32(sBl);
#pragma unroll
      for (int s = 0; s < kChunk / 8; ++s) {
        const uint32_t o = (uint32_t)s * 2 * kLbo;  // K = 8 per MMA = two core matrices along K
        mma_tf32(tm, smem_desc(al + o), smem_desc(bh + o), first ? 0u : 1u);
        mma_tf32(tm, smem_desc(ah + o), smem_desc(bl + o), 1u);
        mma_tf32(tm, smem_desc(ah + o), smem_desc(bh + o), 1u);
        first = false;
      }
      mma_commit(&bar);
    }
    first = false;
    if (!mbar_wait(&bar, parity)) s_fail = 1;
    parity ^= 1u;
    __syncthreads();
    if (s_fail) break;
  }
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (!s_fail) {
    // epilogue: thread t of warp w holds row i0 + 32w + lane
    const int row = i0 + warp * 32 + (tid & 31);
    const uint32_t lane_base = tm + ((uint32_t)(warp * 32) << 16);
#pragma unroll 1
    for (int c0 = 0; c0 < kTile; c0 += 16) {
      uint32_t v[16];
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
          "%14, %15}, [%16];"
          : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
            "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
          : "r"(lane_base + (uint32_t)c0));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (row < N) {
#pragma unroll
        for (int q = 0; q < 16; ++q) {
          const int col = j0 + c0 + q;
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
    mbar_wait(&bar, parity ^ 1u);  // give MMAs still in flight a bounded chance to drain
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tm), "r"((uint32_t)kTile));
  }
}

}  // namespace tc

void gemm_3xtf32(int N, float alpha, const float* A, const float* B, float beta, float* C, cudaStream_t st) {
  // the dynamic shared memory limit is a per-device function attribute
  static std::mutex mu;
  static bool ready[64] = {};
  int dev = 0;
  HPRQP_CUDA(cudaGetDevice(&dev));
  {
    std::lock_guard<std::mutex> lk(mu);
    if (dev < 0 || dev >= 64) throw Error(-2, "device ordinal out of range");
    if (!ready[dev]) {
      HPRQP_CUDA(cudaFuncSetAttribute(tc::k_gemm_3xtf32, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      tc::kSmemBytes));
      ready[dev] = true;
    }
  }
  if (N <= 0) return;
  const int t = (N + tc::kTile - 1) / tc::kTile;
  tc::k_gemm_3xtf32<<<dim3(t, t), tc::kThreads, tc::kSmemBytes, st>>>(N, alpha, A, B, beta, C);
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
extern "C" int hprqp_gemm_3xtf32(int32_t n, float alpha, const float* A, const float* B, float beta, float* C,
                                 void* stream) {
  try {
    if (n < 0 || (n > 0 && (!A || !B || !C))) return -1;
    const cudaStream_t st = (cudaStream_t)stream;
    hprqp::gemm_3xtf32(n, alpha, A, B, beta, C, st);
    if (hprqp::gemm_3xtf32_failed(st)) return -2;
    return 0;
  } catch (const hprqp::Error& e) {
    std::fprintf(stderr, "hprqp_gemm_3xtf32: %s\n", e.what());
    return e.code;
  } catch (...) {
    return -2;
  }
}
