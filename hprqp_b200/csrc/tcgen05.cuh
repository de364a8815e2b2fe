// tcgen05.cuh — sm_100a tensor-core building blocks shared by the 3xTF32
// kernels (tc_gemm.cu, batch_qp.cu): TF32 split, the canonical K-major
// no-swizzle shared-memory layout of a 128-row x 32-k operand chunk and its
// UMMA descriptor, the kind::tf32 MMA (M = N = 128, K = 8), commit to an
// mbarrier, and a bounded mbarrier wait.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace hprqp {
namespace tc {

constexpr int kTile = 128;   // M and N of one MMA tile
constexpr int kChunk = 32;   // K elements staged per round
constexpr int kThreads = 128;
constexpr int kOpBytes = kTile * kChunk * 4;  // one split half of one operand chunk: 16 KiB
constexpr unsigned long long kWaitNs = 1000000000ull;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ uint32_t to_tf32(float a) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(a));
  return r;
}

// byte offset of element (row r, k) in a K-major no-swizzle chunk of 128 rows
// x 32 k: core matrix (k/4, r/8) of 8 rows x 16 bytes; K-adjacent core
// matrices are kLbo apart, row-group-adjacent ones 128 bytes apart.
constexpr uint32_t kSbo = 128;
constexpr uint32_t kLbo = (kTile / 8) * 128;  // 2048
__device__ __forceinline__ uint32_t kmaj_off(int r, int k) {
  return (uint32_t)((k >> 2) * kLbo + (r >> 3) * kSbo + (r & 7) * 16 + (k & 3) * 4);
}

__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFF);
  d |= (uint64_t)((kLbo >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((kSbo >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version (sm_100)
  // base offset 0, LBO mode 0, layout type 0 (no swizzle)
  return d;
}

// kind::tf32, D = F32, A = B = TF32, both K-major, M = 128, N = 128
constexpr uint32_t kIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(kTile >> 3) << 17) |
                            ((uint32_t)(kTile >> 4) << 24);

__device__ __forceinline__ void mma_tf32(uint32_t dtm, uint64_t ad, uint64_t bd, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(dtm),
      "l"(ad), "l"(bd), "r"(kIdesc), "r"(accumulate));
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  const uint32_t a = smem_u32(bar);
  unsigned long long t0 = 0;
  for (uint32_t it = 0;; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred P1;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    if (it == 0) t0 = t;
    else if (t - t0 > kWaitNs || it > (1u << 26)) return false;
  }
}


// split a = hi + lo (both TF32) and store them at byte offset `off` of the
// hi and lo chunks
__device__ __forceinline__ void put_split(unsigned char* hi, unsigned char* lo, uint32_t off, float a) {
  const uint32_t h = to_tf32(a);
  *(uint32_t*)(hi + off) = h;
  *(uint32_t*)(lo + off) = to_tf32(a - __uint_as_float(h));
}

// the same for 4 consecutive k of one row (off 16-byte aligned): one
// 16-byte store per half, so a warp writing 32 consecutive rows fills 512
// contiguous bytes without bank conflicts
__device__ __forceinline__ void put_split4(unsigned char* hi, unsigned char* lo, uint32_t off, float a0, float a1,
                                           float a2, float a3) {
  uint4 h, l;
  h.x = to_tf32(a0);
  h.y = to_tf32(a1);
  h.z = to_tf32(a2);
  h.w = to_tf32(a3);
  l.x = to_tf32(a0 - __uint_as_float(h.x));
  l.y = to_tf32(a1 - __uint_as_float(h.y));
  l.z = to_tf32(a2 - __uint_as_float(h.z));
  l.w = to_tf32(a3 - __uint_as_float(h.w));
  *(uint4*)(hi + off) = h;
  *(uint4*)(lo + off) = l;
}

// 3xTF32 product of one staged K chunk into the accumulator at TMEM column
// `dtm`: D (+)= Alo*Bhi + Ahi*Blo + Ahi*Bhi for the chunk's 4 k-steps.
// `first` starts the accumulation (D = ...) with the chunk's first MMA.
__device__ __forceinline__ void mma_chunk_3x(uint32_t dtm, uint32_t ah, uint32_t al, uint32_t bh, uint32_t bl,
                                             bool first) {
#pragma unroll
  for (int s = 0; s < kChunk / 8; ++s) {
    const uint32_t o = (uint32_t)s * 2 * kLbo;  // K = 8 per MMA = two core matrices along K
    mma_tf32(dtm, smem_desc(al + o), smem_desc(bh + o), (first && s == 0) ? 0u : 1u);
    mma_tf32(dtm, smem_desc(ah + o), smem_desc(bl + o), 1u);
    mma_tf32(dtm, smem_desc(ah + o), smem_desc(bh + o), 1u);
  }
}

// 16 consecutive accumulator columns of this thread's TMEM lane
__device__ __forceinline__ void tmem_ld16(uint32_t addr, uint32_t (&v)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
        "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
      : "r"(addr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// 32 consecutive accumulator columns of this thread's TMEM lane
__device__ __forceinline__ void tmem_ld32(uint32_t addr, uint32_t (&v)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
        "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
        "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
        "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
      : "r"(addr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

}  // namespace tc
}  // namespace hprqp
