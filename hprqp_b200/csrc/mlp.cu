// mlp.cu — the warm-start network: a 3-layer MLP (ReLU) with BF16 weights
// and activations, FP32 accumulation, FP32 master weights and Adam, with
// hand-written forward, backward and update kernels.
//
// It maps instance features of a problem family to a proposed solution and
// log sigma; the HPR engine then starts from that proposal and certifies the
// result itself, so a poor proposal costs iterations, never correctness.
//
// Layout: every matrix is row-major with leading dimensions padded to
// multiples of 64 (zero padding stays zero: padded inputs are zero, padded
// weight rows/columns start at zero and receive zero gradient).  Products
// run on the tcgen05 tensor cores (kind::f16, BF16 operands, FP32
// accumulators in TMEM), one 128 x 128 output tile per CTA.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "pool.h"
#include "../../include/hprqp.h"
#include "../../include/hprqp_mlp.h"
#include "common.cuh"
#include "tcgen05.cuh"

namespace hprqp {
namespace mlp {

using bf16 = __nv_bfloat16;

constexpr int kTile = 64;
inline int64_t pad64(int64_t v) { return (v + 63) / 64 * 64; }

// C[M x N] = opA(A) opB(B), FP32 out, on the tcgen05 tensor cores
// (kind::f16 with BF16 operands, FP32 accumulator in TMEM).  TA: A is
// stored K x M (row-major), i.e. used transposed; TB: B is stored N x K
// (row-major) and used transposed.  M, N, K are multiples of 64; lda, ldb,
// ldc are row strides (multiples of 64).  One CTA of 128 threads computes a
// 128 x 128 tile of C: per 64-wide K chunk the threads stage both operands
// in the canonical K-major no-swizzle layout (8-row x 16-byte core
// matrices: 8 BF16 of one row per 16 bytes; K-adjacent core matrices 2 KiB
// apart, row-adjacent ones 128 bytes), one thread issues the chunk's four
// MMAs (M = N = 128, K = 16) and commits them to an mbarrier, and the
// epilogue reads the accumulator rows from TMEM (warp w: lanes 32w..).
// Rows and columns of the tile beyond M or N are staged as zeros and not
// stored.  Every mbarrier wait is bounded; on a timeout the CTA raises
// g_mlp_tc_err, frees its TMEM and returns.
__device__ int g_mlp_tc_err = 0;
constexpr int kTcK = 64;                          // K elements per staged chunk
constexpr int kTcOpBytes = tc::kTile * kTcK * 2;  // one operand chunk: 16 KiB
constexpr int kTcSmem = 2 * kTcOpBytes + 1024;
// kind::f16: D = F32, A = B = BF16 (the same type on both sides), K-major, M = N = 128
constexpr uint32_t kIdescBf16 = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(tc::kTile >> 3) << 17) |
                                ((uint32_t)(tc::kTile >> 4) << 24);

__device__ __forceinline__ uint32_t kmaj16_off(int r, int k) {  // element (r, k) of a 128 x 64 chunk
  return (uint32_t)((k >> 3) * tc::kLbo + (r >> 3) * tc::kSbo + (r & 7) * 16 + (k & 7) * 2);
}

__device__ __forceinline__ void mma_bf16(uint32_t dtm, uint64_t ad, uint64_t bd, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(dtm),
      "l"(ad), "l"(bd), "r"(kIdescBf16), "r"(accumulate));
}

// 8 consecutive K elements of row `r` of an operand: contiguous (one 16-byte
// load) when the operand is stored K-contiguous, else gathered with stride ld
__device__ __forceinline__ uint4 load8(const bf16* base, bool kcontig, int64_t ld) {
  if (kcontig) return *reinterpret_cast<const uint4*>(base);
  uint4 v;
  uint16_t* h = reinterpret_cast<uint16_t*>(&v);
#pragma unroll
  for (int q = 0; q < 8; ++q) h[q] = *reinterpret_cast<const uint16_t*>(base + q * ld);
  return v;
}

template <bool TA, bool TB>
__global__ void __launch_bounds__(tc::kThreads) k_gemm(int M, int N, int K, const bf16* __restrict__ A, int lda,
                                                       const bf16* __restrict__ B, int ldb, float* __restrict__ C,
                                                       int ldc) {
  extern __shared__ unsigned char smem_raw[];
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint32_t tmem_base;
  __shared__ int s_fail;
  unsigned char* sm = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  unsigned char *sA = sm, *sB = sm + kTcOpBytes;
  const int tid = threadIdx.x, warp = tid >> 5;
  const int m0 = blockIdx.y * tc::kTile, n0 = blockIdx.x * tc::kTile;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tc::smem_u32(&tmem_base)),
                 "r"(128u));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(tc::smem_u32(&bar)), "r"(1u));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    s_fail = 0;
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t acc = tmem_base;
  uint32_t parity = 0;
  for (int k0 = 0; k0 < K; k0 += kTcK) {
    // 128 rows x 8 groups of 8 K elements per operand: 8 pairs per thread
    for (int e = tid; e < tc::kTile * (kTcK / 8); e += tc::kThreads) {
      const int r = e & (tc::kTile - 1), g = e >> 7;
      const int k = k0 + 8 * g;
      const int m = m0 + r, n = n0 + r;
      const uint4 z = make_uint4(0u, 0u, 0u, 0u);
      // opA(m, k): TA ? A[k][m] : A[m][k];  opB(k, n) as the N x K operand: TB ? B[n][k] : B[k][n]
      const uint4 av = m < M ? (TA ? load8(A + (int64_t)k * lda + m, false, lda) : load8(A + (int64_t)m * lda + k, true, 1))
                             : z;
      const uint4 bv = n < N ? (TB ? load8(B + (int64_t)n * ldb + k, true, 1) : load8(B + (int64_t)k * ldb + n, false, ldb))
                             : z;
      *reinterpret_cast<uint4*>(sA + kmaj16_off(r, 8 * g)) = av;
      *reinterpret_cast<uint4*>(sB + kmaj16_off(r, 8 * g)) = bv;
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
      for (int s = 0; s < kTcK / 16; ++s) {
        const uint32_t o = (uint32_t)s * 2 * tc::kLbo;  // K = 16 per MMA: two core matrices along K
        mma_bf16(acc, tc::smem_desc(tc::smem_u32(sA) + o), tc::smem_desc(tc::smem_u32(sB) + o),
                 (k0 == 0 && s == 0) ? 0u : 1u);
      }
      tc::mma_commit(&bar);
    }
    if (!tc::mbar_wait(&bar, parity)) s_fail = 1;
    parity ^= 1u;
    __syncthreads();
    if (s_fail) break;
  }
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (!s_fail) {
    const int row = warp * 32 + (tid & 31);
    const uint32_t lane_base = (uint32_t)(warp * 32) << 16;
    for (int c0 = 0; c0 < tc::kTile; c0 += 32) {
      uint32_t v[32];
      tc::tmem_ld32(acc + lane_base + (uint32_t)c0, v);
      const int m = m0 + row;
      if (m < M) {
#pragma unroll
        for (int q = 0; q < 32; ++q) {
          const int n = n0 + c0 + q;
          if (n < N) C[(int64_t)m * ldc + n] = __uint_as_float(v[q]);
        }
      }
    }
  } else if (tid == 0) {
    atomicExch(&g_mlp_tc_err, 1);
    tc::mbar_wait(&bar, parity ^ 1u);  // a bounded chance for MMAs in flight to drain
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(acc), "r"(128u));
  }
}

// Z = Z + bias (per column); relu -> H (bf16); keeps Z for the ReLU mask.
__global__ void k_bias_act(int rows, int cols, int ld, float* Z, const float* bias, bf16* H, bool relu) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (int64_t)rows * ld) return;
  const int c = (int)(i % ld);
  float v = Z[i] + (c < cols ? bias[c] : 0.0f);
  if (c >= cols) v = 0.0f;
  Z[i] = v;
  if (H) H[i] = __float2bfloat16(relu ? fmaxf(v, 0.0f) : v);
}

// dY = (Y - T) / B on real rows/columns (zero elsewhere); returns squared error partials.
__global__ void k_loss_grad(int rows_real, int rows, int cols, int ld, const float* Y, const float* T, float invB,
                            bf16* dY, float* dYf, double* sq) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  double e2 = 0.0;
  if (i < (int64_t)rows * ld) {
    const int r = (int)(i / ld), c = (int)(i % ld);
    float g = 0.0f;
    if (r < rows_real && c < cols) {
      const float e = Y[i] - T[i];
      e2 = (double)e * e;
      g = e * invB;
    }
    dY[i] = __float2bfloat16(g);
    dYf[i] = g;
  }
  for (int off = 16; off > 0; off >>= 1) e2 += __shfl_down_sync(0xffffffffu, e2, off);
  if ((threadIdx.x & 31) == 0 && e2 != 0.0) atomicAdd(sq, e2);
}

// dZ = dH * (Z > 0), as bf16 for the next products
__global__ void k_relu_back(int64_t total, const float* dH, const float* Z, bf16* dZ) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < total) dZ[i] = __float2bfloat16(Z[i] > 0.0f ? dH[i] : 0.0f);
}

// db[c] = sum_r dZ[r, c]
__global__ void k_colsum(int rows, int cols, int ld, const bf16* dZ, float* db) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= cols) return;
  float s = 0.0f;
  for (int r = 0; r < rows; ++r) s += __bfloat162float(dZ[(size_t)r * ld + c]);
  db[c] = s;
}

__global__ void k_f32_to_bf16(int64_t n, const float* src, bf16* dst) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = __float2bfloat16(src[i]);
}

// Adam on the FP32 master weights, then refresh the BF16 working copy.
__global__ void k_adam(int64_t n, float* w, const float* g, float* m, float* v, bf16* wb, float lr, float b1, float b2,
                       float c1, float c2, float eps) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.0f - b1) * gi;
  const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  w[i] = wi;
  if (wb) wb[i] = __float2bfloat16(wi);
}

struct Layer {
  int in, out, ldi, ldo;  // real and padded sizes
  float *W, *b, *gW, *gb, *mW, *vW, *mb, *vb;  // fp32 [ldo x ldi], [ldo]
  bf16* Wb;                                    // bf16 working copy
};

struct Net {
  int device = 0;
  cudaStream_t st = nullptr;
  int n_in, width, n_out, batch;
  std::vector<Layer> L;
  // activations for one batch (rows padded to 64)
  bf16 *X = nullptr, *H1 = nullptr, *H2 = nullptr, *dYb = nullptr, *dZ2 = nullptr, *dZ1 = nullptr;
  float *Z1 = nullptr, *Z2 = nullptr, *Y = nullptr, *T = nullptr, *dYf = nullptr, *dH2 = nullptr, *dH1 = nullptr;
  double* sq = nullptr;
  int64_t step = 0;
  PoolBlocks mem;  // blocks of the library's device memory pool
  std::string err;
  template <typename T>
  T* alloc(int64_t n) {
    void* p = mem.get(sizeof(T) * (size_t)std::max<int64_t>(n, 1));
    HPRQP_CUDA(cudaMemset(p, 0, sizeof(T) * (size_t)std::max<int64_t>(n, 1)));
    HPRQP_CUDA(cudaStreamSynchronize(cudaStreamLegacy));  // the net's stream does not wait for it
    return (T*)p;
  }
  ~Net() {
    pool_free(mem.blocks, mem.dev);
    if (st) cudaStreamDestroy(st);
  }
};

// C = opA(A) opB(B) (the callers never accumulate into C)
static void gemm(Net& N, bool TA, bool TB, int M, int Ncols, int K, const bf16* A, int lda, const bf16* B, int ldb,
                 float* C, int ldc, bool acc) {
  if (acc) throw Error(HPRQP_E_ARG, "mlp gemm: accumulation into C is not supported");
  static bool ready[64][4] = {};
  int dev = 0;
  HPRQP_CUDA(cudaGetDevice(&dev));
  const int v = (TA ? 2 : 0) | (TB ? 1 : 0);
  if (dev < 64 && !ready[dev][v]) {
    auto f = !TA && TB ? k_gemm<false, true> : !TA ? k_gemm<false, false> : !TB ? k_gemm<true, false> : k_gemm<true, true>;
    HPRQP_CUDA(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, kTcSmem));
    ready[dev][v] = true;
  }
  const dim3 grid((Ncols + tc::kTile - 1) / tc::kTile, (M + tc::kTile - 1) / tc::kTile);
  if (!TA && TB) k_gemm<false, true><<<grid, tc::kThreads, kTcSmem, N.st>>>(M, Ncols, K, A, lda, B, ldb, C, ldc);
  else if (!TA && !TB) k_gemm<false, false><<<grid, tc::kThreads, kTcSmem, N.st>>>(M, Ncols, K, A, lda, B, ldb, C, ldc);
  else if (TA && !TB) k_gemm<true, false><<<grid, tc::kThreads, kTcSmem, N.st>>>(M, Ncols, K, A, lda, B, ldb, C, ldc);
  else k_gemm<true, true><<<grid, tc::kThreads, kTcSmem, N.st>>>(M, Ncols, K, A, lda, B, ldb, C, ldc);
  HPRQP_LAUNCH_CHECK();
}

static inline int blocks(int64_t n) { return (int)((n + 255) / 256); }

// Forward for `rows_real` rows already in N.X; fills Z1, H1, Z2, H2, Y.
static void forward(Net& N) {
  const int R = N.batch;
  Layer &l1 = N.L[0], &l2 = N.L[1], &l3 = N.L[2];
  gemm(N, false, true, R, l1.ldo, l1.ldi, N.X, l1.ldi, l1.Wb, l1.ldi, N.Z1, l1.ldo, false);
  k_bias_act<<<blocks((int64_t)R * l1.ldo), 256, 0, N.st>>>(R, l1.out, l1.ldo, N.Z1, l1.b, N.H1, true);
  gemm(N, false, true, R, l2.ldo, l2.ldi, N.H1, l2.ldi, l2.Wb, l2.ldi, N.Z2, l2.ldo, false);
  k_bias_act<<<blocks((int64_t)R * l2.ldo), 256, 0, N.st>>>(R, l2.out, l2.ldo, N.Z2, l2.b, N.H2, true);
  gemm(N, false, true, R, l3.ldo, l3.ldi, N.H2, l3.ldi, l3.Wb, l3.ldi, N.Y, l3.ldo, false);
  k_bias_act<<<blocks((int64_t)R * l3.ldo), 256, 0, N.st>>>(R, l3.out, l3.ldo, N.Y, l3.b, nullptr, false);
  HPRQP_LAUNCH_CHECK();
}

// Backward for rows_real samples of the batch; gradients into gW/gb.
static void backward(Net& N, int rows_real) {
  const int R = N.batch;
  Layer &l1 = N.L[0], &l2 = N.L[1], &l3 = N.L[2];
  HPRQP_CUDA(cudaMemsetAsync(N.sq, 0, sizeof(double), N.st));
  k_loss_grad<<<blocks((int64_t)R * l3.ldo), 256, 0, N.st>>>(rows_real, R, l3.out, l3.ldo, N.Y, N.T,
                                                            1.0f / (float)rows_real, N.dYb, N.dYf, N.sq);
  // layer 3: gW3 = dY^T H2 ; gb3 = colsum dY ; dH2 = dY W3
  gemm(N, true, false, l3.ldo, l3.ldi, R, N.dYb, l3.ldo, N.H2, l3.ldi, l3.gW, l3.ldi, false);
  k_colsum<<<blocks(l3.ldo), 256, 0, N.st>>>(R, l3.out, l3.ldo, N.dYb, l3.gb);
  gemm(N, false, false, R, l3.ldi, l3.ldo, N.dYb, l3.ldo, l3.Wb, l3.ldi, N.dH2, l3.ldi, false);
  k_relu_back<<<blocks((int64_t)R * l2.ldo), 256, 0, N.st>>>((int64_t)R * l2.ldo, N.dH2, N.Z2, N.dZ2);
  // layer 2
  gemm(N, true, false, l2.ldo, l2.ldi, R, N.dZ2, l2.ldo, N.H1, l2.ldi, l2.gW, l2.ldi, false);
  k_colsum<<<blocks(l2.ldo), 256, 0, N.st>>>(R, l2.out, l2.ldo, N.dZ2, l2.gb);
  gemm(N, false, false, R, l2.ldi, l2.ldo, N.dZ2, l2.ldo, l2.Wb, l2.ldi, N.dH1, l2.ldi, false);
  k_relu_back<<<blocks((int64_t)R * l1.ldo), 256, 0, N.st>>>((int64_t)R * l1.ldo, N.dH1, N.Z1, N.dZ1);
  // layer 1
  gemm(N, true, false, l1.ldo, l1.ldi, R, N.dZ1, l1.ldo, N.X, l1.ldi, l1.gW, l1.ldi, false);
  k_colsum<<<blocks(l1.ldo), 256, 0, N.st>>>(R, l1.out, l1.ldo, N.dZ1, l1.gb);
  HPRQP_LAUNCH_CHECK();
}

static void upload_rows(Net& N, bf16* dst, float* dstf, int ld, const float* src, int rows, int cols) {
  // host rows (cols wide) -> padded device rows; rows beyond `rows` zero
  std::vector<float> buf((size_t)N.batch * ld, 0.0f);
  for (int r = 0; r < rows; ++r) std::memcpy(&buf[(size_t)r * ld], src + (size_t)r * cols, sizeof(float) * cols);
  if (dstf) HPRQP_CUDA(cudaMemcpyAsync(dstf, buf.data(), sizeof(float) * buf.size(), cudaMemcpyHostToDevice, N.st));
  if (dst) {
    std::vector<bf16> bb(buf.size());
    for (size_t i = 0; i < buf.size(); ++i) bb[i] = __float2bfloat16(buf[i]);
    HPRQP_CUDA(cudaMemcpyAsync(dst, bb.data(), sizeof(bf16) * bb.size(), cudaMemcpyHostToDevice, N.st));
    HPRQP_CUDA(cudaStreamSynchronize(N.st));
  }
  HPRQP_CUDA(cudaStreamSynchronize(N.st));
}

}  // namespace mlp
}  // namespace hprqp

using namespace hprqp;
using namespace hprqp::mlp;

struct hprqp_mlp : Net {};
static thread_local std::string g_mlp_err;

#define MLP_GUARD(h, ...)                        \
  try {                                          \
    if (h) cudaSetDevice(h->device);             \
    __VA_ARGS__;                                 \
    return HPRQP_OK;                             \
  } catch (const Error& e) {                     \
    (h ? h->err : g_mlp_err) = e.what();         \
    return e.code;                               \
  }

extern "C" {

int hprqp_mlp_create(hprqp_mlp_handle* out, int32_t device, int32_t n_in, int32_t width, int32_t n_out,
                     int32_t batch, uint64_t seed) {
  hprqp_mlp* h = nullptr;
  try {
    if (!out || n_in <= 0 || width <= 0 || n_out <= 0 || batch <= 0) throw Error(HPRQP_E_ARG, "bad MLP sizes");
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count)
      throw Error(HPRQP_E_CUDA, "CUDA device unavailable");
    HPRQP_CUDA(cudaSetDevice(device));
    h = new hprqp_mlp();
    h->device = device;
    HPRQP_CUDA(cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking));
    h->n_in = n_in;
    h->width = width;
    h->n_out = n_out;
    h->batch = (int)pad64(batch);
    const int dims[4] = {n_in, width, width, n_out};
    uint64_t s = seed ? seed : 1;
    auto rnd = [&s]() {  // splitmix64 -> uniform (-1, 1)
      uint64_t v = (s += 0x9E3779B97F4A7C15ULL);
      v = (v ^ (v >> 30)) * 0xBF58476D1CE4E5B9ULL;
      v = (v ^ (v >> 27)) * 0x94D049BB133111EBULL;
      v ^= v >> 31;
      return (double)(v >> 11) * 0x1.0p-52 - 1.0;
    };
    for (int k = 0; k < 3; ++k) {
      Layer l{};
      l.in = dims[k];
      l.out = dims[k + 1];
      l.ldi = (int)pad64(l.in);
      l.ldo = (int)pad64(l.out);
      const int64_t nw = (int64_t)l.ldo * l.ldi;
      l.W = h->alloc<float>(nw);
      l.gW = h->alloc<float>(nw);
      l.mW = h->alloc<float>(nw);
      l.vW = h->alloc<float>(nw);
      l.Wb = h->alloc<bf16>(nw);
      l.b = h->alloc<float>(l.ldo);
      l.gb = h->alloc<float>(l.ldo);
      l.mb = h->alloc<float>(l.ldo);
      l.vb = h->alloc<float>(l.ldo);
      // He-uniform init on the real block, zero padding
      std::vector<float> w(nw, 0.0f);
      const double a = std::sqrt(6.0 / l.in);
      for (int o = 0; o < l.out; ++o)
        for (int i = 0; i < l.in; ++i) w[(size_t)o * l.ldi + i] = (float)(a * rnd());
      std::vector<bf16> wb(nw);
      for (int64_t i = 0; i < nw; ++i) wb[i] = __float2bfloat16(w[i]);
      HPRQP_CUDA(cudaMemcpyAsync(l.W, w.data(), sizeof(float) * nw, cudaMemcpyHostToDevice, h->st));
      HPRQP_CUDA(cudaStreamSynchronize(h->st));
      HPRQP_CUDA(cudaMemcpyAsync(l.Wb, wb.data(), sizeof(bf16) * nw, cudaMemcpyHostToDevice, h->st));
      HPRQP_CUDA(cudaStreamSynchronize(h->st));
      h->L.push_back(l);
    }
    const int R = h->batch;
    Layer &l1 = h->L[0], &l2 = h->L[1], &l3 = h->L[2];
    h->X = h->alloc<bf16>((int64_t)R * l1.ldi);
    h->Z1 = h->alloc<float>((int64_t)R * l1.ldo);
    h->H1 = h->alloc<bf16>((int64_t)R * l1.ldo);
    h->Z2 = h->alloc<float>((int64_t)R * l2.ldo);
    h->H2 = h->alloc<bf16>((int64_t)R * l2.ldo);
    h->Y = h->alloc<float>((int64_t)R * l3.ldo);
    h->T = h->alloc<float>((int64_t)R * l3.ldo);
    h->dYb = h->alloc<bf16>((int64_t)R * l3.ldo);
    h->dYf = h->alloc<float>((int64_t)R * l3.ldo);
    h->dH2 = h->alloc<float>((int64_t)R * l2.ldo);
    h->dZ2 = h->alloc<bf16>((int64_t)R * l2.ldo);
    h->dH1 = h->alloc<float>((int64_t)R * l1.ldo);
    h->dZ1 = h->alloc<bf16>((int64_t)R * l1.ldo);
    h->sq = h->alloc<double>(1);
    *out = h;
    return HPRQP_OK;
  } catch (const Error& e) {
    g_mlp_err = e.what();
    delete h;
    return e.code;
  }
}

int hprqp_mlp_train_batch(hprqp_mlp_handle h, const float* X, const float* T, int32_t rows, float lr,
                          double* loss_out) {
  if (!h || !X || !T || rows <= 0) return HPRQP_E_ARG;
  MLP_GUARD(h, {
    if (rows > h->batch) throw Error(HPRQP_E_ARG, "rows exceed the batch size");
    upload_rows(*h, h->X, nullptr, h->L[0].ldi, X, rows, h->n_in);
    upload_rows(*h, nullptr, h->T, h->L[2].ldo, T, rows, h->n_out);
    forward(*h);
    backward(*h, rows);
    h->step++;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.0f - std::pow(b1, (float)h->step), c2 = 1.0f - std::pow(b2, (float)h->step);
    for (auto& l : h->L) {
      const int64_t nw = (int64_t)l.ldo * l.ldi;
      k_adam<<<blocks(nw), 256, 0, h->st>>>(nw, l.W, l.gW, l.mW, l.vW, l.Wb, lr, b1, b2, c1, c2, 1e-8f);
      k_adam<<<blocks(l.ldo), 256, 0, h->st>>>(l.ldo, l.b, l.gb, l.mb, l.vb, nullptr, lr, b1, b2, c1, c2, 1e-8f);
    }
    HPRQP_LAUNCH_CHECK();
    double sq = 0;
    HPRQP_CUDA(cudaMemcpyAsync(&sq, h->sq, sizeof(double), cudaMemcpyDeviceToHost, h->st));
    HPRQP_CUDA(cudaStreamSynchronize(h->st));
    if (loss_out) *loss_out = 0.5 * sq / rows;
  })
}

int hprqp_mlp_gradients(hprqp_mlp_handle h, const float* X, const float* T, int32_t rows, float* grads,
                        double* loss_out) {
  if (!h || !X || !T || rows <= 0 || !grads) return HPRQP_E_ARG;
  MLP_GUARD(h, {
    if (rows > h->batch) throw Error(HPRQP_E_ARG, "rows exceed the batch size");
    upload_rows(*h, h->X, nullptr, h->L[0].ldi, X, rows, h->n_in);
    upload_rows(*h, nullptr, h->T, h->L[2].ldo, T, rows, h->n_out);
    forward(*h);
    backward(*h, rows);
    double sq = 0;
    HPRQP_CUDA(cudaMemcpyAsync(&sq, h->sq, sizeof(double), cudaMemcpyDeviceToHost, h->st));
    HPRQP_CUDA(cudaStreamSynchronize(h->st));
    if (loss_out) *loss_out = 0.5 * sq / rows;
    // unpadded [W1, b1, W2, b2, W3, b3], W row-major out x in
    size_t off = 0;
    for (auto& l : h->L) {
      std::vector<float> g((size_t)l.ldo * l.ldi), gb(l.ldo);
      HPRQP_CUDA(cudaMemcpyAsync(g.data(), l.gW, sizeof(float) * g.size(), cudaMemcpyDeviceToHost, h->st));
      HPRQP_CUDA(cudaStreamSynchronize(h->st));
      HPRQP_CUDA(cudaMemcpyAsync(gb.data(), l.gb, sizeof(float) * gb.size(), cudaMemcpyDeviceToHost, h->st));
      HPRQP_CUDA(cudaStreamSynchronize(h->st));
      for (int o = 0; o < l.out; ++o)
        for (int i = 0; i < l.in; ++i) grads[off++] = g[(size_t)o * l.ldi + i];
      for (int o = 0; o < l.out; ++o) grads[off++] = gb[o];
    }
  })
}

int hprqp_mlp_predict(hprqp_mlp_handle h, const float* X, int64_t rows, float* Y) {
  if (!h || !X || !Y || rows < 0) return HPRQP_E_ARG;
  MLP_GUARD(h, {
    const Layer& l3 = h->L[2];
    std::vector<float> out((size_t)h->batch * l3.ldo);
    for (int64_t r0 = 0; r0 < rows; r0 += h->batch) {
      const int cnt = (int)std::min<int64_t>(h->batch, rows - r0);
      upload_rows(*h, h->X, nullptr, h->L[0].ldi, X + (size_t)r0 * h->n_in, cnt, h->n_in);
      forward(*h);
      HPRQP_CUDA(cudaMemcpyAsync(out.data(), h->Y, sizeof(float) * out.size(), cudaMemcpyDeviceToHost, h->st));
      HPRQP_CUDA(cudaStreamSynchronize(h->st));
      for (int r = 0; r < cnt; ++r)
        std::memcpy(Y + (size_t)(r0 + r) * h->n_out, &out[(size_t)r * l3.ldo], sizeof(float) * h->n_out);
    }
  })
}

int hprqp_mlp_get_params(hprqp_mlp_handle h, float* params, int64_t* count) {
  if (!h || !count) return HPRQP_E_ARG;
  MLP_GUARD(h, {
    int64_t total = 0;
    for (auto& l : h->L) total += (int64_t)l.out * l.in + l.out;
    if (params) {
      size_t off = 0;
      for (auto& l : h->L) {
        std::vector<float> w((size_t)l.ldo * l.ldi), b(l.ldo);
        HPRQP_CUDA(cudaMemcpyAsync(w.data(), l.W, sizeof(float) * w.size(), cudaMemcpyDeviceToHost, h->st));
      HPRQP_CUDA(cudaStreamSynchronize(h->st));
        HPRQP_CUDA(cudaMemcpyAsync(b.data(), l.b, sizeof(float) * b.size(), cudaMemcpyDeviceToHost, h->st));
      HPRQP_CUDA(cudaStreamSynchronize(h->st));
        for (int o = 0; o < l.out; ++o)
          for (int i = 0; i < l.in; ++i) params[off++] = w[(size_t)o * l.ldi + i];
        for (int o = 0; o < l.out; ++o) params[off++] = b[o];
      }
    }
    *count = total;
  })
}

int hprqp_mlp_set_params(hprqp_mlp_handle h, const float* params) {
  if (!h || !params) return HPRQP_E_ARG;
  MLP_GUARD(h, {
    size_t off = 0;
    for (auto& l : h->L) {
      std::vector<float> w((size_t)l.ldo * l.ldi, 0.0f), b(l.ldo, 0.0f);
      for (int o = 0; o < l.out; ++o)
        for (int i = 0; i < l.in; ++i) w[(size_t)o * l.ldi + i] = params[off++];
      for (int o = 0; o < l.out; ++o) b[o] = params[off++];
      std::vector<bf16> wb(w.size());
      for (size_t i = 0; i < w.size(); ++i) wb[i] = __float2bfloat16(w[i]);
      HPRQP_CUDA(cudaMemcpyAsync(l.W, w.data(), sizeof(float) * w.size(), cudaMemcpyHostToDevice, h->st));
      HPRQP_CUDA(cudaStreamSynchronize(h->st));
      HPRQP_CUDA(cudaMemcpyAsync(l.Wb, wb.data(), sizeof(bf16) * wb.size(), cudaMemcpyHostToDevice, h->st));
      HPRQP_CUDA(cudaStreamSynchronize(h->st));
      HPRQP_CUDA(cudaMemcpyAsync(l.b, b.data(), sizeof(float) * b.size(), cudaMemcpyHostToDevice, h->st));
      HPRQP_CUDA(cudaStreamSynchronize(h->st));
    }
  })
}

const char* hprqp_mlp_last_error(hprqp_mlp_handle h) { return h ? h->err.c_str() : g_mlp_err.c_str(); }

int hprqp_mlp_destroy(hprqp_mlp_handle h) {
  if (h) {
    cudaSetDevice(h->device);
    delete h;
  }
  return HPRQP_OK;
}

}  // extern "C"
