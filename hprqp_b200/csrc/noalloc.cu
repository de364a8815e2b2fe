// noalloc.cu — hprqp_power_lambda_noalloc: lambda_max(A A') by the power
// method on a caller-owned device CSR matrix, with no device allocation.
//
// Why it exists: some callers of this library cannot call cudaMalloc at the
// point where they need the estimate — programs whose device memory belongs
// to another framework's pool allocator (a second allocator on the same GPU
// would fragment or overcommit that pool), and real-time or long-running
// loops that forbid allocation after start-up (an allocation there can
// block on the driver or fail at an unpredictable moment).  For them this
// entry point works entirely in memory the caller already owns plus one
// fixed block of scratch that the library reserves when it is loaded.
//
// The call is synchronous: every 32 steps it reads the (lambda, err) log
// back to the host, waiting on the caller's stream, and it returns after the
// stream has finished its work.  The first call in each CUDA context does
// the set-up below; make that first call before any stream capture.
//
// The scratch is the file-scope array g_noalloc_scratch below: the power
// method's three work vectors (two m-vectors, one n-vector), the reduction
// partials and ticket, and the (lambda, err) log.  Its size is fixed at
// build time (kNoAllocVecCap doubles for the vectors, i.e. 8 MiB, plus a
// 256 KiB control block), and every GPU that loads libhprqp holds it until
// the process exits.  Problems with 2m + n > kNoAllocVecCap are rejected.
//
// Host code must not pass the array's name to a kernel: in host code it is
// a host-side stand-in, not a device address.  The device address is looked
// up with cudaGetSymbolAddress, with the device current, by the first call
// made in each CUDA context (the primary context of a device, or a context
// the caller made current), and cached under that context's unique id; a
// new context (after cudaDeviceReset, say) gets a fresh look-up.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <string>

#include "../../include/hprqp.h"
#include "kernels.cuh"

namespace hprqp {

extern void set_global_error(const std::string& msg);

namespace {

constexpr int64_t kNoAllocVecCap = int64_t(1) << 20;  // doubles for z, z_next, t
constexpr int64_t kCtrl = 32768;                       // doubles of control block
constexpr int64_t kOffPartials = 1024;                 // partials start (double index)
constexpr int64_t kOffScal = 64;                       // zz, lambda, zz_next, qq
constexpr int64_t kOffLog = 128;                       // (lambda, err) per chunk step
constexpr int kChunk = 32;
constexpr int kMaxDevices = 64;
static_assert(kOffPartials + (int64_t)kMaxReduceGrid * 16 <= kCtrl, "control block too small");

// Index 0 holds the reduction ticket (as an unsigned int).
static __device__ __align__(256) double g_noalloc_scratch[kCtrl + kNoAllocVecCap];

std::mutex g_mu;                                   // serialises host-side use
double* g_dev_ptr[kMaxDevices] = {nullptr};        // device address, per device ...
unsigned long long g_ctx_id[kMaxDevices] = {0};    // ... valid in this context only

#define NA_CHECK(call)                                                                 \
  do {                                                                                 \
    cudaError_t e_ = (call);                                                           \
    if (e_ != cudaSuccess) {                                                           \
      set_global_error(std::string("hprqp_power_lambda_noalloc: ") + #call + ": " +   \
                       cudaGetErrorString(e_));                                        \
      return HPRQP_E_CUDA;                                                             \
    }                                                                                  \
  } while (0)

// The products and the stopping test of the engine's power method (its
// two-product form, one CTA fold per step), so lambda agrees with
// hprqp_solve's lambda_max_A / eig_factor for the same matrix to rounding:
// the engine folds the chains once per 32-step chunk or runs the A A' chain
// on the Gram matrix A'A, which sums the same dot products in another order.
template <int TPR>
int power_steps(int m, int n, CsrSrc<double, double> At_z, CsrSrc<double, double> A_t, double* za, double* zb,
                double* t, double* scal, double* log, ReduceWs ws, cudaStream_t st, int k) {
  double* zz = scal + 2;
  const bool odd = (k & 1) != 0;
  double* zc = odd ? zb : za;
  double* zn = odd ? za : zb;
  At_z.x = zc;
  A_t.x = t;
  {
    const long long threads = (long long)n * TPR;
    const int grid = (int)((threads + kBlock - 1) / kBlock);
    k_row_pass<TPR, double><<<grid, kBlock, 0, st>>>(n, At_z, EpiStoreInvNorm<double>{t, zz});
  }
  {
    const int grid = reduce_grid(m, TPR);
    k_row_reduce<TPR, 3, 0u, double><<<grid, kBlock, 0, st>>>(m, A_t, EpiPowerFused<double>{zc, zn, zz, false}, ws,
                                                               scal + 1, PowerFin{log, k % kChunk});
  }
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

}  // namespace
}  // namespace hprqp

extern "C" int hprqp_power_lambda_noalloc(int64_t m, int64_t n, const int32_t* A_rowptr, const int32_t* A_colind,
                                          const double* A_val, const int32_t* AT_rowptr, const int32_t* AT_colind,
                                          const double* AT_val, int32_t threads_per_row, double tol, int32_t max_iter,
                                          void* stream, double* lambda_out, int32_t* iters_out) {
  using namespace hprqp;
  std::lock_guard<std::mutex> lock(g_mu);
  if (m <= 0 || n <= 0 || !A_rowptr || !A_colind || !A_val || !AT_rowptr || !AT_colind || !AT_val || !lambda_out ||
      !(tol > 0) || max_iter <= 0) {
    set_global_error("hprqp_power_lambda_noalloc: invalid argument");
    return HPRQP_E_ARG;
  }
  // m and n are each checked first, so 2m + n cannot overflow
  if (m > kNoAllocVecCap || n > kNoAllocVecCap || 2 * m + n > kNoAllocVecCap) {
    const std::string need = (m > kNoAllocVecCap || n > kNoAllocVecCap)
                                  ? std::string("m = ") + std::to_string(m) + ", n = " + std::to_string(n)
                                  : std::to_string(2 * m + n);
    set_global_error("hprqp_power_lambda_noalloc: problem too large for the fixed scratch: needs 2m + n = " + need +
                     " doubles, capacity is " + std::to_string(kNoAllocVecCap));
    return HPRQP_E_ARG;
  }
  int tpr = threads_per_row;
  if (tpr != 1 && tpr != 2 && tpr != 4 && tpr != 8 && tpr != 16 && tpr != 32) {
    set_global_error("hprqp_power_lambda_noalloc: threads_per_row must be 1, 2, 4, 8, 16 or 32");
    return HPRQP_E_ARG;
  }
  int dev = 0;
  NA_CHECK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) {
    set_global_error("hprqp_power_lambda_noalloc: device index out of range");
    return HPRQP_E_CUDA;
  }
  // Set-up, once per context, with the device current: the array's device
  // address.  The context's id (unique for the life of the process) tells
  // whether a cached address still belongs to the current context.
  unsigned long long ctx_id = 0;
  {
    static CUresult (*get_current)(CUcontext*) = nullptr;
    static CUresult (*get_id)(CUcontext, unsigned long long*) = nullptr;
    if (!get_current || !get_id) {
      cudaDriverEntryPointQueryResult q1, q2;
      NA_CHECK(cudaGetDriverEntryPoint("cuCtxGetCurrent", (void**)&get_current, cudaEnableDefault, &q1));
      NA_CHECK(cudaGetDriverEntryPoint("cuCtxGetId", (void**)&get_id, cudaEnableDefault, &q2));
      if (q1 != cudaDriverEntryPointSuccess || q2 != cudaDriverEntryPointSuccess || !get_current || !get_id) {
        get_current = nullptr;
        get_id = nullptr;
        set_global_error("hprqp_power_lambda_noalloc: the driver lacks cuCtxGetCurrent / cuCtxGetId");
        return HPRQP_E_CUDA;
      }
    }
    CUcontext ctx = nullptr;
    if (get_current(&ctx) == CUDA_SUCCESS && !ctx) {
      NA_CHECK(cudaSetDevice(dev));  // no context yet: start the device's primary one
      get_current(&ctx);
    }
    if (!ctx || get_id(ctx, &ctx_id) != CUDA_SUCCESS) {
      set_global_error("hprqp_power_lambda_noalloc: no current CUDA context");
      return HPRQP_E_CUDA;
    }
  }
  if (!g_dev_ptr[dev] || g_ctx_id[dev] != ctx_id) {
    void* p = nullptr;
    NA_CHECK(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    g_dev_ptr[dev] = (double*)p;
    g_ctx_id[dev] = ctx_id;
  }
  cudaStream_t st = (cudaStream_t)stream;
  double* base = g_dev_ptr[dev];
  double* scal = base + kOffScal;
  double* log = base + kOffLog;
  ReduceWs ws{base + kOffPartials, reinterpret_cast<unsigned*>(base)};
  double* za = base + kCtrl;
  double* zb = za + m;
  double* t = zb + m;
  // The ticket and the scalar slots must start at zero; the rest of the
  // scratch keeps whatever the previous call left and is overwritten.
  NA_CHECK(cudaMemsetAsync(base, 0, sizeof(double) * kOffPartials, st));
  // the start vector of hprqp_solve's power method, generated in place
  k_start_vector<double><<<(int)((m + kBlock - 1) / kBlock), kBlock, 0, st>>>(m, za);
  NA_CHECK(cudaGetLastError());
  {
    const int grid = reduce_grid(m, 1);
    k_row_reduce<1, 1, 0u, double><<<grid, kBlock, 0, st>>>((int)m, ZeroSrc{}, EpiSumSq<double>{za}, ws, scal + 2);
    NA_CHECK(cudaGetLastError());
  }
  CsrSrc<double, double> At_z{AT_rowptr, AT_colind, AT_val, nullptr};
  CsrSrc<double, double> A_t{A_rowptr, A_colind, A_val, nullptr};
  double lam = 1.0, hostlog[2 * kChunk];
  int it = 0, found = -1;
  while (it < max_iter && found < 0) {
    for (int k = 0; k < kChunk; ++k) {
      int rc = 0;
      switch (tpr) {
        case 1: rc = power_steps<1>((int)m, (int)n, At_z, A_t, za, zb, t, scal, log, ws, st, k); break;
        case 2: rc = power_steps<2>((int)m, (int)n, At_z, A_t, za, zb, t, scal, log, ws, st, k); break;
        case 4: rc = power_steps<4>((int)m, (int)n, At_z, A_t, za, zb, t, scal, log, ws, st, k); break;
        case 8: rc = power_steps<8>((int)m, (int)n, At_z, A_t, za, zb, t, scal, log, ws, st, k); break;
        case 16: rc = power_steps<16>((int)m, (int)n, At_z, A_t, za, zb, t, scal, log, ws, st, k); break;
        default: rc = power_steps<32>((int)m, (int)n, At_z, A_t, za, zb, t, scal, log, ws, st, k); break;
      }
      if (rc) NA_CHECK(cudaGetLastError());
    }
    NA_CHECK(cudaMemcpyAsync(hostlog, log, sizeof(hostlog), cudaMemcpyDeviceToHost, st));
    NA_CHECK(cudaStreamSynchronize(st));
    for (int k = 0; k < kChunk && it + k < max_iter; ++k) {
      lam = hostlog[2 * k];
      if (hostlog[2 * k + 1] < tol) {
        found = it + k + 1;
        break;
      }
    }
    it += kChunk;
  }
  *lambda_out = lam;
  if (iters_out) *iters_out = found > 0 ? found : std::min(it, (int)max_iter);
  return HPRQP_OK;
}
