// engine.cu — Engine<V>: uploads, launch wrappers and the device-side steps
// of the HPR loop.  See engine.cuh.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstring>
#include <cstdlib>
#include <functional>
#include <unordered_map>
#include <mutex>
#include <type_traits>

#include "engine.cuh"
#include "qap_gemm.cuh"
#include "power.cuh"
#include "tc_gemm.h"

namespace hprqp {


static double wall_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// ---------------------------------------------------------------------------
// Common
// ---------------------------------------------------------------------------
void Common::init() {
  HPRQP_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
  HPRQP_CUDA(cudaStreamCreateWithFlags(&stream2, cudaStreamNonBlocking));
  d_scal = mem.alloc<double>(kNumSlots);
  HPRQP_CUDA(cudaMemsetAsync(d_scal, 0, sizeof(double) * kNumSlots, stream));
  h_scal = (double*)pinned_take(sizeof(double) * kNumSlots);
  rws.partials = mem.alloc<double>((int64_t)kReduceGridLimit * 16);
  rws.counter = mem.alloc<unsigned>(4);
  HPRQP_CUDA(cudaMemsetAsync(rws.counter, 0, sizeof(unsigned) * 4, stream));
  rws2.partials = mem.alloc<double>((int64_t)kReduceGridLimit * 16);
  rws2.counter = mem.alloc<unsigned>(4);
  HPRQP_CUDA(cudaMemsetAsync(rws2.counter, 0, sizeof(unsigned) * 4, stream));
  HPRQP_CUDA(cudaStreamSynchronize(stream));  // (the second chain's stream uses rws2 too)
  int dev = 0;
  HPRQP_CUDA(cudaGetDevice(&dev));
  HPRQP_CUDA(cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, dev));
  const char* e = std::getenv("HPRQP_PDL");
  pdl = !(e && e[0] == '0');
  pow_part = mem.alloc<double>(2 * 2 * kPowMaxGrid * 3);
  pow_bar = mem.alloc<unsigned>(64);  // [0] arrivals, [1] status, [32] released phase
  const char* pe = std::getenv("HPRQP_POWER_PERSISTENT");
  pow_persistent = pe && pe[0] == '1';
  const char* tq = std::getenv("HPRQP_QAP_TC");
  tc_qap = !(tq && tq[0] == '0');
  const char* ps = std::getenv("HPRQP_POWER_SPLIT");
  pow_split = ps && ps[0] == '1';
  const char* rc = std::getenv("HPRQP_REDUCE_CAP");
  if (rc) reduce_cap = std::max(1, std::min(std::atoi(rc), kReduceGridLimit));
  const char* pel = std::getenv("HPRQP_POWER_ELL");
  pow_prefer_ell = pel && pel[0] == '1';
  const char* cf = std::getenv("HPRQP_POWER_CHUNK_FOLD");
  pow_chunk_fold = !(cf && cf[0] == '0');
  const char* at = std::getenv("HPRQP_AUTOTUNE");
  autotune = !(at && at[0] == '0');
  const char* sc = std::getenv("HPRQP_SCHED_CACHE");
  sched_cache = !(sc && sc[0] == '0');
  const char* ppr = std::getenv("HPRQP_POWER_PRELOAD_ROWS");
  if (ppr) pow_rows_preloaded = std::atoi(ppr) == 1 ? 1 : 2;
  const char* ept = std::getenv("HPRQP_ELL_PROLOGUE");
  if (ept) ell_prologue = std::max(0, std::min(std::atoi(ept), 2));
  const char* ep = std::getenv("HPRQP_EPI_PREFETCH");
  if (ep) epi_prefetch = std::max(0, std::min(std::atoi(ep), 2));
  const char* pg = std::getenv("HPRQP_POWER_GRAM");
  if (pg) pow_gram = pg[0] == '0' ? 0 : 1;
  const char* pc = std::getenv("HPRQP_POWER_CTAS_PER_SM");
  if (pc) pow_ctas_per_sm = std::atoi(pc);
}

Common::~Common() {
  const double t0 = wall_s();
  if (h_scal) pinned_give(h_scal, sizeof(double) * kNumSlots);
  const double t1 = wall_s();
  if (stream) cudaStreamDestroy(stream);
  if (stream2) cudaStreamDestroy(stream2);
  const double t2 = wall_s();
  pool_free(mem.blocks, mem.dev);
  if (const char* tv = std::getenv("HPRQP_TIMING"))
    if (tv[0] == '1')
      std::fprintf(stderr, "[hprqp] handle resources: pinned %.3f s, streams %.3f s, device blocks %.3f s\n", t1 - t0,
                   t2 - t1, wall_s() - t2);
}

void Common::sync_read(int first, int count) {
  to_host(h_scal + first, d_scal + first, sizeof(double) * count);
  HPRQP_CUDA(cudaStreamSynchronize(stream));
}

// ---------------------------------------------------------------------------
// Launch wrappers.  Every kernel of the engine starts with pdl_enter(), so
// all are launched with programmatic stream serialisation.
// ---------------------------------------------------------------------------
template <typename... KArgs, typename... Args>
static void launch(Common& cm, void (*kernel)(KArgs...), dim3 grid, int block, Args... args) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = grid;
  cfg.blockDim = dim3((unsigned)block);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = cm.stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = cm.pdl ? 1 : 0;
  HPRQP_CUDA(cudaLaunchKernelEx(&cfg, kernel, args...));
  cm.launches++;
}

// launch() with dynamic shared memory; the kernel's limit is raised once per
// device to the staged pass's column block and row-sum slots
template <typename... KArgs, typename... Args>
static void launch_smem(Common& cm, void (*kernel)(KArgs...), dim3 grid, int block, size_t smem, Args... args) {
  static std::atomic<uint64_t> raised{0};  // bit d: done on device d
  int dev = 0;
  HPRQP_CUDA(cudaGetDevice(&dev));
  const uint64_t bit = 1ull << (dev & 63);
  if (!(raised.load() & bit)) {
    HPRQP_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    kStageSmem + kStageSlots * (int)sizeof(double)));
    raised.fetch_or(bit);
  }
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = grid;
  cfg.blockDim = dim3((unsigned)block);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = cm.stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = cm.pdl ? 1 : 0;
  HPRQP_CUDA(cudaLaunchKernelEx(&cfg, kernel, args...));
  cm.launches++;
}

// ---------------------------------------------------------------------------
// Schedule cache: the autotuner's timed choices by sparsity signature, for
// the process.  A handle that loads a problem of a pattern tuned before (the
// load -> solve -> destroy cycle of a caller solving a family of problems)
// builds only the chosen format copy and times nothing.
// ---------------------------------------------------------------------------
namespace {
enum SchedKind { SK_CSR = 0, SK_SELL = 1, SK_ELL = 2, SK_SPLIT = 3, SK_STAGE = 4 };
struct SchedChoice {
  int kind, tpr;
};
std::mutex g_sched_mu;
std::unordered_map<uint64_t, SchedChoice>& sched_map() {
  static std::unordered_map<uint64_t, SchedChoice> m;
  return m;
}

uint64_t mix64(uint64_t z) {  // splitmix64 finaliser
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

// Signature of a pattern (sizes, row pointers, columns) and a tag: 64 fixed
// chunks hashed in parallel, combined in order, so the key does not depend
// on the thread count.
uint64_t pattern_key(const HCsr& h, uint64_t tag) {
  constexpr int kParts = 64;
  const int64_t np = (int64_t)h.ptr.size(), nc = (int64_t)h.col.size(), total = np + nc;
  uint64_t part[kParts];
#pragma omp parallel for schedule(static) num_threads(host_threads(total))
  for (int q = 0; q < kParts; ++q) {
    uint64_t x = 0x9E3779B97F4A7C15ULL * (uint64_t)(q + 1);
    for (int64_t i = total * q / kParts; i < total * (q + 1) / kParts; ++i)
      x = mix64(x ^ (uint64_t)(uint32_t)(i < np ? h.ptr[i] : h.col[i - np]));
    part[q] = x;
  }
  uint64_t k = mix64(tag ^ 0xD6E8FEB86659FD93ULL);
  k = mix64(k ^ (uint64_t)h.rows) ^ mix64((uint64_t)h.cols + 0x2545F4914F6CDD1DULL);
  for (int q = 0; q < kParts; ++q) k = mix64(k ^ part[q]);
  return k;
}

bool sched_lookup(uint64_t key, SchedChoice& c) {
  std::lock_guard<std::mutex> lk(g_sched_mu);
  auto it = sched_map().find(key);
  if (it == sched_map().end()) return false;
  c = it->second;
  return true;
}
void sched_store(uint64_t key, SchedChoice c) {
  std::lock_guard<std::mutex> lk(g_sched_mu);
  sched_map()[key] = c;
}
}  // namespace

// threads per row of a CSR pass by the mean row length (the fixed rule)
static int csr_tpr(double avg) {
  int t = 1;
  while (t < 32 && avg >= 4.0 * t) t *= 2;
  return t;
}

template <int TPR, typename Acc, typename Src, typename Epi>
static void rows_t(Common& cm, int nrows, const Src& src, const Epi& epi) {
  const long long threads = (long long)nrows * TPR;
  const int grid = (int)((threads + kBlock - 1) / kBlock);
  launch(cm, k_row_pass<TPR, Acc, Src, Epi>, grid, kBlock, nrows, src, epi, cm.epi_prefetch);
}

template <typename Acc, typename Src, typename Epi>
static void rows(Common& cm, int tpr, int64_t nrows, const Src& src, const Epi& epi) {
  if (nrows <= 0) return;
  switch (tpr) {
    case 1: rows_t<1, Acc>(cm, (int)nrows, src, epi); break;
    case 2: rows_t<2, Acc>(cm, (int)nrows, src, epi); break;
    case 4: rows_t<4, Acc>(cm, (int)nrows, src, epi); break;
    case 8: rows_t<8, Acc>(cm, (int)nrows, src, epi); break;
    case 16: rows_t<16, Acc>(cm, (int)nrows, src, epi); break;
    case 32: rows_t<32, Acc>(cm, (int)nrows, src, epi); break;
    default: throw Error(HPRQP_E_ARG, "bad threads-per-row");
  }
}

template <int TPR, int K, unsigned MM, typename Acc, typename Src, typename Epi, typename Fin>
static void reduce_t(Common& cm, int nrows, const Src& src, const Epi& epi, double* out, const Fin& fin) {
  const int grid = reduce_grid(nrows, TPR, cm.reduce_cap);
  launch(cm, k_row_reduce<TPR, K, MM, Acc, Src, Epi, Fin>, grid, kBlock, nrows, src, epi, cm.rws, out, fin);
}

template <int K, unsigned MM, typename Acc, typename Src, typename Epi, typename Fin = NoFin>
static void reduce(Common& cm, int tpr, int64_t nrows, const Src& src, const Epi& epi, double* out,
                   const Fin& fin = Fin()) {
  switch (tpr) {
    case 1: reduce_t<1, K, MM, Acc>(cm, (int)nrows, src, epi, out, fin); break;
    case 2: reduce_t<2, K, MM, Acc>(cm, (int)nrows, src, epi, out, fin); break;
    case 4: reduce_t<4, K, MM, Acc>(cm, (int)nrows, src, epi, out, fin); break;
    case 8: reduce_t<8, K, MM, Acc>(cm, (int)nrows, src, epi, out, fin); break;
    case 16: reduce_t<16, K, MM, Acc>(cm, (int)nrows, src, epi, out, fin); break;
    case 32: reduce_t<32, K, MM, Acc>(cm, (int)nrows, src, epi, out, fin); break;
    default: throw Error(HPRQP_E_ARG, "bad threads-per-row");
  }
}

template <typename F>
static void elem(Common& cm, int64_t len, const F& f) {
  if (len <= 0) return;
  const int grid = (int)((len + kBlock - 1) / kBlock);
  launch(cm, k_elementwise<F>, grid, kBlock, (int)len, f);
}

#define HPRQP_BOOL(cond, NAME, ...)   \
  if (cond) {                         \
    constexpr bool NAME = true;       \
    __VA_ARGS__                       \
  } else {                            \
    constexpr bool NAME = false;      \
    __VA_ARGS__                       \
  }

// ---------------------------------------------------------------------------
// Extra epilogues / kernels local to the engine
// ---------------------------------------------------------------------------

// do_restart! (src/algorithm.jl:522-555), n-part: acc = (A' y_bar)_i
template <typename V>
struct EpiRestartN {
  V *x, *w, *ATy, *ATy_bar, *Qw;
  const V *x_bar, *w_bar, *Qw_bar;
  V *last_x, *last_w, *last_ATy, *last_Qw;
  bool has_m, noC;
  template <typename A>
  __device__ __forceinline__ void operator()(int i, A acc) const {
    const V xb = x_bar[i], wb = w_bar[i];
    x[i] = xb;
    w[i] = wb;
    last_x[i] = xb;
    last_w[i] = wb;
    if (has_m) {
      ATy_bar[i] = (V)acc;
      last_ATy[i] = (V)acc;
      ATy[i] = (V)acc;
    }
    if (noC) {
      Qw[i] = Qw_bar[i];
      last_Qw[i] = Qw_bar[i];
    }
  }
};

template <typename D, typename S>
struct CastCopy {
  D* dst;
  const S* src;
  __device__ __forceinline__ void operator()(int i) const { dst[i] = (D)src[i]; }
};

// Golden-section search of unified_golden_Q_diag (src/unified_operations.jl:
// 348-386) on one CTA: f(x) = a x + b/x + x^2 sum_i c_i d_i / (1 + x Q_i).
template <typename V>
__global__ void __launch_bounds__(1024) k_golden_diag(int n, double a, double b, const V* Q,
                                                      const V* cc, const V* dd, double lo, double hi,
                                                      double tol, int maxiter, double* out) {
  __shared__ double sh[32];
  auto f = [&](double x) {
    double s = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x)
      s += (double)cc[i] * ((double)dd[i] / (1.0 + x * (double)Q[i]));
    for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x < 32) {
      t = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : 0.0;
      for (int off = 16; off > 0; off >>= 1) t += __shfl_down_sync(0xffffffffu, t, off);
      if (threadIdx.x == 0) sh[0] = t;
    }
    __syncthreads();
    t = sh[0];
    return a * x + b / x + x * x * t;
  };
  const double phi = (sqrt(5.0) - 1.0) / 2.0;
  double x1 = hi - phi * (hi - lo), x2 = lo + phi * (hi - lo);
  double f1 = f(x1), f2 = f(x2);
  int it = 0;
  while (fabs(hi - lo) > tol * fmax(1.0, fabs(lo)) && it < maxiter) {
    if (f1 > f2) {
      lo = x1; x1 = x2; f1 = f2;
      x2 = lo + phi * (hi - lo);
      f2 = f(x2);
    } else {
      hi = x2; x2 = x1; f2 = f1;
      x1 = hi - phi * (hi - lo);
      f1 = f(x1);
    }
    ++it;
  }
  if (threadIdx.x == 0) *out = (f1 < f2) ? x1 : x2;
}

// ---------------------------------------------------------------------------
// Engine: construction and uploads
// ---------------------------------------------------------------------------
template <typename V, typename A>
static V* upload(Common& cm, DeviceMem& mem, const std::vector<double, A>& h, int64_t len) {
  V* d = mem.alloc<V>(len);
  if (len > 0) {
    if constexpr (std::is_same<V, double>::value) {
      cm.to_dev(d, h.data(), sizeof(V) * len);
      HPRQP_CUDA(cudaStreamSynchronize(cm.stream));
    } else {
      std::vector<V> t(len);
#pragma omp parallel for schedule(static) num_threads(host_threads(len))
      for (int64_t i = 0; i < len; ++i) t[i] = (V)h[i];
      cm.to_dev(d, t.data(), sizeof(V) * len);
      HPRQP_CUDA(cudaStreamSynchronize(cm.stream));
    }
  }
  return d;
}

// A vector of the scaled problem: copied (FP64) or cast (FP32) from the
// GPU scaling's device copy when there is one, else uploaded from the host.
template <typename V>
V* Engine<V>::vec_in(const hvec<double>& h, const double* dsrc, int64_t len) {
  if (!dsrc || len <= 0) return upload<V>(cm, mem, h, len);
  V* d = mem.alloc<V>(len);
  if constexpr (std::is_same<V, double>::value)
    HPRQP_CUDA(cudaMemcpyAsync(d, dsrc, sizeof(double) * len, cudaMemcpyDeviceToDevice, cm.stream));
  else
    elem(cm, len, CastCopy<V, double>{d, dsrc});
  return d;
}

template <typename V>
void Engine<V>::upload_csr(const HCsr& h, DCsr<V>& d, int tpr_mode, const DevCsrView* dsrc) {
  d.rows = (int)h.rows;
  d.cols = (int)h.cols;
  d.nnz = h.nnz();
  int* ptr = mem.alloc<int>(h.rows + 1);
  int* col = mem.alloc<int>(d.nnz);
  if (dsrc && dsrc->ptr) {  // the pattern is the host one; the copy is on the device already
    HPRQP_CUDA(cudaMemcpyAsync(ptr, dsrc->ptr, sizeof(int) * (h.rows + 1), cudaMemcpyDeviceToDevice, cm.stream));
    if (d.nnz)
      HPRQP_CUDA(cudaMemcpyAsync(col, dsrc->col, sizeof(int) * d.nnz, cudaMemcpyDeviceToDevice, cm.stream));
  } else {
    cm.to_dev(ptr, h.ptr.data(), sizeof(int) * (h.rows + 1));
    cm.to_dev(col, h.col.data(), sizeof(int) * d.nnz);
  }
  d.ptr = ptr;
  d.col = col;
  d.val = vec_in(h.val, dsrc ? dsrc->val : nullptr, d.nnz);
  d.sell = false;
  d.ell = false;
  if (tpr_mode == 7) {  // SELL-32 requested
    build_sell(h, d);
    d.sell = d.sell_len > 0;
    d.tpr = d.sell ? 1 : 4;
  } else if (tpr_mode == 8) {  // ELL requested
    build_ell(h, d);
    d.ell = d.ell_w > 0;
    d.tpr = d.ell ? 1 : 4;
  } else if (tpr_mode == 9) {  // row split requested
    build_split(h, d);
    d.split = d.npieces > 0;
    d.tpr = 4;
  } else if (tpr_mode == 10) {  // staged column blocks requested
    build_stage(h, d);
    d.stage = d.st_nblk > 0;
    d.tpr = csr_tpr((double)d.nnz / std::max(d.rows, 1));
  } else if (tpr_mode > 0) {
    d.tpr = 1 << std::min(tpr_mode - 1, 5);
  } else {
    // a pattern timed before: only the chosen copy is built
    const bool cached = cm.autotune && cm.sched_cache && h.nnz() > 0;
    const uint64_t key = cached ? pattern_key(h, 0x100 * sizeof(V) + cm.ell_prologue) : 0;
    SchedChoice c{};
    if (cached && sched_lookup(key, c)) {
      if (c.kind == SK_SELL) build_sell(h, d);
      if (c.kind == SK_ELL) build_ell(h, d);
      if (c.kind == SK_SPLIT) build_split(h, d);
      if (c.kind == SK_STAGE) build_stage(h, d);
      d.sell = c.kind == SK_SELL && d.sell_len > 0;
      d.ell = c.kind == SK_ELL && d.ell_w > 0;
      d.split = c.kind == SK_SPLIT && d.npieces > 0;
      d.stage = c.kind == SK_STAGE && d.st_nblk > 0;
      if (d.sell || d.ell || d.split || d.stage || c.kind == SK_CSR) {
        d.tpr = c.tpr;
        return;
      }
    }
    build_sell(h, d);
    build_ell(h, d);
    build_split(h, d);
    // (an ELL copy of width <= 8 is taken untimed: no other copy is needed)
    if (!(cm.ell_prologue > 0 && d.ell_w > 0 && d.ell_w <= 8)) build_stage(h, d);
    d.tpr = autotune(d);
    if (cached)
      sched_store(key, SchedChoice{d.stage ? SK_STAGE : d.split ? SK_SPLIT : d.ell ? SK_ELL : d.sell ? SK_SELL : SK_CSR,
                                   d.tpr});
  }
}

// ELL copy of a CSR matrix: only for short rows (width <= 16) whose padding
// stays within 25% of the nonzeros.
// Scatter of the device CSR into a padded copy: row r's entry k goes to
// base(r) + k * stride (ELL: base = r, stride = rows; SELL-32: base =
// sptr[r / 32] + r % 32, stride = 32).  The padding was zeroed beforehand.
template <typename V>
__global__ void __launch_bounds__(kBlock) k_pad_copy(int rows, const int* __restrict__ ptr, const int* __restrict__ col,
                                                     const V* __restrict__ val, const int* __restrict__ sptr,
                                                     int stride, int* __restrict__ pcol, V* __restrict__ pval) {
  const int r = blockIdx.x * kBlock + threadIdx.x;
  if (r >= rows) return;
  const int64_t base = sptr ? (int64_t)sptr[r >> 5] + (r & 31) : (int64_t)r;
  const int b = ptr[r], e = ptr[r + 1];
  for (int k = b; k < e; ++k) {
    const int64_t j = base + (int64_t)(k - b) * stride;
    pcol[j] = col[k];
    pval[j] = val[k];
  }
}

// ELL copy of a CSR matrix, built on the device from its CSR: only for
// short rows (width <= 16) whose padding stays within 25% of the nonzeros.
template <typename V>
void Engine<V>::build_ell(const HCsr& h, DCsr<V>& d) {
  d.ell_w = 0;
  if (h.rows <= 0 || h.nnz() == 0) return;
  int w = 0;
  for (int64_t r = 0; r < h.rows; ++r) w = std::max(w, h.ptr[r + 1] - h.ptr[r]);
  const int64_t total = (int64_t)w * h.rows;
  if (w > 16 || total > (int64_t)(1.25 * h.nnz()) + 64 || total > INT32_MAX) return;
  int* dc = mem.alloc<int>(total);
  V* dv = mem.alloc<V>(total);
  HPRQP_CUDA(cudaMemsetAsync(dc, 0, sizeof(int) * total, cm.stream));
  HPRQP_CUDA(cudaMemsetAsync(dv, 0, sizeof(V) * total, cm.stream));
  k_pad_copy<V><<<(int)((h.rows + kBlock - 1) / kBlock), kBlock, 0, cm.stream>>>((int)h.rows, d.ptr, d.col, d.val,
                                                                                  nullptr, (int)h.rows, dc, dv);
  HPRQP_LAUNCH_CHECK();
  d.ecol = dc;
  d.evalv = dv;
  d.ell_w = w;
}

// Row-split schedule (DCsr::split) for a matrix with a heavy tail of long
// rows: built when the longest row exceeds 1,024 entries and 8x the mean.
// Rows longer than T = max(1024, longest / 64) (a multiple of 32) are cut
// into pieces of T entries; pieces are ordered by length, longest first.
template <typename V>
void Engine<V>::build_split(const HCsr& h, DCsr<V>& d) {
  d.npieces = 0;
  if (h.rows <= 0 || h.nnz() == 0) return;
  int64_t maxlen = 0;
  for (int64_t r = 0; r < h.rows; ++r) maxlen = std::max<int64_t>(maxlen, h.ptr[r + 1] - h.ptr[r]);
  const double avg = (double)h.nnz() / (double)h.rows;
  if (maxlen <= 1024 || (double)maxlen <= 8.0 * avg) return;
  int64_t T = std::max<int64_t>(1024, (maxlen + 63) / 64);
  T = (T + 31) / 32 * 32;
  std::vector<int4> pcs;
  std::vector<int2> srow;
  int64_t slots = 0;
  for (int64_t r = 0; r < h.rows; ++r) {
    const int b = h.ptr[r], e = h.ptr[r + 1];
    if (e - b <= T) {
      pcs.push_back(make_int4((int)r, b, e, -1));
      continue;
    }
    const int np = (int)((e - b + T - 1) / T);
    const int s = (int)srow.size();
    srow.push_back(make_int2((int)slots, np));
    for (int j = 0; j < np; ++j) pcs.push_back(make_int4((int)r, b + (int)(j * T), (int)std::min<int64_t>(e, b + (j + 1) * T), s));
    slots += np;
  }
  std::stable_sort(pcs.begin(), pcs.end(), [](const int4& a, const int4& b) { return (a.z - a.y) > (b.z - b.y); });
  int4* dp = mem.alloc<int4>(pcs.size());
  int2* ds = mem.alloc<int2>(std::max<size_t>(srow.size(), 1));
  double* part = mem.alloc<double>(std::max<int64_t>(slots, 1));
  unsigned* cnt = mem.alloc<unsigned>(std::max<size_t>(srow.size(), 1));
  cm.to_dev(dp, pcs.data(), sizeof(int4) * pcs.size());
  cm.to_dev(ds, srow.data(), sizeof(int2) * srow.size());
  HPRQP_CUDA(cudaMemsetAsync(cnt, 0, sizeof(unsigned) * std::max<size_t>(srow.size(), 1), cm.stream));
  HPRQP_CUDA(cudaStreamSynchronize(cm.stream));  // host staging vectors go out of scope
  d.pieces = dp;
  d.srow = ds;
  d.spart = part;
  d.scnt = cnt;
  d.npieces = (int)pcs.size();
  d.split_T = (int)T;
}

// Set-up of the staged copy.  Chunks of row r in block b: the entries of
// row r whose column lies in [b bw, (b + 1) bw), 8 per chunk, at least one
// chunk per row.  One thread per (row, block).
__global__ void __launch_bounds__(kBlock) k_stage_count(int rows, int nblk, int bw, const int* __restrict__ ptr,
                                                        const int* __restrict__ col, int* __restrict__ chunks) {
  const int64_t t = (int64_t)blockIdx.x * kBlock + threadIdx.x;
  if (t >= (int64_t)rows * nblk) return;
  const int r = (int)(t % rows), b = (int)(t / rows);
  const int lo = b * bw, hi = lo + bw;
  int n = 0;
  for (int k = ptr[r]; k < ptr[r + 1]; ++k) n += (col[k] >= lo && col[k] < hi) ? 1 : 0;
  chunks[t] = n > 0 ? (n + 7) / 8 : 1;
}

// Fill: row r's entries of block b, in CSR order, from chunk cptr[b][r]
// on (the copy was zeroed first, so the padding is column 0, value 0).
// Entry e of chunk c = 32 g + l: its column at 8 c + e; its value in the
// lane-interleaved slices of warp tile g (slice e / S of lane l, S values
// of 16 bytes each).
template <typename V>
__global__ void __launch_bounds__(kBlock) k_stage_fill(int rows, int nblk, int bw, const int* __restrict__ ptr,
                                                       const int* __restrict__ col, const V* __restrict__ val,
                                                       const int* __restrict__ cptr, uint16_t* __restrict__ scol,
                                                       V* __restrict__ sval) {
  constexpr int S = 16 / (int)sizeof(V);
  const int64_t t = (int64_t)blockIdx.x * kBlock + threadIdx.x;
  if (t >= (int64_t)rows * nblk) return;
  const int r = (int)(t % rows), b = (int)(t / rows);
  const int lo = b * bw, hi = lo + bw;
  int64_t j = (int64_t)cptr[(int64_t)b * (rows + 1) + r] * 8;
  for (int k = ptr[r]; k < ptr[r + 1]; ++k) {
    const int c = col[k];
    if (c >= lo && c < hi) {
      const int64_t ch = j >> 3, g = ch >> 5, l = ch & 31;
      const int e = (int)(j & 7);
      scol[j] = (uint16_t)(c - lo);
      sval[((g * (8 / S) + e / S) * 32 + l) * S + e % S] = val[k];
      ++j;
    }
  }
}

// Staged copy (DCsr::stage) of a CSR matrix whose products are bound by their
// gathers: built for rows of at least 16 entries on average, at least 65,536
// entries, and an input vector of at most 32 column blocks of kStageSmem
// bytes.  Counts on the device; slots, windows, tiles and the CTA split on
// the host; the scatter on the device.
template <typename V>
void Engine<V>::build_stage(const HCsr& h, DCsr<V>& d) {
  d.st_nblk = 0;
  if (h.rows <= 0 || h.cols <= 0 || h.nnz() < 65536) return;
  if ((double)h.nnz() / (double)h.rows < 16.0) return;
  const int64_t per = kStageSmem / (int64_t)sizeof(V);
  const int64_t nblk = (h.cols + per - 1) / per;
  if (nblk > 32 || nblk >= cm.num_sms) return;
  // block width a multiple of 8 (16-byte staging loads); at most
  // kStageSmem / 4 = 51,200 columns, so block-local columns fit 16 bits
  const int bw = (int)(((h.cols + nblk - 1) / nblk + 7) / 8 * 8);
  const int rows = (int)h.rows;
  const int nb = (int)nblk;
  const int64_t pairs = (int64_t)rows * nb;
  int* dch = mem.alloc<int>(pairs);
  const int g1 = (int)((pairs + kBlock - 1) / kBlock);
  k_stage_count<<<g1, kBlock, 0, cm.stream>>>(rows, nb, bw, d.ptr, d.col, dch);
  HPRQP_LAUNCH_CHECK();
  std::vector<int> ch((size_t)pairs);
  cm.to_host(ch.data(), dch, sizeof(int) * (size_t)pairs);
  HPRQP_CUDA(cudaStreamSynchronize(cm.stream));
  // chunk offsets, block-major
  const size_t R1 = (size_t)rows + 1;
  std::vector<int> cptr((size_t)nb * R1), srow((size_t)nb * R1);
  int64_t tot = 0;
  std::vector<double> bcost(nb, 0.0);  // chunks + 1 a row (its slot and epilogue)
  for (int b = 0; b < nb; ++b) {
    const int64_t b0 = tot;
    for (int r = 0; r < rows; ++r) {
      cptr[(size_t)b * R1 + r] = (int)tot;
      tot += ch[(size_t)b * rows + r];
      if (tot > INT32_MAX / 8) return;
    }
    cptr[(size_t)b * R1 + rows] = (int)tot;
    bcost[b] = (double)(tot - b0) + rows;
  }
  // one CTA per SM; block b gets a share of them by its cost (at least one,
  // at most one per row)
  const int G = cm.num_sms;
  double total = 0;
  for (double c : bcost) total += c;
  std::vector<int> kb(nb);
  int sum = 0;
  for (int b = 0; b < nb; ++b) {
    kb[b] = std::max(1, std::min(rows, (int)std::floor(G * bcost[b] / total)));
    sum += kb[b];
  }
  while (sum < G) {  // the block with the most cost per CTA gets one more
    int best = -1;
    double bv = 0;
    for (int b = 0; b < nb; ++b)
      if (kb[b] < rows && bcost[b] / kb[b] > bv) { bv = bcost[b] / kb[b]; best = b; }
    if (best < 0) break;
    ++kb[best];
    ++sum;
  }
  while (sum > G) {  // the block with the least cost per CTA gives one back
    int best = -1;
    double bv = 1e300;
    for (int b = 0; b < nb; ++b)
      if (kb[b] > 1 && bcost[b] / kb[b] < bv) { bv = bcost[b] / kb[b]; best = b; }
    if (best < 0) return;
    --kb[best];
    --sum;
  }
  // Each block's rows cut into kb[b] runs of about equal cost, each run into
  // tiles of whole rows with at most kStageSlots slots.  A tile's chunks are
  // cut into 32-chunk warp tiles from its first chunk on, and a tile starts at
  // a whole warp tile of the copy (pc = a row's first chunk there); a row has
  // one slot per warp tile it touches (its segments), numbered in row order.
  std::vector<int> pc((size_t)nb * R1);
  std::vector<int2> wt;
  std::vector<int4> tile, item;
  std::vector<unsigned> heads;
  std::vector<int> first;
  for (int b = 0; b < nb; ++b) {
    const int* cb = ch.data() + (size_t)b * rows;
    const int* pb = cptr.data() + (size_t)b * R1;
    int* sb = srow.data() + (size_t)b * R1;
    int* pcb = pc.data() + (size_t)b * R1;
    int64_t slot = 0;
    int r = 0;
    double acc = 0;
    for (int i = 0; i < kb[b]; ++i) {
      const double end = bcost[b] * (double)(i + 1) / kb[b];
      int re = r;
      if (i == kb[b] - 1) {
        re = rows;
      } else {
        while (re < rows && (re == r || acc + 0.5 * (cb[re] + 1) <= end)) acc += cb[re++] + 1;
      }
      const int t0 = (int)tile.size();
      int q = r;
      while (q < re) {  // one tile from row q
        const int r0 = q;
        int64_t slots = 0;
        while (q < re) {  // the warp tiles row q touches, from the tile's first chunk
          const int o = pb[q] - pb[r0];
          const int64_t touch = (o + cb[q] - 1) / 32 - o / 32 + 1;
          if (slots + touch > kStageSlots) break;
          slots += touch;
          ++q;
        }
        if (q == r0) return;  // one row with more slots than a tile holds
        const int nwt = (pb[q] - pb[r0] + 31) / 32;
        heads.assign(nwt, 0u);
        first.assign(nwt, -1);
        if ((int64_t)(wt.size() + nwt) * 32 > INT32_MAX / 8) return;
        for (int rr = r0; rr < q; ++rr) {
          const int o = pb[rr] - pb[r0];
          sb[rr] = (int)slot;
          pcb[rr] = (int)(32 * wt.size()) + o;
          for (int w = o / 32; w <= (o + cb[rr] - 1) / 32; ++w) {
            heads[w] |= 1u << (std::max(o, 32 * w) - 32 * w);
            if (first[w] < 0) first[w] = (int)slot;
            ++slot;
          }
        }
        if (slot > INT32_MAX / 2) return;
        tile.push_back(make_int4((int)wt.size(), pb[q] - pb[r0], r0, q));
        for (int w = 0; w < nwt; ++w) wt.push_back(make_int2(first[w], (int)heads[w]));
      }
      item.push_back(make_int4(b, t0, (int)tile.size(), 0));
      r = re;
    }
    sb[rows] = (int)slot;
  }
  tot = 32 * (int64_t)wt.size();  // chunks of the copy, the tiles' tails padded
  int* dcp = mem.alloc<int>((int64_t)pc.size());
  int* dsr = mem.alloc<int>((int64_t)srow.size());
  int2* dwt = mem.alloc<int2>((int64_t)wt.size());
  int4* dtile = mem.alloc<int4>((int64_t)tile.size());
  int4* ditem = mem.alloc<int4>((int64_t)item.size());
  uint16_t* scol = mem.alloc<uint16_t>(tot * 8);
  V* sval = mem.alloc<V>(tot * 8);
  if ((reinterpret_cast<uintptr_t>(scol) | reinterpret_cast<uintptr_t>(sval)) & 15u) return;  // 16-byte chunk loads
  cm.to_dev(dcp, pc.data(), sizeof(int) * pc.size());
  cm.to_dev(dsr, srow.data(), sizeof(int) * srow.size());
  cm.to_dev(dwt, wt.data(), sizeof(int2) * wt.size());
  cm.to_dev(dtile, tile.data(), sizeof(int4) * tile.size());
  cm.to_dev(ditem, item.data(), sizeof(int4) * item.size());
  HPRQP_CUDA(cudaMemsetAsync(scol, 0, sizeof(uint16_t) * (size_t)tot * 8, cm.stream));
  HPRQP_CUDA(cudaMemsetAsync(sval, 0, sizeof(V) * (size_t)tot * 8, cm.stream));
  k_stage_fill<V><<<g1, kBlock, 0, cm.stream>>>(rows, nb, bw, d.ptr, d.col, d.val, dcp, scol, sval);
  HPRQP_LAUNCH_CHECK();
  if (nb > 1) {
    d.st_part = mem.alloc<double>(pairs);
    unsigned* cnt = mem.alloc<unsigned>(rows);
    HPRQP_CUDA(cudaMemsetAsync(cnt, 0, sizeof(unsigned) * rows, cm.stream));
    d.st_cnt = cnt;
  }
  HPRQP_CUDA(cudaStreamSynchronize(cm.stream));  // host staging vectors go out of scope
  d.st_col = scol;
  d.st_val = sval;
  d.st_wt = dwt;
  d.st_tile = dtile;
  d.st_item = ditem;
  d.st_cptr = dcp;
  d.st_srow = dsr;
  d.st_chunks = tot;
  d.st_nwt = (int64_t)wt.size();
  d.st_ntile = (int)tile.size();
  d.st_grid = (int)item.size();
  d.st_bw = bw;
  d.st_nblk = nb;
}

// SELL-32 copy of a CSR matrix, built on the device from its CSR; skipped
// when padding would exceed 50%.
template <typename V>
void Engine<V>::build_sell(const HCsr& h, DCsr<V>& d) {
  d.sell_len = 0;
  if (h.rows <= 0 || h.nnz() == 0) return;
  const int64_t ns = (h.rows + 31) / 32;
  std::vector<int> sptr(ns + 1, 0);
  for (int64_t sl = 0; sl < ns; ++sl) {
    int w = 0;
    for (int64_t r = sl * 32; r < std::min<int64_t>(h.rows, sl * 32 + 32); ++r) w = std::max(w, h.ptr[r + 1] - h.ptr[r]);
    sptr[sl + 1] = sptr[sl] + 32 * w;
  }
  const int64_t total = sptr[ns];
  if (total > (int64_t)(1.5 * h.nnz()) + 64 || total > INT32_MAX) return;
  int* dsp = mem.alloc<int>(ns + 1);
  int* dsc = mem.alloc<int>(total);
  V* dsv = mem.alloc<V>(total);
  cm.to_dev(dsp, sptr.data(), sizeof(int) * (ns + 1));
  HPRQP_CUDA(cudaMemsetAsync(dsc, 0, sizeof(int) * total, cm.stream));
  HPRQP_CUDA(cudaMemsetAsync(dsv, 0, sizeof(V) * total, cm.stream));
  k_pad_copy<V><<<(int)((h.rows + kBlock - 1) / kBlock), kBlock, 0, cm.stream>>>((int)h.rows, d.ptr, d.col, d.val,
                                                                                  dsp, 32, dsc, dsv);
  HPRQP_LAUNCH_CHECK();
  HPRQP_CUDA(cudaStreamSynchronize(cm.stream));  // sptr staging buffer
  d.sptr = dsp;
  d.scol = dsc;
  d.sval = dsv;
  d.sell_len = total;
}

template <typename V>
template <typename Epi>
void Engine<V>::mat_rows(const DCsr<V>& M, const V* xin, const Epi& e) {
  if (M.stage) {
    const StageView<V> sv{(int)M.rows, (int)M.cols, M.st_bw, M.st_nblk, M.st_col, M.st_val, M.st_wt,
                          M.st_tile, M.st_item, M.st_srow, M.st_part, M.st_cnt};
    launch_smem(cm, k_stage_pass<V, V, V, Epi>, M.st_grid, stage_block<V>(),
                (size_t)kStageSlots * sizeof(V) + (size_t)M.st_bw * sizeof(V), sv, xin, e);
  } else if (M.split) {
    const int grid = (int)(((int64_t)M.npieces * 32 + kBlock - 1) / kBlock);
    launch(cm, k_split_pass<V, V, V, Epi>, grid, kBlock, M.npieces, M.pieces, M.ptr, M.col, M.val, xin, M.srow,
           M.split_T, M.spart, M.scnt, e);
  } else if (M.ell && M.ell_w <= 8 && cm.ell_prologue > 0 && M.rows > 0) {
    const int grid = (int)((M.rows + kBlock - 1) / kBlock);
    launch(cm, k_ell_pass<8, V, V, V, Epi>, grid, kBlock, (int)M.rows,
           EllSrc<V, V>{M.ecol, M.evalv, xin, (int)M.rows, M.ell_w}, e, cm.ell_prologue >= 2 ? 1 : 0);
  } else if (M.ell) rows<V>(cm, 1, M.rows, EllSrc<V, V>{M.ecol, M.evalv, xin, M.rows, M.ell_w}, e);
  else if (M.sell) rows<V>(cm, 1, M.rows, SellSrc<V, V>{M.sptr, M.ptr, M.scol, M.sval, xin}, e);
  else rows<V>(cm, M.tpr, M.rows, CsrSrc<V, V>{M.ptr, M.col, M.val, xin}, e);
}

// Fused product + reduction on M's format (FP64 accumulation).
// (The input vector may be wider than the matrix values: the Gram chain
// keeps its FP64 state under an FP32 Gram matrix.)
template <int K, unsigned MM, typename V, typename X, typename Epi, typename Fin = NoFin>
static void mat_reduce(Common& cm, const DCsr<V>& M, const X* xin, const Epi& e, double* out, const Fin& fin = Fin()) {
  // An ELL copy serves the plain passes; the reductions measured faster on
  // SELL-32 or CSR (the ELL reduction's rows in flight cost registers and
  // occupancy), except when HPRQP_POWER_ELL=1 asks for it
  if (M.ell && cm.pow_prefer_ell) {  // 4 rows per thread in flight
    const int grid = reduce_grid(M.rows, 1, cm.reduce_cap);
    launch(cm, k_ell_reduce<4, K, MM, double, V, X, Epi, Fin>, grid, kBlock, M.rows,
           EllSrc<V, X>{M.ecol, M.evalv, xin, M.rows, M.ell_w}, e, cm.rws, out, fin);
    return;
  }
  if (M.sell || (M.ell && M.sell_len > 0))
    reduce<K, MM, double>(cm, 1, M.rows, SellSrc<V, X>{M.sptr, M.ptr, M.scol, M.sval, xin}, e, out, fin);
  else reduce<K, MM, double>(cm, M.tpr, M.rows, CsrSrc<V, X>{M.ptr, M.col, M.val, xin}, e, out, fin);
}

// CTAs of a partials-only pass over M (the fold needs the count)
template <typename V>
static int partials_grid(const Common& cm, const DCsr<V>& M) {
  const bool sell = M.sell || (M.ell && M.sell_len > 0);
  return reduce_grid(M.rows, sell ? 1 : M.tpr, cm.reduce_cap);
}

// Fused product + per-CTA sums, no fold (the power steps of a chunk)
template <int K, typename V, typename X, typename Epi>
static void mat_partials(Common& cm, const DCsr<V>& M, const X* xin, const Epi& e, double* partials) {
  const int grid = partials_grid(cm, M);
  if (M.sell || (M.ell && M.sell_len > 0)) {
    if (cm.ell_prologue > 0 && cm.pow_rows_preloaded == 1)  // the first row's matrix entries before the wait
      launch(cm, k_sell_partials<1, 8, K, double, V, X, Epi>, grid, kBlock, M.rows,
             SellSrc<V, X>{M.sptr, M.ptr, M.scol, M.sval, xin}, e, partials);
    else if (cm.ell_prologue > 0)  // the first 2 rows' per thread
      launch(cm, k_sell_partials<2, 8, K, double, V, X, Epi>, grid, kBlock, M.rows,
             SellSrc<V, X>{M.sptr, M.ptr, M.scol, M.sval, xin}, e, partials);
    else
      launch(cm, k_row_partials<1, K, double, SellSrc<V, X>, Epi>, grid, kBlock, M.rows,
             SellSrc<V, X>{M.sptr, M.ptr, M.scol, M.sval, xin}, e, partials);
    return;
  }
  switch (M.tpr) {
#define HPRQP_PARTIALS(T)                                                                                      \
  case T:                                                                                                      \
    launch(cm, k_row_partials<T, K, double, CsrSrc<V, X>, Epi>, grid, kBlock, M.rows,                          \
           CsrSrc<V, X>{M.ptr, M.col, M.val, xin}, e, partials);                                               \
    break;
    HPRQP_PARTIALS(1) HPRQP_PARTIALS(2) HPRQP_PARTIALS(4) HPRQP_PARTIALS(8) HPRQP_PARTIALS(16) HPRQP_PARTIALS(32)
#undef HPRQP_PARTIALS
    default: throw Error(HPRQP_E_ARG, "bad threads-per-row");
  }
}

// Row-schedule autotuner: time the plain product for each threads-per-row
// candidate on this matrix and keep the fastest (replaces the reference's
// cuSPARSE-vs-inline micro-benchmark, src/algorithm.jl:1557-1752).
template <typename V>
int Engine<V>::autotune(DCsr<V>& d) {
  if (d.rows <= 0 || d.nnz == 0) return 1;
  const double avg = (double)d.nnz / d.rows;
  if (!cm.autotune) {  // fixed rule: ELL, else staged, else SELL-32, else threads per row by mean row length
    d.ell = d.ell_w > 0;
    d.stage = !d.ell && d.st_nblk > 0;
    d.sell = !d.ell && !d.stage && d.sell_len > 0;
    d.split = !d.ell && !d.stage && !d.sell && d.npieces > 0;
    if (d.ell || d.sell) return 1;
    if (d.split) return 32;
    return csr_tpr(avg);
  }
  // An ELL copy of width <= 8 runs the passes with its loads before the wait
  // on the previous pass (k_ell_pass).  Timing products alone cannot see that
  // overlap (repeated products run from L2, one after another), and inside the
  // iteration it wins: 700x700 grid, FP32 iteration 28.6 us with ELL against
  // 31.8 us with the schedules timed products chose.  So it is taken untimed.
  if (cm.ell_prologue > 0 && d.ell_w > 0 && d.ell_w <= 8) {
    d.ell = true;
    d.sell = false;
    d.split = false;
    d.stage = false;
    return 1;
  }
  cudaEvent_t e0, e1;
  HPRQP_CUDA(cudaEventCreate(&e0));
  HPRQP_CUDA(cudaEventCreate(&e1));
  float best = 1e30f;
  int best_t = 4;
  bool best_sell = false, best_ell = false, best_split = false, best_stage = false;
  // candidate -1 = SELL-32, -2 = ELL (one thread per row each), -3 = row
  // split, -4 = staged column blocks; each timed as the best of 3 rounds of 4
  // back-to-back products, so a noisy round cannot decide.
  for (int t : {-4, -3, -2, -1, 1, 2, 4, 8, 16, 32}) {
    if (t == -4 && d.st_nblk == 0) continue;
    if (t == -3 && d.npieces == 0) continue;
    if (t == -2 && d.ell_w == 0) continue;
    if (t == -1 && d.sell_len == 0) continue;
    if (t == 1 && avg > 12) continue;
    if (t == 32 && avg < 8) continue;
    d.stage = (t == -4);
    d.split = (t == -3);
    d.ell = (t == -2);
    d.sell = (t == -1);
    // (the reductions of a split matrix run on CSR with 32 lanes per row, of
    // a staged one with the fixed rule's lanes)
    d.tpr = t == -4 ? csr_tpr(avg) : t == -3 ? 32 : t < 0 ? 1 : t;
    spmv(d, pz, pt);
    float tbest = 1e30f;
    for (int round = 0; round < 3; ++round) {
      HPRQP_CUDA(cudaEventRecord(e0, cm.stream));
      for (int r = 0; r < 4; ++r) spmv(d, pz, pt);
      HPRQP_CUDA(cudaEventRecord(e1, cm.stream));
      HPRQP_CUDA(cudaEventSynchronize(e1));
      float ms = 0;
      HPRQP_CUDA(cudaEventElapsedTime(&ms, e0, e1));
      tbest = std::min(tbest, ms);
    }
    if (tbest < best) {
      best = tbest;
      best_t = d.tpr;
      best_sell = d.sell;
      best_ell = d.ell;
      best_split = d.split;
      best_stage = d.stage;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  d.sell = best_sell;
  d.ell = best_ell;
  d.split = best_split;
  d.stage = best_stage;
  return best_t;
}


// Values of the Gram matrix G = A'A: G_pj = sum over the rows r of A with
// entries in both columns p and j of A_rp A_rj, in increasing r (a merge of
// rows p and j of A'), FP64 sums rounded once to V.  G_jp runs the same
// merge with the factors swapped, so G is exactly symmetric.  Row p's entry
// t goes to out[base(p) + t * stride] (CSR: base = ptr[p], stride 1; ELL:
// base = p, stride = rows; SELL-32: base = sptr[p / 32] + p % 32, stride 32).
template <typename V>
__global__ void __launch_bounds__(kBlock) k_gram_vals(int rows, const int* __restrict__ tptr,
                                                      const int* __restrict__ tcol, const V* __restrict__ tval,
                                                      const int* __restrict__ gptr, const int* __restrict__ gcol,
                                                      int layout, const int* __restrict__ sptr, V* __restrict__ out) {
  const int p = blockIdx.x * kBlock + threadIdx.x;
  if (p >= rows) return;
  const int b1 = tptr[p], e1 = tptr[p + 1];
  const int gb = gptr[p], ge = gptr[p + 1];
  const int64_t base = layout == 0 ? (int64_t)gb : layout == 1 ? (int64_t)p : (int64_t)sptr[p >> 5] + (p & 31);
  const int64_t stride = layout == 0 ? 1 : layout == 1 ? (int64_t)rows : 32;
  for (int k = gb; k < ge; ++k) {
    const int j = gcol[k];
    int a = b1, b = tptr[j];
    const int e2 = tptr[j + 1];
    double acc = 0.0;
    while (a < e1 && b < e2) {
      const int ra = tcol[a], rb = tcol[b];
      if (ra == rb) {
        acc += (double)tval[a] * (double)tval[b];
        ++a;
        ++b;
      } else if (ra < rb) {
        ++a;
      } else {
        ++b;
      }
    }
    out[base + (int64_t)(k - gb) * stride] = (V)acc;
  }
}

// G only feeds the power step (a fused product + two dot products + the
// last CTA's fold), so its schedule is chosen by timing that step itself:
// SELL-32 and CSR with 1, 2, 4 or 8 threads per row, each the best of 3
// rounds of 8 chained steps on a unit start.
template <typename V>
template <typename Step>
void Engine<V>::tune_reduce(DCsr<V>& M, Step step, uint64_t key) {
  SchedChoice c{};
  if (key && sched_lookup(key, c)) {
    M.ell = false;
    M.sell = c.kind == SK_SELL && M.sell_len > 0;
    M.tpr = c.tpr;
    return;
  }
  cudaEvent_t e0, e1;
  HPRQP_CUDA(cudaEventCreate(&e0));
  HPRQP_CUDA(cudaEventCreate(&e1));
  float best = 1e30f;
  int best_t = 1;
  bool best_sell = false;
  const double avg = (double)M.nnz / std::max(M.rows, 1);
  M.ell = false;
  for (int t : {-1, 1, 2, 4, 8}) {
    if (t == -1 && M.sell_len == 0) continue;
    if (t == 8 && avg < 8) continue;
    M.sell = t == -1;
    M.tpr = t < 0 ? 1 : t;
    for (int k = 0; k < 2; ++k) step(k);
    float tb = 1e30f;
    for (int round = 0; round < 3; ++round) {
      HPRQP_CUDA(cudaEventRecord(e0, cm.stream));
      for (int k = 0; k < 8; ++k) step(k);
      HPRQP_CUDA(cudaEventRecord(e1, cm.stream));
      HPRQP_CUDA(cudaEventSynchronize(e1));
      float ms = 0;
      HPRQP_CUDA(cudaEventElapsedTime(&ms, e0, e1));
      tb = std::min(tb, ms);
    }
    if (tb < best) {
      best = tb;
      best_t = M.tpr;
      best_sell = M.sell;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  M.sell = best_sell;
  M.tpr = best_t;
  if (key) sched_store(key, SchedChoice{best_sell ? SK_SELL : SK_CSR, best_t});
}

template <typename V>
void Engine<V>::autotune_gram(uint64_t key) {
  double* inv = cm.d_scal + S_POW + 5;
  double* lg = cm.d_scal + S_POWLOG;
  double* u0 = gu0;
  const int64_t nn = n;
  elem(cm, nn, [=] __device__(int i) { u0[i] = 1.0; });
  elem(cm, 1, [=] __device__(int) { *inv = 1.0; });
  tune_reduce(G, [&](int k) {
    const double* uc = (k & 1) ? gu1 : gu0;
    double* un = (k & 1) ? gu0 : gu1;
    mat_reduce<2, 0u>(cm, G, uc, EpiGramPower<double>{uc, un, inv}, cm.d_scal + S_POW + 6,
                      GramPowerFin{lg, k & 31, inv});
  }, key);
}

// What the power method needs beyond the iteration's matrices (the Gram
// matrix, the power schedule of Q): built once, by the constructor of the
// engine that runs the power method, or on the first power method of the
// other engine (a handle prepared for one precision and then solved in the
// other).
template <typename V>
void Engine<V>::power_setup(const Prepared& pp, int tpr_A, int tpr_Q) {
  if (power_ready) return;
  power_ready = true;
  build_gram(pp, tpr_A);
  if (tpr_Q <= 0)
    autotune_power_Q(cm.sched_cache && pp.Qpat().nnz() > 0 ? pattern_key(pp.Qpat(), 0x300 + sizeof(V)) : 0);
}

// The sparse Q's power step runs on its own copy of Q's schedule, chosen by
// timing that step (Q's own schedule is chosen for the iteration's passes).
template <typename V>
void Engine<V>::autotune_power_Q(uint64_t key) {
  Qp = Q;
  if (!has_Q_sparse || Q.nnz == 0 || !cm.autotune || cm.pow_prefer_ell) return;
  double* inv = cm.d_scal + S_POW_Q + 5;
  double* zz = cm.d_scal + S_POW_Q + 4;
  double* lg = cm.d_scal + S_POWLOG_Q;
  V* z0 = pz2;
  const int64_t nn = n;
  elem(cm, nn, [=] __device__(int i) { z0[i] = (V)1.0; });
  elem(cm, 1, [=] __device__(int) {
    *inv = 1.0;
    *zz = 1.0;
  });
  tune_reduce(Qp, [&](int k) {
    V* zc = (k & 1) ? pq2 : pz2;
    V* zn = (k & 1) ? pz2 : pq2;
    mat_reduce<3, 0u>(cm, Qp, zc, EpiPowerFused<V>{zc, zn, zz, true, inv}, cm.d_scal + S_POW_Q + 1,
                      PowerFin{lg, k & 31, inv});
  }, key);
}

// Values of G into the format its products use (the padding of ELL / SELL
// copies stays zero from their construction)
template <typename V>
void Engine<V>::gram_values() {
  const int layout = G.ell ? 1 : G.sell ? 2 : 0;
  V* out = const_cast<V*>(G.ell ? G.evalv : G.sell ? G.sval : G.val);
  k_gram_vals<V><<<(G.rows + kBlock - 1) / kBlock, kBlock, 0, cm.stream>>>(G.rows, AT.ptr, AT.col, AT.val, G.ptr,
                                                                            G.col, layout, G.sptr, out);
  HPRQP_LAUNCH_CHECK();
  cm.launches++;
}

// The A A' chain's Gram matrix: pattern on the host (gram_pattern), values on
// the device, then the ELL / SELL-32 copies and the row-schedule autotuner
// as for the problem's own matrices.  Skipped (the chain then runs its two
// products per step) for LASSO and QAP operators, when disabled, when the
// product work exceeds its bound, or, in the automatic mode, when A'A has
// more than 3 nnz(A) entries.
template <typename V>
void Engine<V>::build_gram(const Prepared& pp, int tpr_mode) {
  gram = false;
  if (m <= 0 || is_op || is_lasso || cm.pow_gram == 0 || pp.Apat().nnz() == 0) return;
  const bool force = cm.pow_gram == 1;
  const int64_t nnzA = pp.Apat().nnz();
  const double t0 = wall_s();
  HCsr h;
  if (!gram_pattern(pp.Apat(), pp.ATpat(), (force ? 64 : 6) * nnzA, h)) return;
  const double t_pat = wall_s();
  if (!force && h.nnz() > 3 * nnzA) return;
  G = DCsr<V>();
  G.rows = G.cols = (int)n;
  G.nnz = h.nnz();
  int* ptr = mem.alloc<int>(n + 1);
  int* col = mem.alloc<int>(G.nnz);
  cm.to_dev(ptr, h.ptr.data(), sizeof(int) * (n + 1));
  cm.to_dev(col, h.col.data(), sizeof(int) * G.nnz);
  G.ptr = ptr;
  G.col = col;
  G.val = mem.alloc<V>(G.nnz);
  gu0 = mem.alloc<double>(n);
  gu1 = mem.alloc<double>(n);
  gram_values();  // CSR values, copied into the padded formats next
  build_sell(h, G);
  if (cm.pow_prefer_ell) build_ell(h, G);  // G only feeds reductions, which run on SELL-32 or CSR
  if (tpr_mode == 7 || tpr_mode == 8) {  // A's schedule pinned by the caller: G follows it (SELL for ELL)
    G.sell = G.sell_len > 0;
    G.tpr = 1;
  } else if (tpr_mode > 0 && tpr_mode < 7) {
    G.tpr = 1 << std::min(tpr_mode - 1, 5);
  } else if (cm.pow_prefer_ell && G.ell_w > 0) {  // HPRQP_POWER_ELL=1
    G.ell = true;
    G.tpr = 1;
  } else if (!cm.autotune) {
    G.sell = G.sell_len > 0;
    G.tpr = 1;
  } else {
    autotune_gram(cm.sched_cache ? pattern_key(h, 0x200 + sizeof(V)) : 0);
  }
  HPRQP_CUDA(cudaStreamSynchronize(cm.stream));
  gram = true;
  if (const char* tv = std::getenv("HPRQP_TIMING"))
    if (tv[0] == '1')
      std::fprintf(stderr, "[hprqp] Gram matrix A'A: %lld entries (A: %lld), pattern %.3f s, total %.3f s, %s\n",
                   (long long)G.nnz, (long long)nnzA, t_pat - t0, wall_s() - t0,
                   G.ell ? "ELL" : G.sell ? "SELL-32" : "CSR");
}

template <typename V>
Engine<V>::Engine(Common& c_, const HostProblem& hp, const Prepared& pp, int path_, int tpr_Q, int tpr_A,
                  bool power_engine)
    : cm(c_) {
  const double t0 = wall_s();
  n = hp.n;
  m = hp.m;
  path = path_;
  Q_is_diag = pp.Q_is_diag;
  is_qap = hp.Q_kind == HPRQP_Q_QAP;
  is_custom = hp.Q_kind == HPRQP_Q_CUSTOM;
  is_op = is_qap || is_custom;
  is_lasso = hp.Q_kind == HPRQP_Q_LASSO;
  has_Q_sparse = hp.Q_kind == HPRQP_Q_SPARSE;
  b_scale = pp.b_scale;
  c_scale = pp.c_scale;
  norm_b_org = pp.norm_b_org;
  norm_c_org = pp.norm_c_org;
  lasso_lam = hp.lambda;
  const int64_t mx = std::max(std::max(n, m), is_lasso ? hp.L.rows : (int64_t)0);
  V** nv[] = {&x, &x_hat, &x_bar, &dx, &w, &w_bar, &dw, &z_bar, &Qw, &Qw_bar, &ATy, &ATy_bar, &ATdy,
              &QATdy, &dQw, &Qx, &tempv, &fact1, &fact2, &fact, &fact_M};
  for (V** p : nv) *p = mem.alloc<V>(n);
  V** mv[] = {&y, &y_bar, &dy, &s, &Ax};
  for (V** p : mv) *p = mem.alloc<V>(m);
  for (V** p : {&last_x, &last_w, &last_ATy, &last_Qw}) *p = mem.alloc<V>(n);
  last_y = mem.alloc<V>(m);
  stage_n = mem.alloc<double>(n);
  stage_m = mem.alloc<double>(m);
  pz = mem.alloc<V>(mx);
  pq = mem.alloc<V>(mx);
  pt = mem.alloc<V>(mx);
  HPRQP_CUDA(cudaMemsetAsync(pz, 0, sizeof(V) * mx, cm.stream));
  pz2 = mem.alloc<V>(n);
  pq2 = mem.alloc<V>(n);
  pt2 = mem.alloc<V>(n);
  ltemp2 = is_lasso ? mem.alloc<V>(hp.L.rows) : nullptr;
  const DevScaled* ds = pp.dev.get();  // the GPU scaling's device copy, if any
  c = vec_in(pp.c, ds ? ds->c : nullptr, n);
  l = vec_in(pp.l, ds ? ds->l : nullptr, n);
  u = vec_in(pp.u, ds ? ds->u : nullptr, n);
  col_norm = vec_in(pp.col_norm, ds ? ds->col_norm : nullptr, n);
  diag_Q = upload<V>(cm, mem, pp.diag_Q, n);
  AL = vec_in(pp.AL, ds ? ds->AL : nullptr, m);
  AU = vec_in(pp.AU, ds ? ds->AU : nullptr, m);
  row_norm = vec_in(pp.row_norm, ds ? ds->row_norm : nullptr, m);
  HPRQP_CUDA(cudaStreamSynchronize(cm.stream));
  const double t_vec = wall_s();
  upload_csr(pp.Apat(), A, tpr_A, ds ? &ds->A : nullptr);
  const double t_A = wall_s();
  upload_csr(pp.ATpat(), AT, tpr_A, ds ? &ds->AT : nullptr);
  const double t_AT = wall_s();
  if (has_Q_sparse) upload_csr(pp.Qpat(), Q, tpr_Q, ds ? &ds->Q : nullptr);
  const double t_Q = wall_s();
  if (is_lasso) {
    ltemp = mem.alloc<V>(hp.L.rows);
    upload_csr(hp.L, L, tpr_Q);
    upload_csr(hp.LT, LT, tpr_Q);
  }
  if (is_qap) {
    const int64_t N2 = hp.qn * hp.qn;
    qA = upload<V>(cm, mem, hp.qA, N2);
    qB = upload<V>(cm, mem, hp.qB, N2);
    qS = upload<V>(cm, mem, hp.qS, N2);
    qT = upload<V>(cm, mem, hp.qT, N2);
    qTmp = mem.alloc<V>(N2);
    // the one-instance descriptor of the CUDA-core QAP products (k_qap_gemm)
    const int qn1 = (int)hp.qn;
    const int64_t off1 = 0;
    const unsigned char on1 = 1;
    qap_n_d = mem.alloc<int>(1);
    qap_off_d = mem.alloc<int64_t>(1);
    qap_on_d = mem.alloc<unsigned char>(16);
    cm.to_dev(qap_n_d, &qn1, sizeof(int));
    cm.to_dev(qap_off_d, &off1, sizeof(int64_t));
    cm.to_dev(qap_on_d, &on1, 1);
    HPRQP_CUDA(cudaStreamSynchronize(cm.stream));
  }
  Qp = Q;
  const double t_op = wall_s();
  if (power_engine) power_setup(pp, tpr_A, tpr_Q);
  reset_state();
  HPRQP_CUDA(cudaStreamSynchronize(cm.stream));
  if (const char* tv = std::getenv("HPRQP_TIMING"))
    if (tv[0] == '1')
      std::fprintf(stderr,
                   "[hprqp] FP%d engine: vectors %.4f s, A %.4f s, A' %.4f s, Q %.4f s, LASSO/QAP %.4f s, "
                   "power set-up %.4f s\n",
                   (int)(8 * sizeof(V)), t_vec - t0, t_A - t_vec, t_AT - t_A, t_Q - t_AT, t_op - t_Q, wall_s() - t_op);
}

template <typename V>
Engine<V>::~Engine() {
  for (auto& g : pow_exec)
    if (g) cudaGraphExecDestroy(g);
}

template <typename V>
void Engine<V>::reset_state() {
  V* nv[] = {x, x_hat, x_bar, dx, w, w_bar, dw, z_bar, Qw, Qw_bar, ATy, ATy_bar, ATdy, QATdy, dQw, Qx, tempv};
  for (V* p : nv) HPRQP_CUDA(cudaMemsetAsync(p, 0, sizeof(V) * n, cm.stream));
  V* mv[] = {y, y_bar, dy, s, Ax};
  for (V* p : mv)
    if (m) HPRQP_CUDA(cudaMemsetAsync(p, 0, sizeof(V) * m, cm.stream));
  for (V* p : {last_x, last_w, last_ATy, last_Qw}) HPRQP_CUDA(cudaMemsetAsync(p, 0, sizeof(V) * n, cm.stream));
  if (m) HPRQP_CUDA(cudaMemsetAsync(last_y, 0, sizeof(V) * m, cm.stream));
}

// ---------------------------------------------------------------------------
// Products
// ---------------------------------------------------------------------------
template <typename V>
void Engine<V>::spmv(const DCsr<V>& M, const V* xin, V* yout, double scale) {
  mat_rows(M, xin, EpiStore<V>{yout, scale});
}

// QAP Qmap! (src/Q_operators/QAP_operator.jl:52-61): X = reshape(x, N, N)
// column-major; TMP = A X; QX = 2 TMP B - 2 S X - 2 X T.  FP64: the
// library's tiled CUDA-core GEMM (k_qap_gemm: TMP, then 2 TMP B - 2 S X -
// 2 X T as one GEMM over three K segments, FP64 FMAs in a fixed order);
// FP32 phase: the 3xTF32 tcgen05 GEMM (the same k_qap_gemm in FP32 when
// HPRQP_QAP_TC=0).
template <typename V>
void Engine<V>::qap_apply(const V* xin, V* yout) {
  if (is_custom) {  // the user's Qmap! (hprqp_set_qmap), on the engine's current stream
    if (!cm.qmap) throw Error(HPRQP_E_STATE, "custom Q operator: hprqp_set_qmap was not called");
    const int32_t rc = cm.qmap((const void*)xin, (void*)yout, sizeof(V) == 8 ? 0 : 1, cm.qmap_user, (void*)cm.stream);
    if (rc != 0) throw Error(HPRQP_E_CALLBACK, "custom Q operator callback returned " + std::to_string(rc));
    HPRQP_CUDA(cudaGetLastError());
    return;
  }
  const int N = (int)std::lround(std::sqrt((double)n));
  if constexpr (std::is_same<V, float>::value) {
    if (cm.tc_qap) {
      if (!qws) qws = mem.alloc<float>(gemm_3xtf32_ws_floats(N));
      gemm_3xtf32_ws(N, 1.0f, qA, xin, 0.0f, qTmp, qws, cm.stream);
      gemm_3xtf32_ws(N, 2.0f, qTmp, qB, 0.0f, yout, qws, cm.stream);
      gemm_3xtf32_ws(N, -2.0f, qS, xin, 1.0f, yout, qws, cm.stream);
      gemm_3xtf32_ws(N, -2.0f, xin, qT, 1.0f, yout, qws, cm.stream);
      cm.launches += 12;
      return;
    }
  }
  const int nt = (N + kQT - 1) / kQT;
  const dim3 g(1, nt * nt);
  const QapSegs<V, 1> s1{{qA}, {xin}, {V(1)}};
  k_qap_gemm<V, 1><<<g, 256, 0, cm.stream>>>(qap_n_d, qap_off_d, qap_on_d, s1, V(1), qTmp);
  HPRQP_LAUNCH_CHECK();
  const QapSegs<V, 3> s3{{qTmp, qS, xin}, {qB, xin, qT}, {V(1), V(-1), V(-1)}};
  k_qap_gemm<V, 3><<<g, 256, 0, cm.stream>>>(qap_n_d, qap_off_d, qap_on_d, s3, V(2), yout);
  HPRQP_LAUNCH_CHECK();
  cm.launches += 2;
}

template <typename V>
void Engine<V>::apply_Q(const V* xin, V* yout) {
  if (is_lasso) {
    spmv(L, xin, ltemp);
    spmv(LT, ltemp, yout);
  } else if (is_op) {
    qap_apply(xin, yout);
  } else {
    spmv(Q, xin, yout);
  }
}

// ---------------------------------------------------------------------------
// One HPR iteration: main_update_cpu!/gpu! (src/algorithm.jl:945-972, 1250-1279)
// ---------------------------------------------------------------------------
template <typename V>
void Engine<V>::step(bool full, double h1, double h2) {
  const double f2s = 1.0 / (1.0 + sigma * lamQ), f1s = 1.0 - f2s;
  const double fy1 = lamA * sigma, fy2 = 1.0 / fy1;
  mark();
  if (path == PATH_LASSO) {
    spmv(L, w, ltemp);
    mark();
    HPRQP_BOOL(full, F, {
      EpiLasso<V, F, V> e{x, x_hat, w_bar, w, dx, x_bar, z_bar, dw, c, last_x, last_w, sigma, lasso_lam, f1s, f2s, h1, h2};
      mat_rows(LT, ltemp, e);
    })
    mark();
    return;
  }
  if (path == PATH_QP) {
    HPRQP_BOOL(full, F, HPRQP_BOOL(Q_is_diag, D, {
      EpiZxw1<V, F, D, V> e{Qw, x, x_hat, w_bar, dx, x_bar, z_bar, ATy, c, l, u, w, fact1, fact2, last_x,
                         sigma, f1s, f2s, h1, h2};
      if (is_op) {
        qap_apply(w, Qw);
        rows<V>(cm, 1, n, VecSrc<V>{Qw}, e);
      } else {
        mat_rows(Q, w, e);
      }
    }))
    mark();
    if (m > 0) {
      EpiTempv<V> et{tempv, x_hat, Qw, sigma};
      if (is_op) {
        qap_apply(w_bar, Qw_bar);
        rows<V>(cm, 1, n, VecSrc<V>{Qw_bar}, et);
      } else {
        mat_rows(Q, w_bar, et);
      }
      mark();
      HPRQP_BOOL(full, F, {
        EpiY<V, F, true, V> ey{y, y_bar, s, dy, AL, AU, last_y, fy1, fy2, h1, h2};
        mat_rows(A, tempv, ey);
      })
      mark();
    }
    const double fs = sigma / (1.0 + sigma * lamQ);
    HPRQP_BOOL(full, F, HPRQP_BOOL(Q_is_diag, D, {
      EpiW2<V, F, D, V> e{w, ATy, w_bar, dw, ATdy, ATy_bar, fact, last_w, last_ATy, fs, h1, h2};
      if (m > 0) mat_rows(AT, y_bar, e);
      else rows<V>(cm, 1, n, ZeroSrc{}, e);
    }))
    mark();
    return;
  }
  if (path == PATH_NOC) {
    HPRQP_BOOL(full, F, HPRQP_BOOL(Q_is_diag, D, {
      EpiZxwNoC<V, F, D, V> e{x, x_hat, w_bar, w, dx, x_bar, z_bar, dw, Qw, c, l, u, fact1, fact2, last_x, last_w,
                           sigma, f1s, f2s, h1, h2};
      if (m > 0) mat_rows(AT, y, e);
      else rows<V>(cm, 1, n, ZeroSrc{}, e);
    }))
    mark();
    HPRQP_BOOL(full, F, {
      EpiTempvNoC<V, F, V> e{Qw, tempv, Qw_bar, x_hat, last_Qw, sigma, h1, h2};
      if (is_op) {
        qap_apply(w_bar, Qw_bar);
        rows<V>(cm, 1, n, VecSrc<V>{Qw_bar}, e);
      } else {
        mat_rows(Q, w_bar, e);
      }
    })
    mark();
    if (m > 0) {
      HPRQP_BOOL(full, F, {
        EpiY<V, F, true, V> ey{y, y_bar, s, dy, AL, AU, last_y, fy1, fy2, h1, h2};
        mat_rows(A, tempv, ey);
      })
      mark();
    }
    return;
  }
  // PATH_LP
  HPRQP_BOOL(full, F, {
    EpiZxLP<V, F, V> e{x, x_hat, dx, x_bar, z_bar, c, l, u, last_x, sigma, h1, h2};
    if (m > 0) mat_rows(AT, y, e);
    else rows<V>(cm, 1, n, ZeroSrc{}, e);
  })
  mark();
  if (m > 0) {
    HPRQP_BOOL(full, F, {
      EpiY<V, F, false, V> ey{y, y_bar, s, dy, AL, AU, last_y, fy1, fy2, h1, h2};
      mat_rows(A, x_hat, ey);
    })
    mark();
  }
}

// One power step streams the matrices once, gathers the input vector once,
// writes the intermediate and the next iterate and reads the current one in
// the fused dots (counted once each, at the storage size).
template <typename V>
double Engine<V>::power_step_bytes(int which) const {
  const double v = sizeof(V);
  auto csr = [&](const DCsr<V>& M) { return (double)M.nnz * (v + 4.0) + 4.0 * (M.rows + 1); };
  if (which == 0 && gram) return csr(G) + 2.0 * n * 8.0;  // FP64 state
  if (which == 0) return m > 0 ? csr(AT) + csr(A) + 2.0 * n * v + 3.0 * m * v : 0.0;
  if (is_op) return 0.0;
  if (is_lasso) return csr(L) + csr(LT) + 2.0 * L.rows * v + 3.0 * n * v;
  // the chunk-fold Q chain reads and writes an FP64 state
  return csr(Q) + 2.0 * n * (cm.pow_chunk_fold ? 8.0 : v);
}

// Name, algorithmic HBM bytes (plain iteration) and schedule of pass k.
// CSR stream = nnz (sizeof(V) + 4) + 4 (rows + 1); every distinct vector is
// counted once per pass at its storage size (the anchors included);
// the gathered input vector is counted once.
template <typename V>
void Engine<V>::pass_info(int k, const char** name, double* bytes, int* tpr) const {
  const double v = sizeof(V), d = sizeof(V);  // d: the Halpern anchors (storage type too)
  // the staged copy streams its padded chunks (16-bit columns), the warp-tile
  // descriptors, the row slot offsets and, with several column blocks, the
  // block sums
  auto csr = [&](const DCsr<V>& M) {
    if (M.stage)
      return (double)M.st_chunks * 8.0 * (v + 2.0) + 8.0 * M.st_nwt + 16.0 * (M.st_ntile + M.st_grid) +
             4.0 * M.st_nblk * (M.rows + 1) +
             (M.st_nblk > 1 ? 16.0 * M.st_nblk * M.rows + 8.0 * M.rows : 0.0);
    return (double)M.nnz * (v + 4.0) + 4.0 * (M.rows + 1);
  };
  // 0 = SELL-32, -1 = ELL, -3 = row split, -4 = staged column blocks
  auto sched = [](const DCsr<V>& M) { return M.stage ? -4 : M.split ? -3 : M.ell ? -1 : M.sell ? 0 : M.tpr; };
  const double N = (double)n, M_ = (double)m;
  const double dg = Q_is_diag ? 2 * N * v : 0.0;
  *name = "?";
  *bytes = 0;
  *tpr = 1;
  if (path == PATH_LASSO) {
    if (k == 0) { *name = "lasso1 A_d*w"; *bytes = csr(L) + N * v + L.rows * v; *tpr = sched(L); }
    else { *name = "lasso2 A_d'*t+prox"; *bytes = csr(LT) + L.rows * v + 3 * N * v + 2 * N * d + 4 * N * v; *tpr = sched(LT); }
    return;
  }
  const double cq = is_op ? 0.0 : csr(Q);
  const int tq = is_op ? 1 : sched(Q);
  if (path == PATH_QP) {
    if (k == 0) { *name = "zxw1 Q*w"; *bytes = cq + N * v + 5 * N * v + N * d + dg + 4 * N * v; *tpr = tq; }
    else if (m > 0 && k == 1) { *name = "tempv Q*w_bar"; *bytes = cq + N * v + 2 * N * v + N * v; *tpr = tq; }
    else if (m > 0 && k == 2) { *name = "y A*tempv"; *bytes = csr(A) + N * v + 3 * M_ * v + M_ * d + 2 * M_ * v; *tpr = sched(A); }
    else { *name = "w2 A'*y_bar"; *bytes = (m > 0 ? csr(AT) + M_ * v : 0.0) + 3 * N * v + 2 * N * d + (Q_is_diag ? N * v : 0.0) + 2 * N * v; *tpr = m > 0 ? sched(AT) : 1; }
    return;
  }
  if (path == PATH_NOC) {
    if (k == 0) { *name = "zxw A'*y"; *bytes = (m > 0 ? csr(AT) + M_ * v : 0.0) + 6 * N * v + 2 * N * d + dg + 4 * N * v; *tpr = m > 0 ? sched(AT) : 1; }
    else if (k == 1) { *name = "tempv Q*w_bar"; *bytes = cq + N * v + 2 * N * v + N * d + 2 * N * v; *tpr = tq; }
    else { *name = "y A*tempv"; *bytes = csr(A) + N * v + 3 * M_ * v + M_ * d + 2 * M_ * v; *tpr = sched(A); }
    return;
  }
  if (k == 0) { *name = "zx A'*y"; *bytes = (m > 0 ? csr(AT) + M_ * v : 0.0) + 4 * N * v + N * d + 2 * N * v; *tpr = m > 0 ? sched(AT) : 1; }
  else { *name = "y A*x_hat"; *bytes = m > 0 ? csr(A) + N * v + 3 * M_ * v + M_ * d + M_ * v : 0.0; *tpr = m > 0 ? sched(A) : 1; }
}

// ---------------------------------------------------------------------------
// Reductions
// ---------------------------------------------------------------------------
template <typename V>
void Engine<V>::residuals_launch(bool) {
  apply_Q(x_bar, Qx);
  EpiResN<V> e{x_bar, Qx, c, z_bar, col_norm, l, u, lam_l1, c_scale, b_scale};
  if (m > 0)
    mat_reduce<8, kResNMax>(cm, AT, y_bar, e, cm.d_scal + S_RES_N);
  else
    reduce<8, kResNMax, double>(cm, 1, n, ZeroSrc{}, e, cm.d_scal + S_RES_N);
  if (m > 0) {
    EpiResM<V> em{y_bar, s, AL, AU, row_norm, b_scale};
    mat_reduce<3, kResMMax>(cm, A, x_bar, em, cm.d_scal + S_RES_M);
  }
}

template <typename V>
void Engine<V>::mnorm_launch(int slot) {
  apply_Q(dw, dQw);
  if (m > 0) {
    spmv(AT, dy, ATdy);
    apply_Q(ATdy, QATdy);
  }
  reduce<8, 0u, double>(cm, 1, n, ZeroSrc{}, EpiMnormN<V>{dx, dQw, ATdy, QATdy, fact_M, dw, m > 0}, cm.d_scal + slot);
  reduce<1, 0u, double>(cm, 1, m, ZeroSrc{}, EpiSumSq<V>{dy}, cm.d_scal + slot + 8);
}

template <typename V>
void Engine<V>::sigma_stats_launch() {
  {
    V *dx_ = dx, *dw_ = dw, *ATdy_ = ATdy;
    const V *xb = x_bar, *wb = w_bar, *atyb = ATy_bar;
    const V *lx = last_x, *lw = last_w, *laty = last_ATy;
    const bool hm = m > 0;
    elem(cm, n, [=] __device__(int i) {
      dx_[i] = (V)((double)xb[i] - (double)lx[i]);
      dw_[i] = (V)((double)wb[i] - (double)lw[i]);
      if (hm) ATdy_[i] = (V)((double)atyb[i] - (double)laty[i]);
    });
    V* dy_ = dy;
    const V* yb = y_bar;
    const V* ly = last_y;
    elem(cm, m, [=] __device__(int i) { dy_[i] = (V)((double)yb[i] - (double)ly[i]); });
  }
  apply_Q(dw, dQw);
  if (m > 0) apply_Q(ATdy, QATdy);
  reduce<5, 0u, double>(cm, 1, n, ZeroSrc{}, EpiSigmaN<V>{dx, dQw, ATdy, QATdy, dw, m > 0}, cm.d_scal + S_SIG);
  reduce<1, 0u, double>(cm, 1, m, ZeroSrc{}, EpiSumSq<V>{dy}, cm.d_scal + S_SIG + 5);
}

template <typename V>
void Engine<V>::golden_diag_launch(double a, double b) {
  k_golden_diag<V><<<1, 1024, 0, cm.stream>>>((int)n, a, b, diag_Q, ATdy, QATdy, 1e-12, 1e12, 1e-13, 200,
                                              cm.d_scal + S_GOLD);
  cm.launches++;
  HPRQP_LAUNCH_CHECK();
}

template <typename V>
void Engine<V>::set_sigma(double sg) {
  sigma = sg;
  if (!Q_is_diag) return;
  // unified_update_Q_factors! (src/unified_operations.jl:445-459)
  V *f2 = fact2, *f = fact, *f1 = fact1, *fM = fact_M;
  const V* dq = diag_Q;
  const double s2 = sg * sg;
  elem(cm, n, [=] __device__(int i) {
    const double q = dq[i];
    const double t2 = 1.0 / (1.0 + sg * q);
    f2[i] = (V)t2;
    f[i] = (V)(sg * t2);
    f1[i] = (V)(sg * q * t2);
    fM[i] = (V)(s2 * t2);
  });
}

template <typename V>
void Engine<V>::restart() {
  EpiRestartN<V> e{x, w, ATy, ATy_bar, Qw, x_bar, w_bar, Qw_bar, last_x, last_w, last_ATy, last_Qw,
                   m > 0, path == PATH_NOC};
  if (m > 0) mat_rows(AT, y_bar, e);
  else rows<V>(cm, 1, n, ZeroSrc{}, e);
  V *y_ = y;
  const V* yb = y_bar;
  V* ly = last_y;
  elem(cm, m, [=] __device__(int i) {
    y_[i] = yb[i];
    ly[i] = yb[i];
  });
}

// process_initial_points! (src/algorithm.jl:1783-1836)
template <typename V>
void Engine<V>::initial_points(const double* x0, const double* y0) {
  if (x0) {
    cm.to_dev(stage_n, x0, sizeof(double) * n);
    V *x_ = x, *xb = x_bar, *w_ = w, *wb = w_bar;
    V *lx = last_x, *lw = last_w;
    const double* st = stage_n;
    const V* cn = col_norm;
    const double bs = b_scale;
    elem(cm, n, [=] __device__(int i) {
      const double v = st[i] * (double)cn[i] / bs;
      x_[i] = xb[i] = w_[i] = wb[i] = (V)v;
      lx[i] = lw[i] = (V)v;
    });
  }
  if (y0) {
    if (m > 0) {
      cm.to_dev(stage_m, y0, sizeof(double) * m);
      V *y_ = y, *yb = y_bar;
      V* ly = last_y;
      const double* st = stage_m;
      const V* rn = row_norm;
      const double cs = c_scale;
      elem(cm, m, [=] __device__(int i) {
        const double v = st[i] * (double)rn[i] / cs;
        y_[i] = yb[i] = (V)v;
        ly[i] = (V)v;
      });
      spmv(AT, y_bar, ATy_bar);
      V* aty = ATy;
      const V* atyb = ATy_bar;
      V* laty = last_ATy;
      elem(cm, n, [=] __device__(int i) {
        aty[i] = atyb[i];
        laty[i] = atyb[i];
      });
    }
    apply_Q(x_bar, Qx);
    {
      V* zb = z_bar;
      const V *xb = x_bar, *qx = Qx, *atyb = ATy_bar, *cc = c;
      const double sg = sigma;
      elem(cm, n, [=] __device__(int i) {
        const double tmp = -(double)qx[i] + (double)atyb[i] - (double)cc[i];
        const double z_raw = (double)xb[i] + sg * tmp;
        zb[i] = (V)(((double)xb[i] - z_raw) / sg);
      });
    }
    if (m > 0) {
      spmv(A, x_bar, Ax);
      V* s_ = s;
      const V *ax = Ax, *y_ = y, *al = AL, *au = AU;
      const double f1 = lamA * sigma;
      elem(cm, m, [=] __device__(int i) {
        s_[i] = (V)clampd((double)ax[i] - f1 * (double)y_[i], (double)al[i], (double)au[i]);
      });
    }
  }
}

// collect_results! (src/algorithm.jl:611-643)
template <typename V>
void Engine<V>::collect(double* xo, double* yo, double* zo, double* wo) {
  const V *xb = x_bar, *wb = w_bar, *zb = z_bar, *cn = col_norm;
  double* st = stage_n;
  const double bs = b_scale, cs = c_scale;
  auto copy_n = [&](double* dst) {
    cm.to_host(dst, stage_n, sizeof(double) * n);
    HPRQP_CUDA(cudaStreamSynchronize(cm.stream));
  };
  if (xo) {
    elem(cm, n, [=] __device__(int i) { st[i] = bs * ((double)xb[i] / (double)cn[i]); });
    copy_n(xo);
  }
  if (wo) {
    elem(cm, n, [=] __device__(int i) { st[i] = bs * ((double)wb[i] / (double)cn[i]); });
    copy_n(wo);
  }
  if (zo) {
    elem(cm, n, [=] __device__(int i) { st[i] = cs * ((double)zb[i] * (double)cn[i]); });
    copy_n(zo);
  }
  if (yo && m > 0) {
    const V *yb = y_bar, *rn = row_norm;
    double* sm = stage_m;
    elem(cm, m, [=] __device__(int i) { sm[i] = cs * ((double)yb[i] / (double)rn[i]); });
    cm.to_host(yo, stage_m, sizeof(double) * m);
  }
  HPRQP_CUDA(cudaStreamSynchronize(cm.stream));
}

template <typename V>
void Engine<V>::trace_copy(double* xt, double* yt, double* wt) {
  auto out = [&](const V* src, int64_t len, double* stage, double* dst) {
    if (!dst || len == 0) return;
    elem(cm, len, CastCopy<double, V>{stage, src});
    cm.to_host(dst, stage, sizeof(double) * len);
    HPRQP_CUDA(cudaStreamSynchronize(cm.stream));
  };
  out(x, n, stage_n, xt);
  out(y, m, stage_m, yt);
  out(w, n, stage_n, wt);
}

template <typename V>
void Engine<V>::vec_to_host(const V* src, int64_t len, double* dst) {
  if (!dst || len <= 0) return;
  double* stage = len <= n ? stage_n : stage_m;
  if (len > std::max(n, m)) throw Error(HPRQP_E_ARG, "vec_to_host: length beyond the staging buffers");
  elem(cm, len, CastCopy<double, V>{stage, src});
  cm.to_host(dst, stage, sizeof(double) * len);
  HPRQP_CUDA(cudaStreamSynchronize(cm.stream));
}

template <typename V>
void Engine<V>::vec_from_host(V* dst, const double* src, int64_t len) {
  if (!src || len <= 0) return;
  double* stage = len <= n ? stage_n : stage_m;
  if (len > std::max(n, m)) throw Error(HPRQP_E_ARG, "vec_from_host: length beyond the staging buffers");
  cm.to_dev(stage, src, sizeof(double) * len);
  elem(cm, len, CastCopy<V, double>{dst, stage});
  HPRQP_CUDA(cudaStreamSynchronize(cm.stream));
}

template <typename V>
void Engine<V>::bars_to_device(double* xb, double* yb, double* zb, double* wb) {
  elem(cm, n, CastCopy<double, V>{xb, x_bar});
  elem(cm, n, CastCopy<double, V>{zb, z_bar});
  elem(cm, n, CastCopy<double, V>{wb, w_bar});
  if (m > 0) elem(cm, m, CastCopy<double, V>{yb, y_bar});
}

// ---------------------------------------------------------------------------
// Power method (src/utils.jl:1335-1461).  One power step is one fused kernel
// for a sparse Q (the product, z_next, and the q.z / z.z / q.q sums), two
// for A A' and the LASSO operator, a GEMM chain + one reduction for QAP.
// kPowChunk steps (z ping-pongs between two buffers, so an even chunk ends
// where it started) are captured once in a CUDA graph and replayed; the host
// reads the (lambda, err) log once per chunk and stops at the first step
// with err < tol, returning that step's lambda.
// ---------------------------------------------------------------------------
template <typename V>
struct ScaleInvNorm {  // q = z / ||z||, the norm read from the device
  V* q;
  const V* z;
  const double* zz;
  __device__ __forceinline__ void operator()(int i) const { q[i] = (V)((double)z[i] / sqrt(*zz)); }
};

// Both chains in one persistent cooperative kernel (power.cuh).  The start
// vectors and ||z_0||^2 are in place (power_both).  Returns false when the
// kernel cannot be co-resident on this GPU (the caller then runs the
// graph-captured chains).
template <typename V>
bool Engine<V>::power_persistent(bool onA, bool onQ, double tol, int max_it, double* lamA_out, double* lamQ_out,
                                 int64_t* itA, int64_t* itQ) {
  int per = 0;
  HPRQP_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_power_persistent<V>, kPowBlock, 0));
  if (cm.pow_ctas_per_sm > 0) per = std::min(per, cm.pow_ctas_per_sm);
  else per = std::min(per, 2);
  const int grid = std::min(per * cm.num_sms, kPowMaxGrid);
  if (grid < 1) return false;
  PowArgs<V> pa{};
  // the persistent sweeps keep kPowIlp rows in flight only on ELL: use it
  // wherever the matrix has an ELL copy
  auto pick = [&](const DCsr<V>& M) {
    DCsr<V> d = M;
    if (cm.pow_prefer_ell && d.ell_w > 0) {
      d.ell = true;
      d.sell = false;
    }
    return d;
  };
  if (onA) {
    PowChain<V>& c = pa.ch[0];
    c.kind = 2;
    c.M1 = pick(AT);
    c.M2 = pick(A);
    c.z0 = pz;
    c.z1 = pq;
    c.t = pt;
    c.zz0 = cm.d_scal + S_POW + 2;
  }
  if (onQ) {
    PowChain<V>& c = pa.ch[1];
    if (is_lasso) {
      c.kind = 2;
      c.M1 = pick(L);
      c.M2 = pick(LT);
      c.t = ltemp2;
    } else {
      c.kind = 1;
      c.M1 = pick(Q);
    }
    c.z0 = pz2;
    c.z1 = pq2;
    c.zz0 = cm.d_scal + S_POW_Q + 2;
  }
  pa.tol = tol;
  pa.max_it = max_it;
  pa.partials = cm.pow_part;
  pa.bar = cm.pow_bar;
  pa.status = reinterpret_cast<int*>(cm.pow_bar + 1);
  pa.out = cm.d_scal + S_POWLOG;
  HPRQP_CUDA(cudaMemsetAsync(cm.pow_bar, 0, 64 * sizeof(unsigned), cm.stream));
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3((unsigned)grid);
  cfg.blockDim = dim3((unsigned)kPowBlock);
  cfg.stream = cm.stream;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeCooperative;
  at[0].val.cooperative = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  HPRQP_CUDA(cudaLaunchKernelEx(&cfg, k_power_persistent<V>, pa));
  cm.launches++;
  cm.sync_read(S_POWLOG, 9);
  const double* o = cm.h_scal + S_POWLOG;
  if (o[8] != 0.0) throw Error(HPRQP_E_CUDA, "power method: a grid barrier wait timed out");
  const bool on[2] = {onA, onQ};
  for (int c = 0; c < 2; ++c) {
    if (!on[c]) continue;
    const double lam = o[4 * c], found = o[4 * c + 1], steps = o[4 * c + 2];
    if (found < 0)
      std::fprintf(stderr, "Power iteration (%s) did not converge within the specified tolerance.\n",
                   c == 0 ? "A" : "Q");
    const int64_t it = (int64_t)(found >= 0 ? found : steps);
    if (c == 0) {
      if (lamA_out) *lamA_out = lam;
      if (itA) *itA = it;
    } else {
      if (lamQ_out) *lamQ_out = lam;
      if (itQ) *itQ = it;
    }
  }
  if (!onA) {
    if (lamA_out) *lamA_out = 1.0;
    if (itA) *itA = 0;
  }
  if (!onQ) {
    if (lamQ_out) *lamQ_out = 1.0;
    if (itQ) *itQ = 0;
  }
  return true;
}

template <typename V>
void Engine<V>::power_both(bool want_A, bool want_Q, double tol, int max_it, double* lamA_out, double* lamQ_out,
                           int64_t* itA, int64_t* itQ) {
  struct Chain {
    bool on;
    int which;  // 0 = A A', 1 = Q
    V *z0, *z1, *t;
    double *scal, *log;
    ReduceWs ws;
    cudaStream_t st;
    int64_t len;
    double lam;
    int found;
  };
  const cudaStream_t main = cm.stream;
  const ReduceWs main_ws = cm.rws;
  // the QAP operator's cuBLAS calls are bound to the main stream: one stream then
  const cudaStream_t qst = is_op ? main : cm.stream2;
  Chain ca{want_A && m > 0, 0, pz, pq, pt, cm.d_scal + S_POW, cm.d_scal + S_POWLOG, cm.rws, main, m, 1.0, -1};
  Chain cq{want_Q, 1, pz2, pq2, pt2, cm.d_scal + S_POW_Q, cm.d_scal + S_POWLOG_Q, cm.rws2, qst, n, 1.0, -1};
  auto use = [&](const Chain& c, cudaStream_t st) {
    cm.stream = st;
    cm.rws = c.ws;
  };
  auto restore = [&]() {
    cm.stream = main;
    cm.rws = main_ws;
  };
  for (Chain* c : {&ca, &cq}) {
    if (!c->on) continue;
    // the start vector (power_start_vector's stream) generated in place
    k_start_vector<V><<<(int)((c->len + kBlock - 1) / kBlock), kBlock, 0, main>>>(c->len, c->z0);
    HPRQP_LAUNCH_CHECK();
    cm.launches++;
    use(*c, main);
    reduce<1, 0u, double>(cm, 1, c->len, ZeroSrc{}, EpiSumSq<V>{c->z0}, c->scal + 2, InvNormFin{c->scal + 4});
    restore();
  }
  if (cm.pow_persistent && !is_op && power_persistent(ca.on, cq.on, tol, max_it, lamA_out, lamQ_out, itA, itQ))
    return;
  // HPRQP_POWER_ELL=1: the chained steps use ELL wherever the matrix has an
  // ELL copy (its reduction keeps 4 rows per thread in flight); measured
  // slower than the autotuned formats on the 700x700 grid (107 vs 97 ms)
  auto ellp = [&](const DCsr<V>& M) {
    DCsr<V> d = M;
    if (cm.pow_prefer_ell && d.ell_w > 0) {
      d.ell = true;
      d.sell = false;
    }
    return d;
  };
  const DCsr<V> pA = ellp(A), pAT = ellp(AT), pQ = ellp(Qp.rows ? Qp : Q), pL = ellp(L), pLT = ellp(LT);
  // A A' on the Gram matrix: G's values for this solve, u_0 = A' z_0 (the
  // chain's n-space state; 1/||z_0|| is already in scal + 4), then one
  // sweep of G per step
  const bool use_gram = gram && ca.on;
  // Chunk fold (HPRQP_POWER_CHUNK_FOLD, default on): the Gram chain and a
  // sparse Q's chain run unnormalised, each step writing only its per-CTA
  // sums; one fold per chunk gives every step's (lambda, err) and
  // renormalises the state (kernels.cuh).  The other chains keep the
  // per-step fold.
  const bool cfA = cm.pow_chunk_fold && use_gram;
  const bool cfQ = cm.pow_chunk_fold && cq.on && has_Q_sparse && !is_lasso && !is_op;
  const int nblkA = cfA ? partials_grid(cm, G) : 0, nblkQ = cfQ ? partials_grid(cm, pQ) : 0;
  if ((cfA || cfQ) && !pow_cf_part) {
    // one region per chain, each kPowChunk steps x (at most reduce_cap CTAs) x 3 sums
    pow_cf_region = (int64_t)kPowChunk * std::max(cm.reduce_cap, 1) * 3;
    pow_cf_part = mem.alloc<double>(2 * pow_cf_region);
    pow_cf_tot = mem.alloc<double>(2 * kPowChunk * 3);
  }
  // the unnormalised Q chain keeps an FP64 state: within a chunk it grows by
  // about lambda^32, which FP32 cannot hold for lambda above ~15
  if (cfQ) {
    if (!gq0) {
      gq0 = mem.alloc<double>(n);
      gq1 = mem.alloc<double>(n);
    }
    k_start_vector<double><<<(int)((n + kBlock - 1) / kBlock), kBlock, 0, main>>>(n, gq0);
    HPRQP_LAUNCH_CHECK();
    cm.launches++;
  }
  if (use_gram) {
    gram_values();
    // u_0 = A' z_0 / ||z_0|| = w_0 (the chunk fold starts from a normalised state)
    mat_rows(pAT, pz, EpiStoreInvNorm<double>{gu0, ca.scal + 2, ca.scal + 4});
  }
  auto chunk_chain = [&](bool on, int kind, int nblk, double* log) {
    PowChunkChain d{};
    if (!on) return d;
    d.kind = kind;
    d.K = kind == 0 ? 2 : 3;
    d.nblk = nblk;
    d.steps = kPowChunk;
    d.partials = pow_cf_part + (size_t)kind * pow_cf_region;
    d.totals = pow_cf_tot + kind * kPowChunk * 3;
    d.log = log;
    d.len = n;
    if (kind == 0) d.state64 = gu0;
    else d.stateQ64 = gq0;
    return d;
  };
  auto step = [&](const Chain& c, cudaStream_t st, int k) {
    use(c, st);
    V* zc = (k & 1) ? c.z1 : c.z0;
    V* zn = (k & 1) ? c.z0 : c.z1;
    double* zz = c.scal + 2;
    // 1/||z|| is formed once per step (PowerFin / InvNormFin) into scal + 4
    const double* inv = c.scal + 4;
    const PowerFin fin{c.log, k, c.scal + 4};
    // HPRQP_POWER_SPLIT=1: the last product of a step as a plain row pass
    // (one row per thread, no reduction) and the three dots as a separate
    // streaming reduction over (z, z_next)
    auto dots = [&](int64_t len) {
      reduce<3, 0u, double>(cm, 1, len, VecSrc<V>{zn}, EpiPowerFused<V>{zc, nullptr, zz, false, inv}, c.scal + 1,
                            fin);
    };
    if (c.which == 0 && cfA) {  // chunk fold: partials of step k only
      const double* uc = (k & 1) ? gu1 : gu0;
      double* un = (k & 1) ? gu0 : gu1;
      mat_partials<2>(cm, G, uc, EpiGramRaw{uc, un}, pow_cf_part + (size_t)k * nblkA * 2);
    } else if (c.which == 1 && cfQ) {
      const double* yc = (k & 1) ? gq1 : gq0;
      double* yn = (k & 1) ? gq0 : gq1;
      mat_partials<3>(cm, pQ, yc, EpiPowRaw<double>{yc, yn},
                      pow_cf_part + (size_t)pow_cf_region + (size_t)k * nblkQ * 3);
    } else if (c.which == 0 && use_gram) {  // u ping-pongs between gu0 and gu1
      const double* uc = (k & 1) ? gu1 : gu0;
      double* un = (k & 1) ? gu0 : gu1;
      mat_reduce<2, 0u>(cm, G, uc, EpiGramPower<double>{uc, un, inv}, c.scal + 1, GramPowerFin{c.log, k, c.scal + 4});
    } else if (c.which == 0) {  // A A' (power_iteration_A)
      mat_rows(pAT, zc, EpiStoreInvNorm<V>{c.t, zz, inv});
      if (cm.pow_split) {
        mat_rows(pA, c.t, EpiStore<V>{zn, 1.0});
        dots(m);
      } else {
        mat_reduce<3, 0u>(cm, pA, c.t, EpiPowerFused<V>{zc, zn, zz, false, inv}, c.scal + 1, fin);
      }
    } else if (is_lasso) {
      mat_rows(pL, zc, EpiStoreInvNorm<V>{ltemp2, zz, inv});
      if (cm.pow_split) {
        mat_rows(pLT, ltemp2, EpiStore<V>{zn, 1.0});
        dots(n);
      } else {
        mat_reduce<3, 0u>(cm, pLT, ltemp2, EpiPowerFused<V>{zc, zn, zz, false, inv}, c.scal + 1, fin);
      }
    } else if (is_op) {
      elem(cm, n, ScaleInvNorm<V>{c.t, zc, zz});
      qap_apply(c.t, zn);
      reduce<3, 0u, double>(cm, 1, n, VecSrc<V>{zn}, EpiPowerFused<V>{zc, zn, zz, false, inv}, c.scal + 1, fin);
    } else {
      if (cm.pow_split) {
        mat_rows(pQ, zc, EpiStoreInvNorm<V>{zn, zz, inv});
        dots(n);
      } else {
        mat_reduce<3, 0u>(cm, pQ, zc, EpiPowerFused<V>{zc, zn, zz, true, inv}, c.scal + 1, fin);
      }
    }
    restore();
  };
  // one chunk = kPowChunk steps of every active chain; A on the main stream,
  // Q forked onto the second stream when both run (captured in a graph)
  // the instantiated chunk graphs are kept for the engine's later power
  // methods: they depend only on the engine's buffers and on this key
  const int key = (ca.on ? 1 : 0) | (cq.on ? 2 : 0) | (use_gram ? 4 : 0) | (cfA ? 8 : 0) | (cfQ ? 16 : 0) |
                  (cm.pow_split ? 32 : 0) | (cm.pow_prefer_ell ? 64 : 0);
  if (key != pow_exec_key) {
    for (auto& g : pow_exec)
      if (g) {
        cudaGraphExecDestroy(g);
        g = nullptr;
      }
    pow_exec_key = key;
  }
  cudaGraphExec_t* graphs = pow_exec;
  int64_t* graph_launches = pow_exec_launches;
  cudaEvent_t fork = nullptr, join = nullptr;
  HPRQP_CUDA(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
  HPRQP_CUDA(cudaEventCreateWithFlags(&join, cudaEventDisableTiming));
  auto issue_chunk = [&](bool doA, bool doQ) {
    const bool two = doA && doQ && qst != main;
    if (two) {
      HPRQP_CUDA(cudaEventRecord(fork, main));
      HPRQP_CUDA(cudaStreamWaitEvent(qst, fork, 0));
    }
    for (int k = 0; k < kPowChunk; ++k) {
      if (doA) step(ca, main, k);
      if (doQ) step(cq, two ? qst : main, k);
    }
    if (two) {
      HPRQP_CUDA(cudaEventRecord(join, qst));
      HPRQP_CUDA(cudaStreamWaitEvent(main, join, 0));
    }
    const PowChunkChain c0 = chunk_chain(doA && cfA, 0, nblkA, ca.log);
    const PowChunkChain c1 = chunk_chain(doQ && cfQ, 1, nblkQ, cq.log);
    if (c0.steps || c1.steps) {
      launch(cm, k_pow_chunk_fold, dim3(kPowChunk, 2), kBlock, c0, c1);
      const int g = (int)std::min<int64_t>(kMaxReduceGrid, (n + kBlock - 1) / kBlock);
      launch(cm, k_pow_chunk_finish, dim3(g, 2), kBlock, c0, c1);
    }
  };
  int it = 0;
  bool cf_failed = false;
  while (it < max_it && ((ca.on && ca.found < 0) || (cq.on && cq.found < 0))) {
    const bool doA = ca.on && ca.found < 0, doQ = cq.on && cq.found < 0;
    const int gi = (doA ? 1 : 0) | (doQ ? 2 : 0);
    if (is_op) {
      issue_chunk(doA, doQ);  // cuBLAS inside: run eagerly
    } else {
      if (!graphs[gi]) {
        HPRQP_CUDA(cudaStreamSynchronize(main));
        HPRQP_CUDA(cudaStreamSynchronize(cm.stream2));
        cudaGraph_t g = nullptr;
        const int64_t l0 = cm.launches;
        HPRQP_CUDA(cudaStreamBeginCapture(main, cudaStreamCaptureModeThreadLocal));
        issue_chunk(doA, doQ);
        HPRQP_CUDA(cudaStreamEndCapture(main, &g));
        graph_launches[gi] = cm.launches - l0;
        cm.launches = l0;
        HPRQP_CUDA(cudaGraphInstantiate(&graphs[gi], g, 0));
        cudaGraphDestroy(g);
      }
      HPRQP_CUDA(cudaGraphLaunch(graphs[gi], main));
      cm.launches += graph_launches[gi];
    }
    cm.sync_read(S_POWLOG, 4 * kPowChunk);
    for (Chain* c : {&ca, &cq}) {
      if (!c->on || c->found >= 0) continue;
      const double* lg = cm.h_scal + (c->which == 0 ? S_POWLOG : S_POWLOG_Q);
      for (int k = 0; k < kPowChunk && it + k < max_it; ++k) {
        if (std::isnan(lg[2 * k]) && (c->which == 0 ? cfA : cfQ)) cf_failed = true;
        c->lam = lg[2 * k];
        if (lg[2 * k + 1] < tol) {
          c->found = it + k + 1;
          break;
        }
      }
    }
    it += kPowChunk;
    if (cf_failed) break;
  }
  cudaEventDestroy(fork);
  cudaEventDestroy(join);
  if (cf_failed) {  // a chunk-fold state left FP64 range: the per-step fold instead
    cm.pow_chunk_fold = false;
    try {
      power_both(want_A, want_Q, tol, max_it, lamA_out, lamQ_out, itA, itQ);
    } catch (...) {
      cm.pow_chunk_fold = true;
      throw;
    }
    cm.pow_chunk_fold = true;
    return;
  }
  for (Chain* c : {&ca, &cq})
    if (c->on && c->found < 0)
      std::fprintf(stderr, "Power iteration (%s) did not converge within the specified tolerance.\n",
                   c->which == 0 ? "A" : "Q");
  if (lamA_out) *lamA_out = ca.lam;
  if (lamQ_out) *lamQ_out = cq.lam;
  if (itA) *itA = ca.found >= 0 ? ca.found : std::min(it, max_it);
  if (itQ) *itQ = cq.found >= 0 ? cq.found : std::min(it, max_it);
}

// FP32 -> FP64 hand-over of the full iteration state (precision switch)
template <typename V>
template <typename W>
void Engine<V>::import_state(const Engine<W>& o) {
  auto cv = [&](V* dst, const W* src, int64_t len) { elem(cm, len, CastCopy<V, W>{dst, src}); };
  cv(x, o.x, n); cv(x_hat, o.x_hat, n); cv(x_bar, o.x_bar, n); cv(dx, o.dx, n);
  cv(w, o.w, n); cv(w_bar, o.w_bar, n); cv(dw, o.dw, n); cv(z_bar, o.z_bar, n);
  cv(Qw, o.Qw, n); cv(Qw_bar, o.Qw_bar, n); cv(ATy, o.ATy, n); cv(ATy_bar, o.ATy_bar, n);
  cv(ATdy, o.ATdy, n); cv(tempv, o.tempv, n);
  cv(y, o.y, m); cv(y_bar, o.y_bar, m); cv(dy, o.dy, m); cv(s, o.s, m);
  auto cp = [&](double* dst, const double* src, int64_t len) {
    if (len) HPRQP_CUDA(cudaMemcpyAsync(dst, src, sizeof(double) * len, cudaMemcpyDeviceToDevice, cm.stream));
  };
  cv(last_x, o.last_x, n); cv(last_w, o.last_w, n); cv(last_ATy, o.last_ATy, n); cv(last_Qw, o.last_Qw, n);
  cv(last_y, o.last_y, m);
  lamA = o.lamA;
  lamQ = o.lamQ;
  lam_l1 = o.lam_l1;
  set_sigma(o.sigma);
}

template class Engine<double>;
template class Engine<float>;
template void Engine<double>::import_state<float>(const Engine<float>&);

}  // namespace hprqp
