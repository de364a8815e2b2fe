// batch.cu — batched HPR solves of a LASSO family in one launch sequence.
//
// B instances (A_k: m_k x n, c_k, lambda_k; Q_k = A_k' A_k) are concatenated
// into one block-diagonal CSR (A_d and A_d'), and every HPR pass is one
// kernel over all instances' rows: a row knows its instance through a
// row -> instance map and reads that instance's sigma, lambda, lambda_max(Q)
// and Halpern counter from per-instance arrays; rows of converged instances
// are skipped (convergence mask).  Per-instance reductions (residuals,
// M-norm, sigma statistics, power method) are segmented: each CTA reduces a
// tile of rows of one instance, and a fold kernel sums each instance's tiles
// in a fixed order (deterministic).
//
// The control logic is the reference's, per instance (src/algorithm.jl:
// 323-576, 689-739, 1977-2038, LASSO path src/kernels.jl:2400-2496): the
// host keeps one restart / sigma / residual record per instance and all
// instances advance in lockstep.  With the FP32 + polish mode each instance
// switches to the FP64 engine on its own when its KKT drops below polish_tol.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <memory>
#include <string>
#include <type_traits>
#include <vector>

#include "pool.h"
#include "../../include/hprqp.h"
#include "../../include/hprqp_batch.h"
#include "batch_qp.h"
#include "host_setup.h"
#include "kernels.cuh"

namespace hprqp {
namespace batch {

constexpr int kTileRows = 1024;  // rows per reduction tile (256 threads x 4)
constexpr int kStallChecks = 3;     // FP32 phase: evaluations without a 10% KKT gain before the switch
constexpr int kStallMinIter = 300;  // ... and not before this iteration
constexpr int kMaxK = 8;
constexpr int kPowWin = 16;      // power steps between host checks

// ---------------------------------------------------------------------------
// Kernels
// ---------------------------------------------------------------------------
struct Inst {  // per-instance device arrays
  const int* inst;          // row -> instance
  const unsigned char* on;  // instance active in this engine
};

template <int TPR, typename V, typename Epi>
__global__ void __launch_bounds__(kBlock) k_rows(int nrows, Inst I, CsrSrc<V, V> src, Epi epi) {
  pdl_enter();
  const long long g = (long long)blockIdx.x * kBlock + threadIdx.x;
  const int row = (int)(g / TPR);
  if (row >= nrows) return;
  const int k = I.inst[row];
  if (!I.on[k]) return;  // uniform over the row group
  const int lane = threadIdx.x & (TPR - 1);
  const V acc = src.template dot<TPR, V>(row, lane);
  if (lane == 0) epi(row, k, acc);
}

// Staged pass over a block-diagonal batch (BStage): instance k's rows only
// touch its own columns [coff[k], coff[k] + ncol[k]), so that column block is
// the CTA's shared-memory copy of the input.  One CTA per tile (whole rows
// of one instance, at most kStageSlots row-sum slots): the CTA stages its
// instance's block, streams the tile's 32-chunk warp tiles (two per warp
// and step, loads in flight together, the next step prefetched into L2) with
// the segmented scan into slots, then one thread per row folds the row's
// slots in order and runs the epilogue.  The chunk layout, the scan and the
// order of every sum are those of k_stage_pass; tiles of inactive instances
// return at once.
template <typename V>
struct BStageView {
  const uint16_t* __restrict__ col;
  const V* __restrict__ val;
  const int2* __restrict__ wt;    // per warp tile {first slot, segment-head mask}
  const int4* __restrict__ tile;  // {first warp tile, chunks, first row, end row}
  const int* __restrict__ tinst;  // tile -> instance
  const int* __restrict__ srow;   // first slot of each row (rows + 1)
  const int* __restrict__ coff;   // instance -> first column
  const int* __restrict__ ncol;   // instance -> columns
};

constexpr int kBStageBlock = 512;  // two CTAs per SM at 64 registers

template <typename V, typename Epi>
__global__ void __launch_bounds__(kBStageBlock, 2) k_bstage_pass(BStageView<V> s, const V* __restrict__ x,
                                                                 const unsigned char* __restrict__ on, Epi epi) {
  extern __shared__ __align__(16) unsigned char bstage_smem[];
  V* sums = reinterpret_cast<V*>(bstage_smem);
  V* xs = reinterpret_cast<V*>(bstage_smem + kStageSlots * sizeof(V));
  constexpr int NW = kBStageBlock / 32, U = 2;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int4 tl = __ldg(s.tile + blockIdx.x);  // the schedule and the matrix are constant: before the wait
  const int k = __ldg(s.tinst + blockIdx.x);
  const int C0 = 32 * tl.x, C1 = C0 + tl.y;
  StageChunk<V> ck[U];
  int2 d[U];
  int kw = warp;
  auto load_step = [&]() {
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int w = kw + u * NW;
      d[u] = C0 + 32 * w < C1 ? __ldg(s.wt + tl.x + w) : make_int2(0, 0);
      if (C0 + 32 * w + lane < C1) stage_load(ck[u], s.col, s.val, (int64_t)tl.x + w, lane);
    }
    if (lane == 0) {
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int w = kw + (U + u) * NW;
        if (C0 + 32 * w < C1) stage_prefetch(s.col, s.val, (int64_t)tl.x + w);
      }
    }
  };
  load_step();
  pdl_enter();
  if (!on[k]) return;  // (uniform over the CTA)
  const int c0 = __ldg(s.coff + k), len = __ldg(s.ncol + k);
  const V* src = x + c0;
  if ((reinterpret_cast<uintptr_t>(src) & 15u) == 0) {
    constexpr int P = 16 / (int)sizeof(V);
    const int nv = len / P;
    for (int q = threadIdx.x; q < nv; q += kBStageBlock)
      reinterpret_cast<uint4*>(xs)[q] = __ldg(reinterpret_cast<const uint4*>(src) + q);
    for (int q = nv * P + threadIdx.x; q < len; q += kBStageBlock) xs[q] = __ldg(src + q);
  } else {
    for (int q = threadIdx.x; q < len; q += kBStageBlock) xs[q] = __ldg(src + q);
  }
  __syncthreads();
  const int slot0 = __ldg(s.srow + tl.z);
  const int nwt = (C1 - C0 + 31) / 32;
  while (kw < nwt) {
    V v[U];
#pragma unroll
    for (int u = 0; u < U; ++u)  // every gather before any slot store
      v[u] = C0 + 32 * (kw + u * NW) + lane < C1 ? stage_dot<V>(ck[u], xs) : V(0);
    unsigned f[U], heads[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      heads[u] = (unsigned)d[u].y;
      f[u] = (heads[u] >> lane) & 1u;
    }
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const V o = __shfl_up_sync(0xffffffffu, v[u], off);
        const unsigned fo = __shfl_up_sync(0xffffffffu, f[u], off);
        if (lane >= off) {
          if (!f[u]) v[u] += o;
          f[u] |= fo;
        }
      }
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int last = min(31, C1 - C0 - 32 * (kw + u * NW) - 1);
      if (lane <= last && (lane == last || ((heads[u] >> (lane + 1)) & 1u)))
        sums[d[u].x - slot0 + __popc(heads[u] & (0xffffffffu >> (31 - lane))) - 1] = v[u];
    }
    kw += U * NW;
    if (kw < nwt) load_step();
  }
  __syncthreads();
  for (int r = tl.z + (int)threadIdx.x; r < tl.w; r += kBStageBlock) {
    const int a = __ldg(s.srow + r) - slot0, e = __ldg(s.srow + r + 1) - slot0;
    V acc = sums[a];
    for (int q = a + 1; q < e; ++q) acc += sums[q];
    epi(r, k, acc);
  }
}

// Fill of a batch's staged copy: row r's entries in CSR order from chunk
// pc[r] on, columns local to the row's instance (the copy was zeroed
// first; no columns when scol is null: a second precision's values for the
// same structure); values lane-interleaved as in k_stage_fill.
template <typename V>
__global__ void __launch_bounds__(kBlock) k_bstage_fill(int rows, const int* __restrict__ ptr,
                                                        const int* __restrict__ col, const V* __restrict__ val,
                                                        const int* __restrict__ inst, const int* __restrict__ coff,
                                                        const int* __restrict__ pc, uint16_t* __restrict__ scol,
                                                        V* __restrict__ sval) {
  constexpr int S = 16 / (int)sizeof(V);
  const int r = blockIdx.x * kBlock + threadIdx.x;
  if (r >= rows) return;
  const int lo = coff[inst[r]];
  int64_t j = (int64_t)pc[r] * 8;
  for (int q = ptr[r]; q < ptr[r + 1]; ++q, ++j) {
    const int64_t ch = j >> 3, g = ch >> 5, l = ch & 31;
    const int e = (int)(j & 7);
    if (scol) scol[j] = (uint16_t)(col[q] - lo);
    sval[((g * (8 / S) + e / S) * 32 + l) * S + e % S] = val[q];
  }
}

template <typename V>
struct EpiStoreB {  // y = M x (optionally / ||z_k||)
  V* y;
  const double* zz;  // per-instance squared norm, or null
  __device__ __forceinline__ void operator()(int i, int k, V acc) const {
    y[i] = zz ? (V)((double)acc / sqrt(zz[k])) : acc;
  }
};

struct Scal {  // per-instance iteration scalars
  const double *sigma, *lam, *lamQ;
  const int* restart_iter;
  int iter;
  __device__ __forceinline__ void halpern(int k, double& h1, double& h2) const {
    h1 = 1.0 / ((double)(iter - restart_iter[k]) + 2.0);
    h2 = 1.0 - h1;
  }
};

// LASSO step, per instance (update_zxw_LASSO_cpu!, src/kernels.jl:2400-2496)
template <typename V, bool Full>
struct EpiLassoB {
  V *x, *x_hat, *w_bar, *w, *dx, *x_bar, *z_bar, *dw;
  const V* c;
  const double *last_x, *last_w;
  Scal S;
  __device__ __forceinline__ void operator()(int i, int k, V acc) const {
    double h1, h2;
    S.halpern(k, h1, h2);
    const double sigma = S.sigma[k];
    const double f2s = 1.0 / (1.0 + sigma * S.lamQ[k]), f1s = 1.0 - f2s;
    const double x_i = x[i], w_i = w[i];
    const double tmp = -(double)acc + 0.0 - (double)c[i];
    const double z_raw = x_i + sigma * tmp;
    const double shrink = fmax(fabs(z_raw) - S.lam[k] * sigma, 0.0);
    const double xb = copysign(shrink, z_raw);
    const double xh = 2.0 * xb - x_i;
    const double xn = fma(h2, xh, h1 * last_x[i]);
    const double wb = fma(f1s, w_i, f2s * xh);
    const double wn = fma(h2, 2.0 * wb - w_i, h1 * last_w[i]);
    if (Full) {
      dx[i] = (V)(xb - x_i);
      x_bar[i] = (V)xb;
      z_bar[i] = (V)((xb - z_raw) / sigma);
      dw[i] = (V)(wb - w_i);
    }
    x[i] = (V)xn;
    x_hat[i] = (V)xh;
    w_bar[i] = (V)wb;
    w[i] = (V)wn;
  }
};

// Segmented reduction over tiles: each CTA owns one tile (instance, rows
// [b, e)); Epi(i, k, acc, r) adds to K slots (MaxMask selects max).
template <int K, unsigned MM, typename V, int TPR = 1, typename Src, typename Epi>
__global__ void __launch_bounds__(kBlock) k_seg(const int* tile_inst, const int* tile_begin, const int* tile_end,
                                                Inst I, Src src, Epi epi, double* partials) {
  pdl_enter();
  const int t = blockIdx.x;
  const int k = tile_inst[t];
  double r[K];
#pragma unroll
  for (int j = 0; j < K; ++j) r[j] = 0.0;
  if (I.on[k]) {  // TPR threads per row (the row schedule of the source matrix)
    const int lane = threadIdx.x & (TPR - 1);
    for (int i = tile_begin[t] + (int)threadIdx.x / TPR; i < tile_end[t]; i += kBlock / TPR) {
      const double acc = src.template dot<TPR, double>(i, lane);
      if (lane == 0) epi(i, k, acc, r);
    }
  }
  block_reduce<K, MM>(r);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int j = 0; j < K; ++j) partials[(size_t)t * K + j] = r[j];
  }
}

// Fold: one warp per instance sums its tiles (fixed order) into out[k*K + j];
// an optional finaliser turns them into derived scalars.
template <int K, unsigned MM, typename Fin>
__global__ void k_fold(int B, const int* inst_tiles, const unsigned char* on, const double* partials, double* out,
                       Fin fin) {
  pdl_enter();
  const int k = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (k >= B || !on[k]) return;
  const int t0 = inst_tiles[k], t1 = inst_tiles[k + 1];
  double acc[K];
#pragma unroll
  for (int j = 0; j < K; ++j) acc[j] = 0.0;
  for (int t = t0 + lane; t < t1; t += 32)
#pragma unroll
    for (int j = 0; j < K; ++j) {
      const double v = partials[(size_t)t * K + j];
      acc[j] = ((MM >> j) & 1u) ? fmax(acc[j], v) : acc[j] + v;
    }
#pragma unroll
  for (int j = 0; j < K; ++j)
    for (int off = 16; off > 0; off >>= 1) {
      const double o = __shfl_down_sync(0xffffffffu, acc[j], off);
      acc[j] = ((MM >> j) & 1u) ? fmax(acc[j], o) : acc[j] + o;
    }
  if (lane == 0) {
#pragma unroll
    for (int j = 0; j < K; ++j) out[(size_t)k * K + j] = acc[j];
    fin(k, acc);
  }
}

struct NoFinB {
  template <int K>
  __device__ void operator()(int, const double (&)[K]) const {}
};

// residual slots: 0 c'x 1 x'Qx 2 z'x 3 |lam x|_1 4 |Rd|inf 5 |Qx|inf   (acc = (Q x_bar)_i)
template <typename V>
struct EpiResB {
  const V *x_bar, *c, *z_bar;
  const double* lam;  // L1 weights (problem_type LASSO) or null
  __device__ __forceinline__ void operator()(int i, int k, double qx, double (&r)[6]) const {
    const double xb = x_bar[i], ci = c[i], zb = z_bar[i];
    r[0] += ci * xb;
    r[1] += xb * qx;
    r[2] += zb * xb;
    if (lam) r[3] += fabs(lam[k] * xb);
    r[4] = fmax(r[4], fabs(qx + ci - zb));
    r[5] = fmax(r[5], fabs(qx));
  }
};
constexpr unsigned kResMax = (1u << 4) | (1u << 5);

// M-norm (m = 0): 0 dx.dx 1 dQw.dx 2 dw.dQw    (acc = (Q dw)_i)
template <typename V>
struct EpiMnormB {
  const V *dx, *dw;
  __device__ __forceinline__ void operator()(int i, int, double dqw, double (&r)[3]) const {
    const double a = dx[i], b = dw[i];
    r[0] += a * a;
    r[1] += dqw * a;
    r[2] += b * dqw;
  }
};

// sigma statistics (m = 0): dx = x_bar - last_x, dw = w_bar - last_w written
// first by k_sigma_diff; here 0 dx.dx 1 dw.dQw  (acc = (Q dw)_i)
template <typename V>
struct EpiSigB {
  const V *dx, *dw;
  __device__ __forceinline__ void operator()(int i, int, double dqw, double (&r)[2]) const {
    const double a = dx[i];
    r[0] += a * a;
    r[1] += (double)dw[i] * dqw;
  }
};

// power method: z_next = (Q z)/||z||, sums q.z_next, z_next.z_next, q.q
template <typename V>
struct EpiPowB {
  const V* zc;
  V* zn;
  const double* zz;
  __device__ __forceinline__ void operator()(int i, int k, double acc, double (&r)[3]) const {
    const double inv = 1.0 / sqrt(zz[k]);
    const double v = acc;  // the A_d product already carried 1/||z||
    zn[i] = (V)v;
    const double q = (double)zc[i] * inv;
    r[0] += q * v;
    r[1] += v * v;
    r[2] += q * q;
  }
};

struct PowFinB {  // per instance: lambda, err into the log; zz for the next step
  double* zz;
  double* log;  // [kPowWin][B][2]
  int B, step;
  __device__ void operator()(int k, const double (&a)[3]) const {
    const double lam = a[0], z2 = a[1], qq = a[2];
    const double rr = fmax(z2 - 2.0 * lam * lam + lam * lam * qq, 0.0);
    log[2 * ((size_t)step * B + k)] = lam;
    log[2 * ((size_t)step * B + k) + 1] = sqrt(rr) / (sqrt(z2) + lam);
    zz[k] = z2;
  }
  template <int K>
  __device__ void operator()(int, const double (&)[K]) const {}
};

template <typename V>
struct EpiSumSqB {
  const V* z;
  __device__ __forceinline__ void operator()(int i, int, double, double (&r)[1]) const {
    const double t = z[i];
    r[0] += t * t;
  }
};

struct ZzFin {
  double* zz;
  __device__ void operator()(int k, const double (&a)[1]) const { zz[k] = a[0]; }
  template <int K>
  __device__ void operator()(int, const double (&)[K]) const {}
};

template <typename V>
struct CastVal {  // dst[i] = (V) src[i]
  V* dst;
  const double* src;
  __device__ __forceinline__ void operator()(int i) const { dst[i] = (V)src[i]; }
};

template <typename F>
__global__ void k_each(int len, F f) {
  pdl_enter();
  const int i = blockIdx.x * kBlock + threadIdx.x;
  if (i < len) f(i);
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
struct Mem : PoolBlocks {  // blocks of the library's device memory pool
  template <typename T>
  T* alloc(int64_t n) {  // zeroed, complete on return (the engines' streams do
                         // not wait for the legacy stream that runs cudaMemset)
    T* p = alloc_raw<T>(n);
    HPRQP_CUDA(cudaMemset(p, 0, sizeof(T) * (size_t)std::max<int64_t>(n, 1)));
    HPRQP_CUDA(cudaStreamSynchronize(cudaStreamLegacy));
    return p;
  }
  template <typename T>
  T* alloc_raw(int64_t n) {  // for buffers that are written in full right away
    return (T*)get(sizeof(T) * (size_t)std::max<int64_t>(n, 1));
  }
};

struct Tiles {  // reduction tiles over a concatenated row space
  int* inst = nullptr;
  int* begin = nullptr;
  int* end = nullptr;
  int* inst_tiles = nullptr;  // [B+1]
  int count = 0;
};

// A host CSR in plain arrays, left uninitialised at allocation: the batch
// intake fills them in parallel, one instance block per thread, so the
// first touch of the pages is parallel too.
struct FlatCsr {
  int64_t rows = 0, cols = 0, nz = 0;
  std::unique_ptr<int[]> ptr, col;
  std::unique_ptr<double[]> val;
  void alloc(int64_t r, int64_t c, int64_t z) {
    rows = r;
    cols = c;
    nz = z;
    ptr.reset(new int[r + 1]);
    col.reset(new int[std::max<int64_t>(z, 1)]);
    val.reset(new double[std::max<int64_t>(z, 1)]);
    ptr[0] = 0;
  }
  int64_t nnz() const { return nz; }
};

struct Family {  // host copy of the batch
  int B = 0;
  int64_t N = 0, R = 0;                 // total columns (variables), total data rows
  std::vector<int64_t> noff, roff;      // [B+1]
  FlatCsr L, LT;                        // block diagonal
  std::vector<double> c, lam;
  std::vector<double> obj_constant, norm_c_org;
};

// A batch matrix's staged copy (k_bstage_pass) on the device
template <typename V>
struct BStage {
  bool built = false, use = false;
  int ntile = 0, ncol_max = 0;
  int64_t chunks = 0;
  const int* pc = nullptr;  // each row's first chunk (for a copy in the other precision)
  BStageView<V> v{};
};

// the dynamic shared-memory limit of a kernel raised once per device
template <typename K>
static void raise_smem(K kernel, int bytes) {
  static std::atomic<uint64_t> done{0};
  int dev = 0;
  HPRQP_CUDA(cudaGetDevice(&dev));
  const uint64_t bit = 1ull << (dev & 63);
  if (done.load() & bit) return;
  HPRQP_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  done.fetch_or(bit);
}

template <typename V>
struct BEngine {
  cudaStream_t st = nullptr;
  Mem mem;
  int B;
  int64_t N, R;
  DCsr<V> L, LT;
  BStage<V> SL, SLT;  // staged copies of L and LT (built when their rows are long enough)
  int tprL = 8, tprLT = 4;
  V *x, *x_hat, *x_bar, *dx, *w, *w_bar, *dw, *z_bar, *c, *ltemp, *Qv, *pz, *pq;
  double *last_x, *last_w;
  int *inst_n, *inst_r;
  unsigned char* on;     // active in this engine
  unsigned char* on_pw;  // active in the power method
  double *sigma, *lam, *lamQ, *zz, *plog, *stage;
  int* restart_iter;
  double* partials;  // [tiles * K]
  double *out_res, *out_mn_cur, *out_mn_last, *out_sig, *out_tmp;  // [B * K] each
  Tiles tn;
  int64_t launches = 0;

  // A CSR on the device.  With `from` (the FP64 engine's copy of the same
  // matrix) the pattern arrays are shared and the values cast on the device,
  // so the FP32 engine moves nothing across PCIe.
  void upload_csr(const FlatCsr& h, DCsr<V>& d, const DCsr<double>* from = nullptr) {
    d.rows = (int)h.rows;
    d.cols = (int)h.cols;
    d.nnz = h.nnz();
    V* v = mem.alloc_raw<V>(d.nnz);
    if (from) {
      d.ptr = from->ptr;
      d.col = from->col;
      const double* src = from->val;
      if (d.nnz) {
        k_each<<<(int)((d.nnz + kBlock - 1) / kBlock), kBlock, 0, st>>>((int)d.nnz,
                                                                        CastVal<V>{v, src});
        HPRQP_LAUNCH_CHECK();
        HPRQP_CUDA(cudaStreamSynchronize(st));
      }
      d.val = v;
      return;
    }
    int* p = mem.alloc_raw<int>(h.rows + 1);
    int* cc = mem.alloc_raw<int>(d.nnz);
    h2d_staged(p, h.ptr.get(), sizeof(int) * (h.rows + 1), st);
    if (d.nnz) h2d_staged(cc, h.col.get(), sizeof(int) * d.nnz, st);
    if (d.nnz) {
      if constexpr (std::is_same<V, double>::value) {
        h2d_staged(v, h.val.get(), sizeof(V) * d.nnz, st);
      } else {
        std::vector<V> vv(d.nnz);
#pragma omp parallel for schedule(static) num_threads(host_threads(d.nnz))
        for (int64_t q = 0; q < d.nnz; ++q) vv[q] = (V)h.val[q];
        h2d_staged(v, vv.data(), sizeof(V) * d.nnz, st);
      }
    }
    HPRQP_CUDA(cudaStreamSynchronize(st));
    d.ptr = p;
    d.col = cc;
    d.val = v;
  }
  template <typename T>
  T* up(const std::vector<T>& h) {
    if (h.empty()) return mem.alloc<T>(0);
    T* d = mem.alloc_raw<T>((int64_t)h.size());
    h2d_staged(d, h.data(), sizeof(T) * h.size(), st);
    HPRQP_CUDA(cudaStreamSynchronize(st));
    return d;
  }

  BEngine(const Family& F, cudaStream_t s, const DCsr<double>* L64 = nullptr, const DCsr<double>* LT64 = nullptr,
          const BStage<double>* SL64 = nullptr, const BStage<double>* SLT64 = nullptr)
      : st(s), B(F.B), N(F.N), R(F.R) {
    upload_csr(F.L, L, L64);
    upload_csr(F.LT, LT, LT64);
    const double avg = F.R ? (double)F.L.nnz() / F.R : 1.0;
    tprL = avg > 48 ? 32 : avg > 24 ? 16 : avg > 12 ? 8 : avg > 6 ? 4 : 2;
    for (V** p : {&x, &x_hat, &x_bar, &dx, &w, &w_bar, &dw, &z_bar, &Qv, &pz, &pq}) *p = mem.alloc<V>(N);
    ltemp = mem.alloc<V>(R);
    last_x = mem.alloc<double>(N);
    last_w = mem.alloc<double>(N);
    stage = mem.alloc<double>(N);
    c = up(std::vector<V>(F.c.begin(), F.c.end()));
    std::vector<int> in(N), ir(R);
    for (int k = 0; k < B; ++k) {
      for (int64_t i = F.noff[k]; i < F.noff[k + 1]; ++i) in[i] = k;
      for (int64_t i = F.roff[k]; i < F.roff[k + 1]; ++i) ir[i] = k;
    }
    inst_n = up(in);
    inst_r = up(ir);
    const char* bst = std::getenv("HPRQP_BATCH_STAGED");
    if (!(bst && bst[0] == '0')) {
      build_bstage(F.L, L, F.roff, F.noff, inst_r, SL, SL64);
      build_bstage(F.LT, LT, F.noff, F.roff, inst_n, SLT, SLT64);
    }
    on = mem.alloc<unsigned char>(B);
    on_pw = mem.alloc<unsigned char>(B);
    sigma = mem.alloc<double>(B);
    lam = up(F.lam);
    lamQ = mem.alloc<double>(B);
    zz = mem.alloc<double>(B);
    plog = mem.alloc<double>(2 * (int64_t)B * kPowWin);
    restart_iter = mem.alloc<int>(B);
    // tiles over the variable rows
    std::vector<int> ti, tb, te, it(B + 1, 0);
    for (int k = 0; k < B; ++k) {
      it[k] = (int)ti.size();
      for (int64_t b = F.noff[k]; b < F.noff[k + 1]; b += kTileRows) {
        ti.push_back(k);
        tb.push_back((int)b);
        te.push_back((int)std::min<int64_t>(b + kTileRows, F.noff[k + 1]));
      }
    }
    it[B] = (int)ti.size();
    tn.count = (int)ti.size();
    tn.inst = up(ti);
    tn.begin = up(tb);
    tn.end = up(te);
    tn.inst_tiles = up(it);
    partials = mem.alloc<double>((int64_t)tn.count * kMaxK);
    for (double** o : {&out_res, &out_mn_cur, &out_mn_last, &out_sig, &out_tmp}) *o = mem.alloc<double>((int64_t)B * kMaxK);
    autotune();
  }

  // Staged copy of a block-diagonal batch matrix M (rows of instance k in
  // [rof[k], rof[k+1]), its columns in [cof[k], cof[k+1])): chunk counts from
  // the host pattern, tiles of whole rows of one instance with at most
  // kStageSlots slots, each starting at a whole warp tile; the scatter on the
  // device from M's device CSR.  Not built when an instance has more
  // columns than 16 bits index or its block does not fit a CTA's shared
  // memory, or when rows average fewer than 8 entries (padding to 8-entry
  // chunks would cost more than the staging saves).
  void build_bstage(const FlatCsr& h, const DCsr<V>& M, const std::vector<int64_t>& rof,
                    const std::vector<int64_t>& cof, const int* inst, BStage<V>& S,
                    const BStage<double>* from = nullptr) {
    S = BStage<V>();
    const int64_t rows = h.rows;
    if (from) {  // the FP64 engine's structure: only the values in this precision
      if (!from->built) return;
      if ((int64_t)from->ncol_max * (int64_t)sizeof(V) > kStageSmem) return;
      V* sval = mem.alloc_raw<V>(from->chunks * 8);
      if (reinterpret_cast<uintptr_t>(sval) & 15u) return;
      HPRQP_CUDA(cudaMemsetAsync(sval, 0, sizeof(V) * (size_t)from->chunks * 8, st));
      k_bstage_fill<V><<<(int)((rows + kBlock - 1) / kBlock), kBlock, 0, st>>>(
          (int)rows, M.ptr, M.col, M.val, inst, from->v.coff, from->pc, nullptr, sval);
      HPRQP_LAUNCH_CHECK();
      const BStageView<double>& f = from->v;
      S.v = BStageView<V>{f.col, sval, f.wt, f.tile, f.tinst, f.srow, f.coff, f.ncol};
      S.ntile = from->ntile;
      S.ncol_max = from->ncol_max;
      S.chunks = from->chunks;
      S.pc = from->pc;
      HPRQP_CUDA(cudaStreamSynchronize(st));
      S.built = true;
      return;
    }
    if (rows <= 0 || h.nnz() < 65536 || (double)h.nnz() / (double)rows < 8.0) return;
    int ncol_max = 0;
    for (int k = 0; k < B; ++k) ncol_max = std::max<int>(ncol_max, (int)(cof[k + 1] - cof[k]));
    if (ncol_max > 65535 || (int64_t)ncol_max * (int64_t)sizeof(V) > kStageSmem) return;
    std::vector<int> ch(rows), pc(rows), srow(rows + 1);
    // each instance planned on its own (local warp-tile and slot numbers),
    // in parallel; then shifted by the instances' prefix offsets
    struct Plan {
      std::vector<int4> tiles;
      std::vector<int2> wts;
      int64_t nslot = 0;
      bool ok = true;
    };
    std::vector<Plan> plans(B);
#pragma omp parallel for schedule(dynamic, 4) num_threads(host_threads(rows))
    for (int k = 0; k < B; ++k) {
      Plan& P = plans[k];
      std::vector<unsigned> heads;
      std::vector<int> first;
      for (int64_t r = rof[k]; r < rof[k + 1]; ++r) {
        const int len = h.ptr[r + 1] - h.ptr[r];
        ch[r] = len > 0 ? (len + 7) / 8 : 1;
      }
      int64_t q = rof[k], slot = 0;
      while (q < rof[k + 1]) {  // one tile from row q
        const int64_t r0 = q;
        int64_t o = 0, slots = 0;
        while (q < rof[k + 1]) {
          const int64_t touch = (o + ch[q] - 1) / 32 - o / 32 + 1;
          if (slots + touch > kStageSlots) break;
          slots += touch;
          o += ch[q];
          ++q;
        }
        if (q == r0) {  // a row with more slots than a tile holds
          P.ok = false;
          break;
        }
        const int nwt = (int)((o + 31) / 32);
        heads.assign(nwt, 0u);
        first.assign(nwt, -1);
        int64_t off = 0;
        for (int64_t rr = r0; rr < q; ++rr) {
          srow[rr] = (int)slot;
          pc[rr] = (int)(32 * (int64_t)P.wts.size() + off);
          for (int64_t w = off / 32; w <= (off + ch[rr] - 1) / 32; ++w) {
            heads[w] |= 1u << (std::max<int64_t>(off, 32 * w) - 32 * w);
            if (first[w] < 0) first[w] = (int)slot;
            ++slot;
          }
          off += ch[rr];
        }
        P.tiles.push_back(make_int4((int)P.wts.size(), (int)o, (int)r0, (int)q));
        for (int w = 0; w < nwt; ++w) P.wts.push_back(make_int2(first[w], (int)heads[w]));
      }
      P.nslot = slot;
    }
    std::vector<int64_t> wb(B + 1, 0), sb(B + 1, 0), tb(B + 1, 0);
    for (int k = 0; k < B; ++k) {
      if (!plans[k].ok) return;
      wb[k + 1] = wb[k] + (int64_t)plans[k].wts.size();
      sb[k + 1] = sb[k] + plans[k].nslot;
      tb[k + 1] = tb[k] + (int64_t)plans[k].tiles.size();
    }
    if (32 * wb[B] > INT32_MAX / 8 || sb[B] > INT32_MAX / 2) return;
    std::vector<int2> wt(wb[B]);
    std::vector<int4> tile(tb[B]);
    std::vector<int> tinst(tb[B]);
#pragma omp parallel for schedule(dynamic, 4) num_threads(host_threads(rows))
    for (int k = 0; k < B; ++k) {
      const Plan& P = plans[k];
      for (size_t i = 0; i < P.tiles.size(); ++i) {
        const int4 t = P.tiles[i];
        tile[tb[k] + (int64_t)i] = make_int4((int)(t.x + wb[k]), t.y, t.z, t.w);
        tinst[tb[k] + (int64_t)i] = k;
      }
      for (size_t j = 0; j < P.wts.size(); ++j)
        wt[wb[k] + (int64_t)j] = make_int2((int)(P.wts[j].x + sb[k]), P.wts[j].y);
      for (int64_t rr = rof[k]; rr < rof[k + 1]; ++rr) {
        srow[rr] += (int)sb[k];
        pc[rr] += (int)(32 * wb[k]);
      }
    }
    srow[rows] = (int)sb[B];
    const int64_t tot = 32 * wb[B];
    std::vector<int> co(B), nc(B);
    for (int k = 0; k < B; ++k) {
      co[k] = (int)cof[k];
      nc[k] = (int)(cof[k + 1] - cof[k]);
    }
    uint16_t* scol = mem.alloc_raw<uint16_t>(tot * 8);
    V* sval = mem.alloc_raw<V>(tot * 8);
    if ((reinterpret_cast<uintptr_t>(scol) | reinterpret_cast<uintptr_t>(sval)) & 15u) return;
    HPRQP_CUDA(cudaMemsetAsync(scol, 0, sizeof(uint16_t) * (size_t)tot * 8, st));
    HPRQP_CUDA(cudaMemsetAsync(sval, 0, sizeof(V) * (size_t)tot * 8, st));
    const int* dpc = up(pc);
    const int* dco = up(co);
    k_bstage_fill<V><<<(int)((rows + kBlock - 1) / kBlock), kBlock, 0, st>>>((int)rows, M.ptr, M.col, M.val, inst,
                                                                             dco, dpc, scol, sval);
    HPRQP_LAUNCH_CHECK();
    S.v = BStageView<V>{scol, sval, up(wt), up(tile), up(tinst), up(srow), dco, up(nc)};
    S.ntile = (int)tile.size();
    S.ncol_max = ncol_max;
    S.chunks = tot;
    S.pc = dpc;
    HPRQP_CUDA(cudaStreamSynchronize(st));
    S.built = true;
  }
  template <typename Epi>
  void rows_stage(const BStage<V>& S, const V* xin, const Epi& e, const unsigned char* mask) {
    const int smem = (int)(sizeof(V) * ((size_t)kStageSlots + (size_t)S.ncol_max));
    raise_smem(k_bstage_pass<V, Epi>, (int)(sizeof(V) * kStageSlots) + kStageSmem);
    k_bstage_pass<V, Epi><<<S.ntile, kBStageBlock, smem, st>>>(S.v, xin, mask, e);
    launches++;
    HPRQP_LAUNCH_CHECK();
  }
  template <typename Epi>
  void rows_csr(const DCsr<V>& M, const int* inst, int tpr, const V* xin, const Epi& e, const unsigned char* mask) {
    const Inst I{inst, mask};
    const CsrSrc<V, V> s{M.ptr, M.col, M.val, xin};
    const long long threads = (long long)M.rows * tpr;
    const int grid = (int)((threads + kBlock - 1) / kBlock);
    switch (tpr) {
      case 1: k_rows<1, V><<<grid, kBlock, 0, st>>>(M.rows, I, s, e); break;
      case 2: k_rows<2, V><<<grid, kBlock, 0, st>>>(M.rows, I, s, e); break;
      case 4: k_rows<4, V><<<grid, kBlock, 0, st>>>(M.rows, I, s, e); break;
      case 8: k_rows<8, V><<<grid, kBlock, 0, st>>>(M.rows, I, s, e); break;
      case 16: k_rows<16, V><<<grid, kBlock, 0, st>>>(M.rows, I, s, e); break;
      default: k_rows<32, V><<<grid, kBlock, 0, st>>>(M.rows, I, s, e); break;
    }
    launches++;
    HPRQP_LAUNCH_CHECK();
  }
  template <typename Epi>
  void rows_L(const V* xin, const Epi& e, const unsigned char* mask) {
    if (SL.use) rows_stage(SL, xin, e, mask);
    else rows_csr(L, inst_r, tprL, xin, e, mask);
  }
  template <typename Epi>
  void rows_LT(const V* xin, const Epi& e) {
    if (SLT.use) rows_stage(SLT, xin, e, on);
    else rows_csr(LT, inst_n, tprLT, xin, e, on);
  }
  // Row-schedule autotuner for this instance class: threads per row of the
  // A_d and A_d' products, the fastest of 3 timed rounds of 3 launches each
  // (all instances active, plain products into scratch).
  void autotune() {
    unsigned char* all = mem.alloc<unsigned char>(B);
    HPRQP_CUDA(cudaMemsetAsync(all, 1, B, st));
    cudaEvent_t a, b;
    HPRQP_CUDA(cudaEventCreate(&a));
    HPRQP_CUDA(cudaEventCreate(&b));
    auto tune = [&](const DCsr<V>& M, const int* inst, const V* xin, V* out, std::initializer_list<int> cands) {
      float best = 1e30f;
      int bt = *cands.begin();
      for (int t : cands) {
        rows_csr(M, inst, t, xin, EpiStoreB<V>{out, nullptr}, all);
        float tb = 1e30f;
        for (int r = 0; r < 3; ++r) {
          HPRQP_CUDA(cudaEventRecord(a, st));
          for (int q = 0; q < 3; ++q) rows_csr(M, inst, t, xin, EpiStoreB<V>{out, nullptr}, all);
          HPRQP_CUDA(cudaEventRecord(b, st));
          HPRQP_CUDA(cudaEventSynchronize(b));
          float ms = 0;
          HPRQP_CUDA(cudaEventElapsedTime(&ms, a, b));
          tb = std::min(tb, ms);
        }
        if (tb < best) { best = tb; bt = t; }
      }
      return bt;
    };
    tprL = tune(L, inst_r, pz, ltemp, {2, 4, 8, 16, 32});
    tprLT = tune(LT, inst_n, ltemp, Qv, {1, 2, 4, 8, 16});
    // the staged copies against the best CSR schedule, timed the same way
    auto time_of = [&](auto&& launch) {
      launch();
      float tb = 1e30f;
      for (int r = 0; r < 3; ++r) {
        HPRQP_CUDA(cudaEventRecord(a, st));
        for (int q = 0; q < 3; ++q) launch();
        HPRQP_CUDA(cudaEventRecord(b, st));
        HPRQP_CUDA(cudaEventSynchronize(b));
        float ms = 0;
        HPRQP_CUDA(cudaEventElapsedTime(&ms, a, b));
        tb = std::min(tb, ms);
      }
      return tb;
    };
    // (HPRQP_BATCH_STAGED=1 takes them untimed)
    const char* bs = std::getenv("HPRQP_BATCH_STAGED");
    const bool force = bs && bs[0] == '1';
    if (SL.built)
      SL.use = force || time_of([&] { rows_stage(SL, pz, EpiStoreB<V>{ltemp, nullptr}, all); }) <
                            time_of([&] { rows_csr(L, inst_r, tprL, pz, EpiStoreB<V>{ltemp, nullptr}, all); });
    if (SLT.built)
      SLT.use = force || time_of([&] { rows_stage(SLT, ltemp, EpiStoreB<V>{Qv, nullptr}, all); }) <
                             time_of([&] { rows_csr(LT, inst_n, tprLT, ltemp, EpiStoreB<V>{Qv, nullptr}, all); });
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    launches = 0;
  }
  // segmented reduction with the A_d' product as the row source, then fold
  template <int K, unsigned MM, typename Epi, typename Fin = NoFinB>
  void seg_LT(const V* xin, const Epi& e, const unsigned char* mask, double* dst, const Fin& fin = Fin()) {
    const Inst I{inst_n, mask};
    const CsrSrc<V, V> src{LT.ptr, LT.col, LT.val, xin};
    switch (tprLT) {
      case 1: k_seg<K, MM, V, 1><<<tn.count, kBlock, 0, st>>>(tn.inst, tn.begin, tn.end, I, src, e, partials); break;
      case 2: k_seg<K, MM, V, 2><<<tn.count, kBlock, 0, st>>>(tn.inst, tn.begin, tn.end, I, src, e, partials); break;
      case 4: k_seg<K, MM, V, 4><<<tn.count, kBlock, 0, st>>>(tn.inst, tn.begin, tn.end, I, src, e, partials); break;
      case 8: k_seg<K, MM, V, 8><<<tn.count, kBlock, 0, st>>>(tn.inst, tn.begin, tn.end, I, src, e, partials); break;
      default: k_seg<K, MM, V, 16><<<tn.count, kBlock, 0, st>>>(tn.inst, tn.begin, tn.end, I, src, e, partials); break;
    }
    k_fold<K, MM><<<(B + 7) / 8, 256, 0, st>>>(B, tn.inst_tiles, mask, partials, dst, fin);
    launches += 2;
    HPRQP_LAUNCH_CHECK();
  }
  template <int K, unsigned MM, typename Epi, typename Fin = NoFinB>
  void seg_plain(const Epi& e, const unsigned char* mask, double* dst, const Fin& fin = Fin()) {
    const Inst I{inst_n, mask};
    k_seg<K, MM, V><<<tn.count, kBlock, 0, st>>>(tn.inst, tn.begin, tn.end, I, ZeroSrc{}, e, partials);
    k_fold<K, MM><<<(B + 7) / 8, 256, 0, st>>>(B, tn.inst_tiles, mask, partials, dst, fin);
    launches += 2;
    HPRQP_LAUNCH_CHECK();
  }
  template <typename F>
  void each(int64_t len, const F& f) {
    if (len <= 0) return;
    k_each<<<(int)((len + kBlock - 1) / kBlock), kBlock, 0, st>>>((int)len, f);
    launches++;
    HPRQP_LAUNCH_CHECK();
  }

  void step(bool full, int iter) {
    rows_L(w, EpiStoreB<V>{ltemp, nullptr}, on);
    const Scal S{sigma, lam, lamQ, restart_iter, iter};
    if (full)
      rows_LT(ltemp, EpiLassoB<V, true>{x, x_hat, w_bar, w, dx, x_bar, z_bar, dw, c, last_x, last_w, S});
    else
      rows_LT(ltemp, EpiLassoB<V, false>{x, x_hat, w_bar, w, dx, x_bar, z_bar, dw, c, last_x, last_w, S});
  }
  void residuals(bool lasso_obj, const unsigned char* mask) {  // -> out_res[k*6 + j]
    rows_L(x_bar, EpiStoreB<V>{ltemp, nullptr}, mask);
    seg_LT<6, kResMax>(ltemp, EpiResB<V>{x_bar, c, z_bar, lasso_obj ? lam : nullptr}, mask, out_res);
  }
  void mnorm(double* dst) {  // -> dst[k*3 + j]
    rows_L(dw, EpiStoreB<V>{ltemp, nullptr}, on);
    seg_LT<3, 0u>(ltemp, EpiMnormB<V>{dx, dw}, on, dst);
  }
  void sigma_stats(const unsigned char* mask) {  // -> out_sig[k*2 + j]
    V *dx_ = dx, *dw_ = dw;
    const V *xb = x_bar, *wb = w_bar;
    const double *lx = last_x, *lw = last_w;
    const int* in = inst_n;
    const unsigned char* mk = mask;
    each(N, [=] __device__(int i) {
      if (!mk[in[i]]) return;
      dx_[i] = (V)((double)xb[i] - lx[i]);
      dw_[i] = (V)((double)wb[i] - lw[i]);
    });
    rows_L(dw, EpiStoreB<V>{ltemp, nullptr}, mask);
    seg_LT<2, 0u>(ltemp, EpiSigB<V>{dx, dw}, mask, out_sig);
  }
  void restart(const unsigned char* mask) {  // do_restart! for flagged instances
    V *x_ = x, *w_ = w;
    const V *xb = x_bar, *wb = w_bar;
    double *lx = last_x, *lw = last_w;
    const int* in = inst_n;
    const unsigned char* mk = mask;
    each(N, [=] __device__(int i) {
      if (!mk[in[i]]) return;
      x_[i] = xb[i];
      w_[i] = wb[i];
      lx[i] = (double)xb[i];
      lw[i] = (double)wb[i];
    });
  }
};

struct Handle {
  int device = 0;
  cudaStream_t st = nullptr;
  Family F;
  std::unique_ptr<BEngine<double>> e64;
  std::unique_ptr<BEngine<float>> e32;
  bqp::QpBatch* qp = nullptr;  // the QAP family (batch_qp.cu), when loaded
  bool qap = false;            // which family the handle holds
  std::string err;
  ~Handle() {
    e64.reset();
    e32.reset();
    if (qp) bqp::destroy(qp);
    if (st) cudaStreamDestroy(st);
  }
};

struct RI {  // per-instance restart record (HPRQP_restart)
  bool first = true;
  double save_gap = std::numeric_limits<double>::infinity(), current_gap = save_gap, last_gap = save_gap,
         best_gap = save_gap, best_sigma = 1.0, weighted = save_gap;
  int64_t inner = 0, times = 0;
  int flag = 0;
};

static double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}
static double print_step(int64_t iter) {
  return std::max(std::pow(10.0, std::floor(std::log10((double)iter))) / 10.0, 10.0);
}

template <typename V>
static std::vector<double> read(BEngine<V>& E, const double* d, int64_t count) {
  std::vector<double> h(count);
  HPRQP_CUDA(cudaMemcpyAsync(h.data(), d, sizeof(double) * count, cudaMemcpyDeviceToHost, E.st));
  HPRQP_CUDA(cudaStreamSynchronize(E.st));
  return h;
}

// lambda_max(A_k' A_k) for every instance, in lockstep (power_iteration_Q,
// src/utils.jl:1419-1461, same start-vector stream per instance).
template <typename V>
static std::vector<double> power_batch(BEngine<V>& E, const Family& F, double tol, int max_it) {
  const int B = F.B;
  {  // every instance's start vector, generated in place
    PoolBlocks tmp;
    int64_t* off = (int64_t*)tmp.get(sizeof(int64_t) * (B + 1));
    HPRQP_CUDA(cudaMemcpyAsync(off, F.noff.data(), sizeof(int64_t) * (B + 1), cudaMemcpyHostToDevice, E.st));
    k_start_vector_seg<V><<<(int)((E.N + kBlock - 1) / kBlock), kBlock, 0, E.st>>>(B, off, E.N, E.pz);
    HPRQP_LAUNCH_CHECK();
    HPRQP_CUDA(cudaStreamSynchronize(E.st));
  }
  std::vector<unsigned char> act(B, 1);
  HPRQP_CUDA(cudaMemcpyAsync(E.on_pw, act.data(), B, cudaMemcpyHostToDevice, E.st));
  HPRQP_CUDA(cudaStreamSynchronize(E.st));
  E.template seg_plain<1, 0u>(EpiSumSqB<V>{E.pz}, E.on_pw, E.out_tmp, ZzFin{E.zz});
  std::vector<double> lam(B, 1.0);
  std::vector<int> done(B, 0);
  int remaining = B;
  for (int it = 0; it < max_it && remaining > 0; ++it) {
    V* zc = (it & 1) ? E.pq : E.pz;
    V* zn = (it & 1) ? E.pz : E.pq;
    const int w = it % kPowWin;
    E.rows_L(zc, EpiStoreB<V>{E.ltemp, E.zz}, E.on_pw);
    E.template seg_LT<3, 0u>(E.ltemp, EpiPowB<V>{zc, zn, E.zz}, E.on_pw, E.out_tmp, PowFinB{E.zz, E.plog, B, w});
    if (w == kPowWin - 1 || it == max_it - 1) {
      std::vector<double> lg = read(E, E.plog, 2 * (int64_t)B * kPowWin);
      bool changed = false;
      for (int k = 0; k < B; ++k) {
        if (done[k]) continue;
        for (int s2 = 0; s2 <= w; ++s2) {  // first step of the window with err < tol
          lam[k] = lg[2 * ((size_t)s2 * B + k)];
          if (lg[2 * ((size_t)s2 * B + k) + 1] < tol) {
            done[k] = 1;
            act[k] = 0;
            --remaining;
            changed = true;
            break;
          }
        }
      }
      if (changed) HPRQP_CUDA(cudaMemcpyAsync(E.on_pw, act.data(), B, cudaMemcpyHostToDevice, E.st));
    }
  }
  return lam;
}

}  // namespace batch
}  // namespace hprqp

namespace hprqp {
namespace batch {

// Warm start of the instances with a given x0 (zero elsewhere).
template <typename V>
struct InitX {
  V *x, *x_bar, *w, *w_bar;
  double *last_x, *last_w;
  const double* src;
  __device__ void operator()(int i) const {
    const V v = (V)src[i];
    x[i] = x_bar[i] = w[i] = w_bar[i] = v;
    last_x[i] = last_w[i] = (double)v;
  }
};

// Copy instance rows (mask) from the FP32 engine into the FP64 engine.
template <typename D, typename S>
struct CopyMasked {
  D* dst;
  const S* src;
  const int* inst;
  const unsigned char* mask;
  __device__ void operator()(int i) const {
    if (mask[inst[i]]) dst[i] = (D)src[i];
  }
};

// The family intake: offsets from the callers' CSC column pointers, then
// one parallel pass per instance that validates its arrays and writes its
// blocks of the concatenated A_d (CSR, by a counting sort of the CSC, which
// keeps the columns of a row in increasing order as load_problem does) and
// A_d' (the CSC read as CSR) in place.  An instance whose row indices are
// not sorted within a column goes through load_problem + transpose instead.
static void build_family(int count, const hprqp_problem* probs, Family& F) {
  if (count <= 0 || !probs) throw Error(HPRQP_E_ARG, "empty batch");
  F = Family();
  F.B = count;
  F.noff.assign(count + 1, 0);
  F.roff.assign(count + 1, 0);
  std::vector<int64_t> zoff(count + 1, 0);
  for (int k = 0; k < count; ++k) {
    const hprqp_problem& p = probs[k];
    if (p.Q_kind != HPRQP_Q_LASSO || p.m != 0)
      throw Error(HPRQP_E_ARG, "batch: every instance must be a LASSO problem (m = 0)");
    if (p.n <= 0 || p.n > INT32_MAX || p.lasso_m <= 0 || p.lasso_m > INT32_MAX || !p.L_colptr ||
        (p.index_base != 0 && p.index_base != 1))
      throw Error(HPRQP_E_ARG, "batch instance " + std::to_string(k) + ": bad sizes or data matrix");
    const int64_t z = (int64_t)p.L_colptr[p.n] - p.index_base;
    if (z < 0) throw Error(HPRQP_E_ARG, "batch instance " + std::to_string(k) + ": bad nnz");
    F.noff[k + 1] = F.noff[k] + p.n;
    F.roff[k + 1] = F.roff[k] + p.lasso_m;
    zoff[k + 1] = zoff[k] + z;
  }
  F.N = F.noff[count];
  F.R = F.roff[count];
  if (F.N > INT32_MAX || F.R > INT32_MAX || zoff[count] > INT32_MAX) throw Error(HPRQP_E_ARG, "batch too large");
  F.L.alloc(F.R, F.N, zoff[count]);
  F.LT.alloc(F.N, F.R, zoff[count]);
  F.c.resize(F.N);
  F.lam.resize(count);
  F.obj_constant.resize(count);
  F.norm_c_org.resize(count);
  std::vector<int> codes(count, 0);
  std::vector<std::string> errs(count);
#pragma omp parallel for schedule(dynamic, 1) num_threads(host_threads(zoff[count]))
  for (int k = 0; k < count; ++k) {
    try {
      const hprqp_problem& p = probs[k];
      const int base = p.index_base;
      const int64_t n = p.n, mk = p.lasso_m, z0 = zoff[k], no = F.noff[k], ro = F.roff[k];
      const int32_t *cp = p.L_colptr, *rv = p.L_rowval;
      const double* nz = p.L_nzval;
      const int64_t z = zoff[k + 1] - z0;
      if (z > 0 && (!rv || !nz)) throw Error(HPRQP_E_ARG, "null rowval/nzval");
      if (cp[0] != base) throw Error(HPRQP_E_ARG, "colptr[0] != index_base");
      bool sorted = true;
      for (int64_t j = 0; j < n; ++j) {
        if (cp[j + 1] < cp[j]) throw Error(HPRQP_E_ARG, "colptr not monotone");
        for (int64_t q = cp[j] - base; q < cp[j + 1] - base; ++q) {
          const int64_t r = (int64_t)rv[q] - base;
          if (r < 0 || r >= mk) throw Error(HPRQP_E_ARG, "row index out of range");
          if (!std::isfinite(nz[q])) throw Error(HPRQP_E_ARG, "LASSO data matrix contains NaN or Inf values.");
          if (q > cp[j] - base && rv[q] <= rv[q - 1]) sorted = false;
        }
      }
      int* Lp = F.L.ptr.get();
      int* Lc = F.L.col.get();
      double* Lv = F.L.val.get();
      int* Tp = F.LT.ptr.get();
      int* Tc = F.LT.col.get();
      double* Tv = F.LT.val.get();
      if (sorted) {
        // A_d' block: the CSC read as CSR, shifted by (noff, roff)
        for (int64_t j = 0; j < n; ++j) Tp[no + j + 1] = (int)(z0 + (cp[j + 1] - base));
        for (int64_t q = 0; q < z; ++q) {
          Tc[z0 + q] = (int)(rv[q] - base + ro);
          Tv[z0 + q] = nz[q];
        }
        // A_d block: counting sort of the CSC by row
        std::vector<int> pos(mk + 1, 0);
        for (int64_t q = 0; q < z; ++q) pos[rv[q] - base + 1]++;
        for (int64_t r = 0; r < mk; ++r) pos[r + 1] += pos[r];
        for (int64_t r = 0; r < mk; ++r) Lp[ro + r + 1] = (int)(z0 + pos[r + 1]);
        for (int64_t j = 0; j < n; ++j)
          for (int64_t q = cp[j] - base; q < cp[j + 1] - base; ++q) {
            const int r = rv[q] - base;
            const int64_t at = z0 + pos[r]++;
            Lc[at] = (int)(j + no);
            Lv[at] = nz[q];
          }
      } else {
        HostProblem hp;
        load_problem(&p, hp);
        const HCsr& Lk = hp.L;
        const HCsr Tk = transpose(Lk);
        for (int64_t r = 0; r < Lk.rows; ++r) Lp[ro + r + 1] = (int)(z0 + Lk.ptr[r + 1]);
        for (int64_t q = 0; q < Lk.nnz(); ++q) {
          Lc[z0 + q] = (int)(Lk.col[q] + no);
          Lv[z0 + q] = Lk.val[q];
        }
        for (int64_t r = 0; r < Tk.rows; ++r) Tp[no + r + 1] = (int)(z0 + Tk.ptr[r + 1]);
        for (int64_t q = 0; q < Tk.nnz(); ++q) {
          Tc[z0 + q] = (int)(Tk.col[q] + ro);
          Tv[z0 + q] = Tk.val[q];
        }
      }
      if (n > 0 && !p.c) throw Error(HPRQP_E_ARG, "c vector: null pointer");
      double nc = 0.0;
      for (int64_t j = 0; j < n; ++j) {
        const double v = p.c[j];
        if (!std::isfinite(v)) throw Error(HPRQP_E_ARG, "c vector contains NaN or Inf values.");
        F.c[no + j] = v;
        nc = std::max(nc, std::fabs(v));
      }
      F.norm_c_org[k] = nc;
      F.lam[k] = p.lambda;
      F.obj_constant[k] = p.obj_constant;
    } catch (const Error& e) {
      codes[k] = e.code;
      errs[k] = e.what();
    }
  }
  for (int k = 0; k < count; ++k)
    if (codes[k]) throw Error(codes[k], "batch instance " + std::to_string(k) + ": " + errs[k]);
}

template <typename V>
static void upload_scalars(BEngine<V>& E, const std::vector<double>& sigma, const std::vector<double>& lamQ,
                           const std::vector<int>& rit) {
  HPRQP_CUDA(cudaMemcpyAsync(E.sigma, sigma.data(), sizeof(double) * E.B, cudaMemcpyHostToDevice, E.st));
  HPRQP_CUDA(cudaMemcpyAsync(E.lamQ, lamQ.data(), sizeof(double) * E.B, cudaMemcpyHostToDevice, E.st));
  HPRQP_CUDA(cudaMemcpyAsync(E.restart_iter, rit.data(), sizeof(int) * E.B, cudaMemcpyHostToDevice, E.st));
}

template <typename V>
static void upload_mask(BEngine<V>& E, const std::vector<unsigned char>& on) {
  HPRQP_CUDA(cudaMemcpyAsync(E.on, on.data(), E.B, cudaMemcpyHostToDevice, E.st));
}

// initial points (process_initial_points!, operator Q: no scaling)
template <typename V>
static void init_engine(BEngine<V>& E, const Family& F, const double* const* x0s, const std::vector<unsigned char>& on,
                        const std::vector<double>& sigma, const std::vector<double>& lamQ, const std::vector<int>& rit) {
  V* vecs[] = {E.x, E.x_hat, E.x_bar, E.dx, E.w, E.w_bar, E.dw, E.z_bar};
  for (V* v : vecs) HPRQP_CUDA(cudaMemsetAsync(v, 0, sizeof(V) * E.N, E.st));
  HPRQP_CUDA(cudaMemsetAsync(E.last_x, 0, sizeof(double) * E.N, E.st));
  HPRQP_CUDA(cudaMemsetAsync(E.last_w, 0, sizeof(double) * E.N, E.st));
  if (x0s) {
    std::vector<double> hx(E.N, 0.0);
    bool any = false;
    for (int k = 0; k < F.B; ++k)
      if (x0s[k] && on[k]) {
        std::memcpy(&hx[F.noff[k]], x0s[k], sizeof(double) * (F.noff[k + 1] - F.noff[k]));
        any = true;
      }
    if (any) {
      HPRQP_CUDA(cudaMemcpyAsync(E.stage, hx.data(), sizeof(double) * E.N, cudaMemcpyHostToDevice, E.st));
      HPRQP_CUDA(cudaStreamSynchronize(E.st));
      E.each(E.N, InitX<V>{E.x, E.x_bar, E.w, E.w_bar, E.last_x, E.last_w, E.stage});
    }
  }
  upload_scalars(E, sigma, lamQ, rit);
  upload_mask(E, on);
}

static void solve(Handle& H, const hprqp_params& p, const double* const* x0s, const double* sig0,
                  hprqp_result* res, double* const* xs) {
  if (p.auto_save) throw Error(HPRQP_E_UNSUPPORTED, "auto_save is not implemented");
  if (!(p.stoptol > 0) || p.check_iter <= 0 || !(p.print_frequency == -1 || p.print_frequency > 0))
    throw Error(HPRQP_E_ARG, "bad parameters");
  const Family& F = H.F;
  const int B = F.B;
  const bool fp32 = p.precision == HPRQP_PRECISION_FP32_POLISH;
  const double tc0 = now_s();
  if (!H.e64) H.e64 = std::make_unique<BEngine<double>>(F, H.st);
  if (fp32 && !H.e32)
    H.e32 = std::make_unique<BEngine<float>>(F, H.st, &H.e64->L, &H.e64->LT, &H.e64->SL, &H.e64->SLT);
  const double t_engines = now_s() - tc0;
  BEngine<double>& E64 = *H.e64;
  const double t0 = now_s();
  // lambda_max(Q_k) per instance
  std::vector<double> lamQ(B, p.lambda_max_Q_override);
  if (!(p.lambda_max_Q_override > 0)) {
    std::vector<double> l = fp32 ? power_batch(*H.e32, F, 1e-4, 5000) : power_batch(E64, F, 1e-4, 5000);
    for (int k = 0; k < B; ++k) lamQ[k] = l[k] * p.eig_factor;
  }
  const double power_time = now_s() - t0;
  // sigma: parameter rule (norm_b = 0 for LASSO, so 1 unless given), or per instance
  std::vector<double> sigma(B, p.sigma > 0 ? p.sigma : 1.0);
  if (sig0)
    for (int k = 0; k < B; ++k)
      if (sig0[k] > 0) sigma[k] = sig0[k];
  std::vector<int> rit(B, 0);
  std::vector<unsigned char> on64(B, fp32 ? 0 : 1), on32(B, fp32 ? 1 : 0);
  init_engine(E64, F, x0s, on64, sigma, lamQ, rit);
  if (fp32) init_engine(*H.e32, F, x0s, on32, sigma, lamQ, rit);
  HPRQP_CUDA(cudaStreamSynchronize(H.st));
  std::vector<RI> ri(B);
  for (int k = 0; k < B; ++k) ri[k].best_sigma = sigma[k];
  std::vector<int> status(B, -1), phase(B, fp32 ? 0 : 1);
  std::vector<int64_t> it_end(B, 0), it_fp32(B, 0), it4(B, 0), it6(B, 0);
  std::vector<double> kkt(B, std::numeric_limits<double>::infinity()), pobj(B, 0), dobj(B, 0), gap(B, 0),
      erd(B, 0), t_end(B, 0), tm4(B, 0), tm6(B, 0);
  std::vector<char> pend_cur(B, 0), pend_last(B, 0);
  std::vector<double> mn_sig_cur(B, 0), mn_sig_last(B, 0);
  const double polish_tol = p.polish_tol > 0 ? p.polish_tol : 10.0 * p.stoptol;
  std::vector<double> best32(B, std::numeric_limits<double>::infinity());
  std::vector<int> stall32(B, 0);
  const bool lasso_obj = p.problem_type == HPRQP_PROBLEM_LASSO;
  int active = B;
  int64_t launches = 0;
  auto on_print = [&](int64_t it) {
    return p.print_frequency == -1 ? std::fmod((double)it, print_step(it)) == 0.0 : it % p.print_frequency == 0;
  };
  for (int64_t iter = 0; iter <= p.max_iter && active > 0; ++iter) {
    const bool print_yes = on_print(iter) || iter == p.max_iter;
    std::vector<int> flag(B, 0);
    if (iter % p.check_iter == 0 || print_yes) {
      // residuals in each engine; a switching instance is re-evaluated in FP64
      std::vector<double> r64, r32, m64c, m64l, m32c, m32l;
      auto gather = [&](auto& E, const std::vector<unsigned char>& on, std::vector<double>& r, std::vector<double>& mc,
                        std::vector<double>& ml) {
        E.residuals(lasso_obj, E.on);
        r = read(E, E.out_res, (int64_t)B * 6);
        mc = read(E, E.out_mn_cur, (int64_t)B * 3);
        ml = read(E, E.out_mn_last, (int64_t)B * 3);
        (void)on;
      };
      gather(E64, on64, r64, m64c, m64l);
      if (fp32) gather(*H.e32, on32, r32, m32c, m32l);
      std::vector<unsigned char> sw(B, 0);
      bool any_sw = false;
      auto eval = [&](int k, const std::vector<double>& r) {
        const double* s = &r[(size_t)k * 6];
        const double xq = s[1];
        double po = (s[0] + 0.5 * xq) + F.obj_constant[k], du = (-0.5 * xq + s[2]) + F.obj_constant[k];
        if (lasso_obj) { po += s[3]; du += s[3]; }
        pobj[k] = po;
        dobj[k] = du;
        gap[k] = std::fabs(po - du) / (1.0 + std::max(std::fabs(po), std::fabs(du)));
        erd[k] = s[4] / (1.0 + std::max(F.norm_c_org[k], s[5]));
        kkt[k] = std::max(erd[k], gap[k]);
      };
      auto mnorm_val = [&](const double* s, double sg, double lq) {  // compute_M_norm!, m = 0, not diagonal
        double M1 = sg * lq * s[2];
        double M2 = (1.0 / sg) * s[0] - 2.0 * s[1] + std::max(M1, 0.0);
        return std::sqrt(std::max(M2, 0.0));
      };
      for (int k = 0; k < B; ++k) {
        if (status[k] >= 0) continue;
        const bool in64 = phase[k] == 1;
        const std::vector<double>& mc = in64 ? m64c : m32c;
        const std::vector<double>& ml = in64 ? m64l : m32l;
        if (pend_cur[k]) { ri[k].current_gap = mnorm_val(&mc[(size_t)k * 3], mn_sig_cur[k], lamQ[k]); pend_cur[k] = 0; }
        if (pend_last[k]) { ri[k].last_gap = mnorm_val(&ml[(size_t)k * 3], mn_sig_last[k], lamQ[k]); pend_last[k] = 0; }
        eval(k, in64 ? r64 : r32);
        if (!in64) {
          // hand over at polish_tol, or once the FP32 iterate stops improving
          // (no 10% gain in the best KKT over kStallChecks evaluations)
          bool go = kkt[k] < polish_tol;
          if (kkt[k] < 0.9 * best32[k]) {
            best32[k] = kkt[k];
            stall32[k] = 0;
          } else if (++stall32[k] >= kStallChecks && iter >= kStallMinIter) {
            go = true;
          }
          if (go) { sw[k] = 1; any_sw = true; }
        }
      }
      if (any_sw) {  // hand the switching instances to the FP64 engine and re-evaluate there
        BEngine<float>& E32 = *H.e32;
        unsigned char* dmask = E64.on_pw;  // scratch device mask
        HPRQP_CUDA(cudaMemcpyAsync(dmask, sw.data(), B, cudaMemcpyHostToDevice, H.st));
        const int* in = E64.inst_n;
        auto cp = [&](double* d, const float* s) { E64.each(E64.N, CopyMasked<double, float>{d, s, in, dmask}); };
        cp(E64.x, E32.x); cp(E64.x_hat, E32.x_hat); cp(E64.x_bar, E32.x_bar); cp(E64.dx, E32.dx);
        cp(E64.w, E32.w); cp(E64.w_bar, E32.w_bar); cp(E64.dw, E32.dw); cp(E64.z_bar, E32.z_bar);
        E64.each(E64.N, CopyMasked<double, double>{E64.last_x, E32.last_x, in, dmask});
        E64.each(E64.N, CopyMasked<double, double>{E64.last_w, E32.last_w, in, dmask});
        for (int k = 0; k < B; ++k)
          if (sw[k]) { phase[k] = 1; on64[k] = 1; on32[k] = 0; it_fp32[k] = iter; }
        upload_mask(E64, on64);
        upload_mask(E32, on32);
        upload_scalars(E64, sigma, lamQ, rit);
        E64.residuals(lasso_obj, dmask);
        std::vector<double> rr = read(E64, E64.out_res, (int64_t)B * 6);
        for (int k = 0; k < B; ++k)
          if (sw[k]) eval(k, rr);
      }
      for (int k = 0; k < B; ++k)
        if (status[k] < 0 && !std::isfinite(kkt[k])) status[k] = HPRQP_STATUS_NUMERICAL_ERROR;
    }
    // check_break, check_restart, per instance
    bool finished_now = false;
    for (int k = 0; k < B; ++k) {
      if (status[k] >= 0) continue;
      if (kkt[k] < p.stoptol) status[k] = HPRQP_STATUS_OPTIMAL;
      else if (iter == p.max_iter) status[k] = HPRQP_STATUS_MAX_ITER;
      else if (now_s() - t0 > p.time_limit) status[k] = HPRQP_STATUS_TIME_LIMIT;
      RI& r = ri[k];
      r.flag = 0;
      if (r.first) {
        if (iter == p.check_iter) {
          r.first = false;
          r.flag = 1;
          r.weighted = r.current_gap;
          r.best_gap = r.current_gap;
          r.best_sigma = sigma[k];
        }
      } else if (iter % p.check_iter == 0) {
        if (r.current_gap < 0) r.current_gap = 1e-6;
        if (r.current_gap <= 0.2 * r.last_gap) r.flag = 1;
        if (r.current_gap <= 0.8 * r.last_gap && r.current_gap > r.save_gap) r.flag = 2;
        const double fct = (r.current_gap / r.weighted > 1e-1) ? 0.5 : 0.2;
        if (r.inner >= fct * iter) r.flag = 3;
        if (r.best_gap > r.current_gap) { r.best_gap = r.current_gap; r.best_sigma = sigma[k]; }
        r.save_gap = r.current_gap;
      }
      if (status[k] >= 0) {
        finished_now = true;
        r.flag = 0;
        it_end[k] = iter;
        t_end[k] = now_s() - t0;
        (phase[k] == 1 ? on64 : on32)[k] = 0;
        --active;
      }
      flag[k] = r.flag;
    }
    // sigma update for restarting instances (update_sigma!, m = 0: sqrt(b/a))
    bool any_flag = false;
    for (int k = 0; k < B; ++k) any_flag |= flag[k] > 0;
    if (any_flag) {
      auto sig = [&](auto& E, int ph) {
        std::vector<unsigned char> fm(B, 0);
        bool any = false;
        for (int k = 0; k < B; ++k)
          if (flag[k] > 0 && phase[k] == ph) { fm[k] = 1; any = true; }
        if (!any) return;
        HPRQP_CUDA(cudaMemcpyAsync(E.on_pw, fm.data(), B, cudaMemcpyHostToDevice, H.st));
        if (!p.sigma_fixed) {
          E.sigma_stats(E.on_pw);
          std::vector<double> s = read(E, E.out_sig, (int64_t)B * 2);
          for (int k = 0; k < B; ++k) {
            if (!fm[k]) continue;
            double a = std::max(lamQ[k] * s[(size_t)k * 2 + 1], 1e-12), b = std::max(s[(size_t)k * 2], 1e-12);
            const double est = std::sqrt(b / a);
            const RI& r = ri[k];
            const double fct = std::exp(-0.05 * (r.current_gap / r.best_gap));
            const double erp = 0.0;  // err_Rp of an unconstrained (m = 0) instance
            const double temp1 = std::max(std::min(erd[k], erp), std::min(gap[k], r.current_gap));
            const double cand = std::exp(fct * std::log(est) + (1 - fct) * std::log(r.best_sigma));
            double kappa;
            if (temp1 > 9e-10) kappa = 1.0;
            else if (temp1 > 5e-10) kappa = std::min(std::max(std::sqrt(erd[k] / erp), 1e-2), 100.0);
            else kappa = std::min(std::max(erd[k] / erp, 1e-2), 100.0);
            sigma[k] = kappa * cand;
          }
        }
        E.restart(E.on_pw);
      };
      sig(E64, 1);
      if (fp32) sig(*H.e32, 0);
      for (int k = 0; k < B; ++k)
        if (flag[k] > 0) {
          ri[k].last_gap = ri[k].current_gap;
          ri[k].save_gap = std::numeric_limits<double>::infinity();
          ri[k].times++;
          ri[k].inner = 0;
          rit[k] = (int)iter;
        }
    }
    for (int k = 0; k < B; ++k) {
      if (status[k] >= 0) continue;
      if (kkt[k] < 1e-4 && it4[k] == 0 && tm4[k] == 0) { it4[k] = iter; tm4[k] = now_s() - t0; }
      if (kkt[k] < 1e-6 && it6[k] == 0 && tm6[k] == 0) { it6[k] = iter; tm6[k] = now_s() - t0; }
    }
    if (active == 0) break;
    if (any_flag || finished_now) {  // per-instance state changed: refresh the device copies
      upload_mask(E64, on64);
      upload_scalars(E64, sigma, lamQ, rit);
      if (fp32) {
        upload_mask(*H.e32, on32);
        upload_scalars(*H.e32, sigma, lamQ, rit);
      }
    }
    const int64_t next = iter + 1;
    const bool to_check = (next % p.check_iter == 0) || any_flag || on_print(next);
    bool any64 = false, any32 = false;
    for (int k = 0; k < B; ++k)
      if (status[k] < 0) (phase[k] == 1 ? any64 : any32) = true;
    if (any64) E64.step(to_check, (int)iter);
    if (any32) H.e32->step(to_check, (int)iter);
    if (any_flag) {
      if (any64) E64.mnorm(E64.out_mn_last);
      if (any32) H.e32->mnorm(H.e32->out_mn_last);
      for (int k = 0; k < B; ++k)
        if (flag[k] > 0) { pend_last[k] = 1; mn_sig_last[k] = sigma[k]; }
    }
    if ((iter + 1) % p.check_iter == 0) {
      if (any64) E64.mnorm(E64.out_mn_cur);
      if (any32) H.e32->mnorm(H.e32->out_mn_cur);
      for (int k = 0; k < B; ++k)
        if (status[k] < 0) { pend_cur[k] = 1; mn_sig_cur[k] = sigma[k]; }
    }
    for (int k = 0; k < B; ++k)
      if (status[k] < 0) ri[k].inner++;
  }
  HPRQP_CUDA(cudaStreamSynchronize(H.st));
  const double t_all = now_s() - t0;
  if (const char* tv = std::getenv("HPRQP_TIMING"))
    if (tv[0] == '1')
      std::fprintf(stderr, "batch solve: engines %.3f s, power %.3f s, loop %.3f s\n", t_engines, power_time,
                   t_all - power_time);
  launches = E64.launches + (H.e32 ? H.e32->launches : 0);
  // collect_results! (operator Q: x = x_bar)
  std::vector<double> x64(F.N), x32(fp32 ? F.N : 0);
  HPRQP_CUDA(cudaMemcpyAsync(x64.data(), E64.x_bar, sizeof(double) * F.N, cudaMemcpyDeviceToHost, E64.st));
  HPRQP_CUDA(cudaStreamSynchronize(E64.st));
  if (fp32) {
    std::vector<float> xf(F.N);
    HPRQP_CUDA(cudaMemcpyAsync(xf.data(), H.e32->x_bar, sizeof(float) * F.N, cudaMemcpyDeviceToHost, H.e32->st));
    HPRQP_CUDA(cudaStreamSynchronize(H.e32->st));
    for (int64_t i = 0; i < F.N; ++i) x32[i] = xf[i];
  }
  for (int k = 0; k < B; ++k) {
    hprqp_result& r = res[k];
    std::memset(&r, 0, sizeof(r));
    r.iter = it_end[k];
    r.time = t_end[k] > 0 ? t_end[k] : t_all;
    r.power_time = power_time;
    r.primal_obj = pobj[k];
    r.dual_obj = dobj[k];
    r.residuals = kkt[k];
    r.gap = gap[k];
    r.err_Rd = erd[k];
    r.status = status[k] < 0 ? HPRQP_STATUS_MAX_ITER : status[k];
    r.sigma = sigma[k];
    r.lambda_max_Q = lamQ[k];
    r.restarts = ri[k].times;
    r.iter_fp32 = it_fp32[k] ? it_fp32[k] : (fp32 ? it_end[k] : 0);
    r.iter_4 = it4[k] ? it4[k] : it_end[k];
    r.iter_6 = it6[k] ? it6[k] : it_end[k];
    r.time_4 = tm4[k] > 0 ? tm4[k] : r.time;
    r.time_6 = tm6[k] > 0 ? tm6[k] : r.time;
    r.gpu_launches = launches;
    r.device_time = t_all;
    if (xs && xs[k]) {
      const std::vector<double>& src = phase[k] == 1 ? x64 : x32;
      std::memcpy(xs[k], &src[F.noff[k]], sizeof(double) * (F.noff[k + 1] - F.noff[k]));
    }
  }
  E64.launches = 0;
  if (H.e32) H.e32->launches = 0;
}

}  // namespace batch
}  // namespace hprqp

struct hprqp_batch : hprqp::batch::Handle {};
static thread_local std::string g_batch_err;

#define BATCH_GUARD(h, ...)                      \
  try {                                          \
    if (h) cudaSetDevice(h->device);             \
    __VA_ARGS__;                                 \
    return HPRQP_OK;                             \
  } catch (const hprqp::Error& e) {              \
    (h ? h->err : g_batch_err) = e.what();       \
    return e.code;                               \
  } catch (const std::exception& e) {            \
    (h ? h->err : g_batch_err) = e.what();       \
    return HPRQP_E_CUDA;                         \
  }

extern "C" {

int hprqp_batch_create(hprqp_batch_handle* out, int32_t device) {
  hprqp_batch* h = nullptr;
  try {
    if (!out) throw hprqp::Error(HPRQP_E_ARG, "null handle pointer");
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count)
      throw hprqp::Error(HPRQP_E_CUDA, "CUDA device unavailable");
    HPRQP_CUDA(cudaSetDevice(device));
    h = new hprqp_batch();
    h->device = device;
    HPRQP_CUDA(cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking));
    *out = h;
    return HPRQP_OK;
  } catch (const hprqp::Error& e) {
    g_batch_err = e.what();
    delete h;
    return e.code;
  }
}

int hprqp_batch_load_lasso(hprqp_batch_handle h, int32_t count, const hprqp_problem* problems) {
  if (!h) return HPRQP_E_ARG;
  BATCH_GUARD(h, {
    h->e64.reset();
    h->e32.reset();
    const double t = hprqp::batch::now_s();
    h->qap = false;
    hprqp::batch::build_family(count, problems, h->F);
    if (const char* tv = std::getenv("HPRQP_TIMING"))
      if (tv[0] == '1') std::fprintf(stderr, "batch load: %.3f s\n", hprqp::batch::now_s() - t);
  })
}

int hprqp_batch_load_qap(hprqp_batch_handle h, int32_t count, const hprqp_problem* problems) {
  if (!h) return HPRQP_E_ARG;
  BATCH_GUARD(h, {
    const double t = hprqp::batch::now_s();
    h->e64.reset();
    h->e32.reset();
    h->F = hprqp::batch::Family();
    if (!h->qp) h->qp = hprqp::bqp::create(h->st);
    h->qap = false;
    hprqp::bqp::load(h->qp, count, problems);
    h->qap = true;
    if (const char* tv = std::getenv("HPRQP_TIMING"))
      if (tv[0] == '1') std::fprintf(stderr, "qp batch load: %.3f s\n", hprqp::batch::now_s() - t);
  })
}

int hprqp_batch_solve(hprqp_batch_handle h, const hprqp_params* params, const double* const* initial_x,
                      const double* sigma0, hprqp_result* results, double* const* x_out) {
  if (!h || !params || !results) return HPRQP_E_ARG;
  BATCH_GUARD(h, {
    if (h->qap) {
      if (hprqp::bqp::count(h->qp) == 0) throw hprqp::Error(HPRQP_E_STATE, "no batch loaded");
      hprqp::bqp::solve(h->qp, *params, initial_x, sigma0, results, x_out);
    } else {
      if (h->F.B == 0) throw hprqp::Error(HPRQP_E_STATE, "no batch loaded");
      hprqp::batch::solve(*h, *params, initial_x, sigma0, results, x_out);
    }
  })
}

int hprqp_batch_qap_apply(hprqp_batch_handle h, int32_t precision, const double* X, double* Y,
                          int32_t* tensor_cores) {
  if (!h || !X || !Y) return HPRQP_E_ARG;
  BATCH_GUARD(h, {
    if (!h->qap || hprqp::bqp::count(h->qp) == 0) throw hprqp::Error(HPRQP_E_STATE, "no QAP batch loaded");
    const int tc = hprqp::bqp::apply_q(h->qp, precision, X, Y);
    if (tensor_cores) *tensor_cores = tc;
  })
}

const char* hprqp_batch_last_error(hprqp_batch_handle h) { return h ? h->err.c_str() : g_batch_err.c_str(); }

int hprqp_batch_destroy(hprqp_batch_handle h) {
  if (h) {
    cudaSetDevice(h->device);
    delete h;
  }
  return HPRQP_OK;
}

}  // extern "C"
