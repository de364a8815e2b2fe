// scale.cu — scaling! for a sparse Q on the GPU (src/utils.jl:350-804, CPU
// branch: 10 Ruiz passes on [Q; A], one Pock-Chambolle pass, Q symmetrised
// afterwards).  The same arithmetic as the host restatement in
// host_setup.cpp, expression by expression, so the result is bitwise the
// host one: column maxima and sums are row sweeps of the transposes A' and
// Q' (kept scaled side by side with A and Q), maxima are exact in any
// order, sums run along each row in stored order, and the factors are
// sqrt / reciprocal / multiply in the host's order.  The symmetrised
// pattern and its index maps come from the host (the pattern does not
// change under scaling); the values are merged on the device.  The scaled
// vectors are copied back into the host Prepared record; the matrices'
// scaled values stay on the device, where the engines copy them from, and
// Q's diagonal check runs there too (k_qcheck).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdlib>
#include <cmath>
#include <type_traits>
#include <limits>
#include <vector>

#include "pool.h"
#include "common.cuh"
#include "host_setup.h"

namespace hprqp {
namespace {

constexpr int kT = 256;

// per-row max |v| (mode 0) or sum |v| (mode 1), in stored order
__global__ void k_row_abs(int rows, const int* __restrict__ ptr, const double* __restrict__ val, int mode,
                          double* __restrict__ out) {
  const int i = blockIdx.x * kT + threadIdx.x;
  if (i >= rows) return;
  double x = 0.0;
  for (int k = ptr[i]; k < ptr[i + 1]; ++k) x = mode == 0 ? fmax(x, fabs(val[k])) : x + fabs(val[k]);
  out[i] = x;
}

// column factors: t = sqrt(max(ca, cq)) (Ruiz) or sqrt(ca + cq) (Pock-Chambolle),
// 1 where that is 0; the running norm *= t; tinv = 1 / t
__global__ void k_col_factors(int n, const double* ca, const double* cq, int mode, double* t, double* tinv,
                              double* norm) {
  const int j = blockIdx.x * kT + threadIdx.x;
  if (j >= n) return;
  double v = mode == 0 ? sqrt(fmax(ca[j], cq[j])) : sqrt(ca[j] + cq[j]);
  if (v == 0.0) v = 1.0;
  t[j] = v;
  tinv[j] = 1.0 / v;
  norm[j] *= v;
}
__global__ void k_row_factors(int m, const double* ra, double* t, double* tinv, double* norm) {
  const int i = blockIdx.x * kT + threadIdx.x;
  if (i >= m) return;
  double v = sqrt(ra[i]);
  if (v == 0.0) v = 1.0;
  t[i] = v;
  tinv[i] = 1.0 / v;
  norm[i] *= v;
}

// M <- diag(1/dr) M diag(1/dc): v = (1/dr_i) v, then v (1/dc_j); on the
// transpose (trans = 1) row j, column i of the same entry
__global__ void k_scale(int rows, const int* __restrict__ ptr, const int* __restrict__ col, double* val,
                        const double* __restrict__ rinv, const double* __restrict__ cinv, int trans) {
  const int r = blockIdx.x * kT + threadIdx.x;
  if (r >= rows) return;
  for (int k = ptr[r]; k < ptr[r + 1]; ++k) {
    double v = val[k];
    const int c = col[k];
    if (trans) {
      v = rinv[c] * v;
      v = v * cinv[r];
    } else {
      v = rinv[r] * v;
      v = v * cinv[c];
    }
    val[k] = v;
  }
}

__global__ void k_fill(int len, double* p, double v) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < len) p[i] = v;
}

__global__ void k_scale_n(int n, const double* tc, double* c, double* l, double* u) {
  const int j = blockIdx.x * kT + threadIdx.x;
  if (j >= n) return;
  c[j] /= tc[j];
  l[j] *= tc[j];
  u[j] *= tc[j];
}
__global__ void k_scale_m(int m, const double* tr, double* AL, double* AU) {
  const int i = blockIdx.x * kT + threadIdx.x;
  if (i >= m) return;
  AL[i] /= tr[i];
  AU[i] /= tr[i];
}

// S = (Q + Q') / 2 on the merged pattern: ia / ib index Q / Q' values (-1:
// absent); both null when Q's pattern is symmetric (entry p of S is entry p
// of Q and of Q')
__global__ void k_sym(int nnz, const int* ia, const int* ib, const double* qv, const double* qtv, double* sv) {
  const int p = blockIdx.x * kT + threadIdx.x;
  if (p >= nnz) return;
  const int a = ia ? ia[p] : p, b = ib ? ib[p] : p;
  const double v = (a >= 0 && b >= 0) ? qv[a] + qtv[b] : (a >= 0 ? qv[a] : qtv[b]);
  sv[p] = v / 2.0;
}

// check_Q_diagonal on the scaled S (src/utils.jl:827-855) and its largest
// entry, on the device: row i's diagonal entry and the sum of |S_ij| in
// stored (column) order.  S is exactly symmetric (entries (i,j) and (j,i)
// are the same sum of the same two scaled values), so that row sum is
// bitwise the column sum the host restatement accumulates in row order.  A
// row fails when the sum and |diagonal| differ by more than rtol relative;
// the failures are counted, and each CTA stores the largest entry it saw.
__global__ void k_qcheck(int n, const int* __restrict__ ptr, const int* __restrict__ col,
                         const double* __restrict__ val, double rtol, double* __restrict__ diag,
                         unsigned* __restrict__ bad, double* __restrict__ bmax) {
  __shared__ double sh[kT / 32];
  const int i = blockIdx.x * kT + threadIdx.x;
  double mx = -INFINITY;
  if (i < n) {
    double d = 0.0, sum = 0.0;
    for (int k = ptr[i]; k < ptr[i + 1]; ++k) {
      const double v = val[k];
      sum += fabs(v);
      if (col[k] == i) d = v;
      mx = fmax(mx, v);
    }
    diag[i] = d;
    const double x = sum, y = fabs(d);
    const bool ok = (x == y) || (isfinite(x) && isfinite(y) && fabs(x - y) <= rtol * fmax(fabs(x), fabs(y)));
    if (!ok) atomicAdd(bad, 1u);
  }
  for (int off = 16; off > 0; off >>= 1) mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, off));
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = mx;
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = sh[0];
    for (int w = 1; w < kT / 32; ++w) m = fmax(m, sh[w]);
    bmax[blockIdx.x] = m;
  }
}

struct DevBuf : PoolBlocks {  // pool scratch freed at scope exit
  template <typename T>
  T* take(int64_t n) {
    return (T*)PoolBlocks::get(sizeof(T) * (size_t)std::max<int64_t>(n, 1));
  }
};

inline int blocks(int64_t n) { return (int)((std::max<int64_t>(n, 1) + kT - 1) / kT); }

}  // namespace

void prepare_problem_gpu(const HostProblem& hp, const hprqp_params& p, Prepared& o, cudaStream_t st,
                         int64_t* h2d, int64_t* d2h) {
  if (hp.Q_kind != HPRQP_Q_SPARSE) {
    prepare_problem(hp, p, o);
    return;
  }
  const char* tv = std::getenv("HPRQP_TIMING");
  const bool timing = tv && tv[0] == '1';
  auto wall = [] { return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count(); };
  double tm[8];
  int nt = 0;
  tm[nt++] = wall();
  const int64_t n = hp.n, m = hp.m;
  o = Prepared();
  o.ruiz = p.use_Ruiz_scaling;
  o.pc = p.use_Pock_Chambolle_scaling;
  // A and A' keep their scaled values on the device only (o.dev); their
  // patterns (from which the engines' formats and the Gram pattern are
  // built) are the loaded problem's.  The vectors are uploaded from the
  // loaded problem and their scaled values downloaded at the end.
  o.A_pat = &hp.A;
  o.AT_pat = &hp.AT;
  o.norm_b_org = m > 0 ? norm_b_inf_org(hp.AL, hp.AU) : 0.0;
  o.norm_c_org = norm_inf(hp.c);
  const HCsr &Q = hp.Q, &QT = hp.QT;
  // merged pattern of Q + Q' with index maps (the values come later); a
  // structurally symmetric Q (the common case) is its own merged pattern
  bool sym_pattern = Q.ptr.size() == QT.ptr.size() && Q.col.size() == QT.col.size();
  if (sym_pattern) {
    const int64_t np = (int64_t)Q.ptr.size(), nc = (int64_t)Q.col.size();
#pragma omp parallel for schedule(static) reduction(&& : sym_pattern) num_threads(host_threads(np + nc))
    for (int64_t k = 0; k < np + nc; ++k)
      sym_pattern = sym_pattern && (k < np ? Q.ptr[k] == QT.ptr[k] : Q.col[k - np] == QT.col[k - np]);
  }
  std::vector<int> len(sym_pattern ? 0 : n, 0);
  auto merge = [&](int64_t i, int* cols, int* ia, int* ib) {
    int a = Q.ptr[i], b = QT.ptr[i], cnt = 0;
    const int ae = Q.ptr[i + 1], be = QT.ptr[i + 1];
    while (a < ae || b < be) {
      const int ca = a < ae ? Q.col[a] : INT32_MAX;
      const int cb = b < be ? QT.col[b] : INT32_MAX;
      int xa = -1, xb = -1, cc;
      if (ca == cb) { xa = a++; xb = b++; cc = ca; }
      else if (ca < cb) { xa = a++; cc = ca; }
      else { xb = b++; cc = cb; }
      if (cols) {
        cols[cnt] = cc;
        ia[cnt] = xa;
        ib[cnt] = xb;
      }
      ++cnt;
    }
    return cnt;
  };
  HCsr& S = o.Q;
  S.rows = S.cols = n;
  std::vector<int> ia, ib;
  if (sym_pattern) {
    o.Q_pat = &hp.Q;  // S's pattern is Q's
  } else {
#pragma omp parallel for schedule(static) num_threads(host_threads(n))
    for (int64_t i = 0; i < n; ++i) len[i] = merge(i, nullptr, nullptr, nullptr);
    S.ptr.assign(n + 1, 0);
    for (int64_t i = 0; i < n; ++i) S.ptr[i + 1] = S.ptr[i] + len[i];
    S.col.resize(S.ptr[n]);
    ia.resize(S.ptr[n]);
    ib.resize(S.ptr[n]);
#pragma omp parallel for schedule(static) num_threads(host_threads(n))
    for (int64_t i = 0; i < n; ++i) merge(i, S.col.data() + S.ptr[i], ia.data() + S.ptr[i], ib.data() + S.ptr[i]);
  }
  const int64_t nnzS = sym_pattern ? Q.nnz() : S.ptr[n];
  // (S's values stay on the device: the engines copy them from there)

  tm[nt++] = wall();  // merged pattern
  // device copies: what the engines copy from afterwards lives in ds->mem,
  // the scaling's scratch in d
  auto ds = std::make_shared<DevScaled>();
  DevBuf d;
  auto up = [&](auto* dst, const auto& v) {
    if (!v.empty()) {
      h2d_staged(dst, v.data(), sizeof(v[0]) * v.size(), st);
      *h2d += (int64_t)(sizeof(v[0]) * v.size());
    }
  };
  struct DM {
    int rows = 0;
    int* ptr = nullptr;
    int* col = nullptr;
    double* val = nullptr;
  };
  auto keep = [&](auto* type_tag, int64_t len) {  // an array the engines copy from
    using T = std::remove_pointer_t<decltype(type_tag)>;
    return (T*)ds->mem.get(sizeof(T) * (size_t)std::max<int64_t>(len, 1));
  };
  auto dev_csr = [&](const HCsr& h, bool kept) {
    DM x;
    x.rows = (int)h.rows;
    x.ptr = kept ? keep((int*)nullptr, h.rows + 1) : d.take<int>(h.rows + 1);
    x.col = kept ? keep((int*)nullptr, h.nnz()) : d.take<int>(h.nnz());
    x.val = kept ? keep((double*)nullptr, h.nnz()) : d.take<double>(h.nnz());
    up(x.ptr, h.ptr);
    up(x.col, h.col);
    up(x.val, h.val);
    return x;
  };
  // Q's pattern is kept when it is also S's (the symmetric case)
  const DM dA = dev_csr(hp.A, true), dAT = dev_csr(hp.AT, true), dQ = dev_csr(Q, sym_pattern),
           dQT = dev_csr(QT, false);
  double *c = keep((double*)nullptr, n), *l = keep((double*)nullptr, n), *u = keep((double*)nullptr, n);
  double* cn = keep((double*)nullptr, n);
  double *AL = keep((double*)nullptr, m), *AU = keep((double*)nullptr, m), *rn = keep((double*)nullptr, m);
  double *ca = d.take<double>(n), *cq = d.take<double>(n), *tc = d.take<double>(n), *tci = d.take<double>(n);
  double *ra = d.take<double>(m), *tr = d.take<double>(m), *tri = d.take<double>(m);
  up(c, hp.c);
  up(l, hp.l);
  up(u, hp.u);
  up(AL, hp.AL);
  up(AU, hp.AU);
  k_fill<<<blocks(n), kT, 0, st>>>((int)n, cn, 1.0);  // the norms' products start at 1
  if (m > 0) k_fill<<<blocks(m), kT, 0, st>>>((int)m, rn, 1.0);
  HPRQP_LAUNCH_CHECK();
  HPRQP_CUDA(cudaStreamSynchronize(st));
  tm[nt++] = wall();  // uploads
  auto pass = [&](int mode) {  // one Ruiz (0) or Pock-Chambolle (1) pass
    k_row_abs<<<blocks(n), kT, 0, st>>>((int)n, dAT.ptr, dAT.val, mode, ca);
    k_row_abs<<<blocks(n), kT, 0, st>>>((int)n, dQT.ptr, dQT.val, mode, cq);
    k_col_factors<<<blocks(n), kT, 0, st>>>((int)n, ca, cq, mode, tc, tci, cn);
    if (m > 0) {
      k_row_abs<<<blocks(m), kT, 0, st>>>((int)m, dA.ptr, dA.val, mode, ra);
      k_row_factors<<<blocks(m), kT, 0, st>>>((int)m, ra, tr, tri, rn);
    }
    k_scale<<<blocks(n), kT, 0, st>>>((int)n, dQ.ptr, dQ.col, dQ.val, tci, tci, 0);
    k_scale<<<blocks(n), kT, 0, st>>>((int)n, dQT.ptr, dQT.col, dQT.val, tci, tci, 1);
    if (m > 0) {
      k_scale<<<blocks(m), kT, 0, st>>>((int)m, dA.ptr, dA.col, dA.val, tri, tci, 0);
      k_scale<<<blocks(n), kT, 0, st>>>((int)n, dAT.ptr, dAT.col, dAT.val, tri, tci, 1);
      k_scale_m<<<blocks(m), kT, 0, st>>>((int)m, tr, AL, AU);
    }
    k_scale_n<<<blocks(n), kT, 0, st>>>((int)n, tc, c, l, u);
    HPRQP_LAUNCH_CHECK();
  };
  if (p.use_Ruiz_scaling)
    for (int k = 0; k < 10; ++k) pass(0);
  if (p.use_Pock_Chambolle_scaling) pass(1);
  int* dia = sym_pattern ? nullptr : d.take<int>(nnzS);
  int* dib = sym_pattern ? nullptr : d.take<int>(nnzS);
  double* sv = keep((double*)nullptr, nnzS);
  if (!sym_pattern) {
    up(dia, ia);
    up(dib, ib);
  }
  k_sym<<<blocks(nnzS), kT, 0, st>>>((int)nnzS, dia, dib, dQ.val, dQT.val, sv);
  HPRQP_LAUNCH_CHECK();
  // S's pattern on the device (Q's when that is symmetric)
  const int *sptr = dQ.ptr, *scol = dQ.col;
  if (!sym_pattern) {
    int* p2 = keep((int*)nullptr, n + 1);
    int* c2 = keep((int*)nullptr, nnzS);
    up(p2, S.ptr);
    up(c2, S.col);
    sptr = p2;
    scol = c2;
  }
  double* dg = d.take<double>(n);
  unsigned* bad = d.take<unsigned>(1);
  const int nb = blocks(n);
  double* bmax = d.take<double>(nb);
  HPRQP_CUDA(cudaMemsetAsync(bad, 0, sizeof(unsigned), st));
  k_qcheck<<<nb, kT, 0, st>>>((int)n, sptr, scol, sv, std::sqrt(std::numeric_limits<double>::epsilon()), dg, bad,
                              bmax);
  HPRQP_LAUNCH_CHECK();
  HPRQP_CUDA(cudaStreamSynchronize(st));
  tm[nt++] = wall();  // scaling kernels
  auto down = [&](auto& dst, const double* src) {  // (synchronous: pinned chunks, copied out in parallel)
    if (!dst.empty()) {
      d2h_staged(dst.data(), src, sizeof(double) * dst.size(), st);
      *d2h += (int64_t)(sizeof(double) * dst.size());
    }
  };
  // (filled by the downloads)
  o.diag_Q.resize(n);
  o.c.resize(n);
  o.l.resize(n);
  o.u.resize(n);
  o.col_norm.resize(n);
  o.AL.resize(m);
  o.AU.resize(m);
  o.row_norm.resize(m);
  down(o.diag_Q, dg);
  std::vector<double> hmax(nb);
  down(hmax, bmax);
  unsigned nbad = 0;
  HPRQP_CUDA(cudaMemcpyAsync(&nbad, bad, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
  *d2h += (int64_t)sizeof(unsigned);
  down(o.c, c);
  down(o.l, l);
  down(o.u, u);
  down(o.col_norm, cn);
  down(o.AL, AL);
  down(o.AU, AU);
  down(o.row_norm, rn);
  HPRQP_CUDA(cudaStreamSynchronize(st));
  o.Q_is_diag = nbad == 0;
  o.Q_maxval = nnzS > 0 ? *std::max_element(hmax.begin(), hmax.end()) : 0.0;
  ds->A = DevCsrView{dA.ptr, dA.col, dA.val};
  ds->AT = DevCsrView{dAT.ptr, dAT.col, dAT.val};
  ds->Q = DevCsrView{sptr, scol, sv};
  ds->c = c;
  ds->l = l;
  ds->u = u;
  ds->AL = AL;
  ds->AU = AU;
  ds->row_norm = rn;
  ds->col_norm = cn;
  o.dev = ds;
  tm[nt++] = wall();  // downloads
  finish_norms(o);
  finish_common(hp, o);
  tm[nt++] = wall();
  if (timing)
    std::fprintf(stderr, "[hprqp] scaling: pattern %.3f, uploads %.3f, kernels %.3f, downloads %.3f, finish %.3f s\n",
                 tm[1] - tm[0], tm[2] - tm[1], tm[3] - tm[2], tm[4] - tm[3], tm[5] - tm[4]);
}

}  // namespace hprqp
