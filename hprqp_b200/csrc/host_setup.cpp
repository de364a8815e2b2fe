// host_setup.cpp — see host_setup.h.
#include "host_setup.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>

#include <omp.h>

#include "common.cuh"

namespace hprqp {

namespace {
const double kInf = std::numeric_limits<double>::infinity();

HCsr csc_to_csr(int64_t rows, int64_t cols, const int32_t* cp, const int32_t* rv, const double* nz,
                int base, const char* what) {
  HCsr M;
  M.rows = rows;
  M.cols = cols;
  if (!cp) throw Error(HPRQP_E_ARG, std::string(what) + ": null colptr");
  if (cp[0] != base) throw Error(HPRQP_E_ARG, std::string(what) + ": colptr[0] != index_base");
  const int64_t nnz = (int64_t)cp[cols] - base;
  if (nnz < 0 || nnz > INT32_MAX) throw Error(HPRQP_E_ARG, std::string(what) + ": bad nnz");
  if (nnz > 0 && (!rv || !nz)) throw Error(HPRQP_E_ARG, std::string(what) + ": null rowval/nzval");
  for (int64_t j = 0; j < cols; ++j)
    if (cp[j + 1] < cp[j]) throw Error(HPRQP_E_ARG, std::string(what) + ": colptr not monotone");
  // A stable counting sort of the entries (column-major order) by row,
  // split among H threads by columns: thread t counts its columns' entries
  // per row in its own histogram, an exclusive sum over the threads gives
  // each thread its first slot in every row, and each thread then scatters
  // its columns in order.  Rows receive their entries in increasing column
  // order, as from a serial pass, with O(nnz / H + rows) work a thread.
  // The H x rows histograms are capped at max(8 nnz, 2^22) entries; past
  // that, the row-range scatter below runs instead.
  const int T = host_threads(nnz);
  const int64_t cap = std::max<int64_t>(8 * nnz, int64_t(1) << 22);
  const int H = rows > 0 ? (int)std::min<int64_t>(T, cap / rows) : 0;
  if (H >= 2) {
    M.ptr.resize(rows + 1);
    M.col.resize(nnz);
    M.val.resize(nnz);
    std::vector<int64_t> cb(H + 1);  // column ranges of about nnz / H entries
    cb[0] = 0;
    cb[H] = cols;
    for (int t = 1; t < H; ++t) {
      const int64_t e = nnz * t / H + base;
      cb[t] = std::max<int64_t>(cb[t - 1], std::upper_bound(cp, cp + cols + 1, (int32_t)e) - cp - 1);
    }
    hvec<int> hist;
    hist.resize((size_t)H * rows);
    bool bad_row = false, bad_val = false;
#pragma omp parallel num_threads(H) reduction(|| : bad_row, bad_val)
    {
      const int t = omp_get_thread_num();
      int* h = hist.data() + (size_t)t * rows;
      std::memset(h, 0, sizeof(int) * (size_t)rows);
      for (int64_t k = cp[cb[t]] - base; k < cp[cb[t + 1]] - base; ++k) {
        const int64_t r = (int64_t)rv[k] - base;
        if (r < 0 || r >= rows) {
          bad_row = true;
          continue;
        }
        if (!std::isfinite(nz[k])) bad_val = true;
        h[r]++;
      }
#pragma omp barrier
#pragma omp for schedule(static)
      for (int64_t r = 0; r < rows; ++r) {
        int sum = 0;
        for (int q = 0; q < H; ++q) {
          int& c = hist[(size_t)q * rows + r];
          const int v = c;
          c = sum;
          sum += v;
        }
        M.ptr[r + 1] = sum;
      }
    }
    if (bad_row) throw Error(HPRQP_E_ARG, std::string(what) + ": row index out of range");
    if (bad_val) throw Error(HPRQP_E_ARG, std::string(what) + " contains NaN or Inf values.");
    M.ptr[0] = 0;
    for (int64_t i = 0; i < rows; ++i) M.ptr[i + 1] += M.ptr[i];
#pragma omp parallel num_threads(H)
    {
      const int t = omp_get_thread_num();
      int* h = hist.data() + (size_t)t * rows;
      for (int64_t j = cb[t]; j < cb[t + 1]; ++j)
        for (int64_t k = cp[j] - base; k < cp[j + 1] - base; ++k) {
          const int64_t r = (int64_t)rv[k] - base;
          const int q = M.ptr[r] + h[r]++;
          M.col[q] = (int)j;
          M.val[q] = nz[k];
        }
    }
    return M;
  }
  M.ptr.assign(rows + 1, 0);
  M.col.resize(nnz);
  M.val.resize(nnz);
  // validation and row counts, in parallel (counts by atomic increments do
  // not depend on the order)
  int* cnt = M.ptr.data() + 1;
  bool bad_row = false, bad_val = false;
#pragma omp parallel for schedule(static) reduction(|| : bad_row, bad_val) num_threads(host_threads(nnz))
  for (int64_t k = 0; k < nnz; ++k) {
    const int64_t r = (int64_t)rv[k] - base;
    if (r < 0 || r >= rows) {
      bad_row = true;
      continue;
    }
    if (!std::isfinite(nz[k])) bad_val = true;
    __atomic_fetch_add(cnt + r, 1, __ATOMIC_RELAXED);
  }
  if (bad_row) throw Error(HPRQP_E_ARG, std::string(what) + ": row index out of range");
  if (bad_val) throw Error(HPRQP_E_ARG, std::string(what) + " contains NaN or Inf values.");
  for (int64_t i = 0; i < rows; ++i) M.ptr[i + 1] += M.ptr[i];
  // scatter: each thread owns a range of rows (balanced by entries) and
  // walks all columns in order, so every row receives its entries in
  // increasing column order, as a serial pass would
#pragma omp parallel num_threads(T)
  {
    const int t = omp_get_thread_num(), nt = omp_get_num_threads();
    const int64_t e0 = nnz * t / nt, e1 = nnz * (t + 1) / nt;
    const int64_t r0 = std::upper_bound(M.ptr.begin(), M.ptr.end(), (int)e0) - M.ptr.begin() - 1;
    const int64_t r1 = t + 1 == nt ? rows : std::upper_bound(M.ptr.begin(), M.ptr.end(), (int)e1) - M.ptr.begin() - 1;
    if (r0 < r1) {
      std::vector<int> pos(M.ptr.begin() + r0, M.ptr.begin() + r1);
      for (int64_t j = 0; j < cols; ++j)
        for (int64_t k = cp[j] - base; k < cp[j + 1] - base; ++k) {
          const int64_t r = (int64_t)rv[k] - base;
          if (r < r0 || r >= r1) continue;
          int& p = pos[r - r0];
          M.col[p] = (int)j;
          M.val[p] = nz[k];
          ++p;
        }
    }
  }
  // CSC rows sorted within each column give CSR columns sorted within rows.
  return M;
}

// The caller's CSC of M (rows x cols) read directly as the CSR of M'
// (cols x rows): the column pointers are the row pointers.  Returns false
// (and leaves T empty) when some column's row indices are not strictly
// increasing, in which case the caller transposes the CSR instead.
bool csc_as_transpose(int64_t rows, int64_t cols, const int32_t* cp, const int32_t* rv, const double* nz, int base,
                      HCsr& T) {
  const int64_t nnz = (int64_t)cp[cols] - base;
  bool sorted = true;
#pragma omp parallel for schedule(static) reduction(&& : sorted) num_threads(host_threads(cols))
  for (int64_t j = 0; j < cols; ++j)
    for (int64_t k = cp[j] - base + 1; k < cp[j + 1] - base; ++k)
      if (rv[k] <= rv[k - 1]) sorted = false;
  if (!sorted) return false;
  T.rows = cols;
  T.cols = rows;
  T.ptr.resize(cols + 1);
  T.col.resize(nnz);
  T.val.resize(nnz);
#pragma omp parallel for schedule(static) num_threads(host_threads(cols))
  for (int64_t j = 0; j <= cols; ++j) T.ptr[j] = cp[j] - base;
#pragma omp parallel for schedule(static) num_threads(host_threads(nnz))
  for (int64_t k = 0; k < nnz; ++k) {
    T.col[k] = rv[k] - base;
    T.val[k] = nz[k];
  }
  return true;
}

hvec<double> copy_vec(const double* p, int64_t len, const char* what, bool allow_inf) {
  if (len > 0 && !p) throw Error(HPRQP_E_ARG, std::string(what) + ": null pointer");
  hvec<double> v;
  par_copy(v, p, len);
  // the first offending entry decides the message, as in a serial scan
  int64_t first_nan = len, first_inf = len;
#pragma omp parallel for schedule(static) reduction(min : first_nan, first_inf) num_threads(host_threads(len))
  for (int64_t i = 0; i < len; ++i) {
    if (std::isnan(v[i])) first_nan = std::min(first_nan, i);
    if (std::isinf(v[i])) first_inf = std::min(first_inf, i);
  }
  if (allow_inf) first_inf = len;
  if (first_nan < first_inf) throw Error(HPRQP_E_ARG, std::string(what) + " contains NaN values.");
  if (first_inf < len) throw Error(HPRQP_E_ARG, std::string(what) + " contains Inf values.");
  return v;
}

double norm_b_of(const hvec<double>& AL, const hvec<double>& AU, bool inf) {
  double s = 0.0;
  for (size_t i = 0; i < AL.size(); ++i) {
    const double a = AL[i] == -kInf ? 0.0 : AL[i];
    const double b = AU[i] == kInf ? 0.0 : AU[i];
    const double t = std::max(std::fabs(a), std::fabs(b));
    s = inf ? std::max(s, t) : s + t * t;
  }
  return inf ? s : std::sqrt(s);
}
double norm2(const hvec<double>& v) {
  double s = 0.0;
  for (double x : v) s += x * x;
  return std::sqrt(s);
}
double norminf(const hvec<double>& v) {
  double s = 0.0;
  for (double x : v) s = std::max(s, std::fabs(x));
  return s;
}

// ((1/dr_i) * m_ij) * (1/dc_j): the entry order of DR * M * DC
// M <- diag(1/dr) M diag(1/dc), computed as ((1/dr_i) * v) * (1/dc_j);
// the reciprocals are formed once per call (the same values).
std::vector<double> recip(const std::vector<double>& d) {
  std::vector<double> r(d.size());
  for (size_t i = 0; i < d.size(); ++i) r[i] = 1.0 / d[i];
  return r;
}

void scale_rows_cols(HCsr& M, const std::vector<double>* dr, const std::vector<double>* dc) {
  const std::vector<double> ir = dr ? recip(*dr) : std::vector<double>(), ic = dc ? recip(*dc) : std::vector<double>();
#pragma omp parallel for schedule(static) num_threads(host_threads(M.rows))
  for (int64_t i = 0; i < M.rows; ++i)
    for (int k = M.ptr[i]; k < M.ptr[i + 1]; ++k) {
      double v = M.val[k];
      if (dr) v = ir[i] * v;
      if (dc) v = v * ic[M.col[k]];
      M.val[k] = v;
    }
}

// The same update on the transpose T = M' (entry (j, i) holds M(i, j)):
// identical arithmetic in identical order, so T stays bitwise M'.
void scale_rows_cols_T(HCsr& T, const std::vector<double>* dr, const std::vector<double>* dc) {
  const std::vector<double> ir = dr ? recip(*dr) : std::vector<double>(), ic = dc ? recip(*dc) : std::vector<double>();
#pragma omp parallel for schedule(static) num_threads(host_threads(T.rows))
  for (int64_t j = 0; j < T.rows; ++j)
    for (int k = T.ptr[j]; k < T.ptr[j + 1]; ++k) {
      double v = T.val[k];
      if (dr) v = ir[T.col[k]] * v;
      if (dc) v = v * ic[j];
      T.val[k] = v;
    }
}

// row-wise max |v| (or sum |v|) of M, in stored order
std::vector<double> row_absmax(const HCsr& M) {
  std::vector<double> r(M.rows, 0.0);
#pragma omp parallel for schedule(static) num_threads(host_threads(M.rows))
  for (int64_t i = 0; i < M.rows; ++i) {
    double x = 0.0;
    for (int k = M.ptr[i]; k < M.ptr[i + 1]; ++k) x = std::max(x, std::fabs(M.val[k]));
    r[i] = x;
  }
  return r;
}

std::vector<double> row_abssum(const HCsr& M) {
  std::vector<double> r(M.rows, 0.0);
#pragma omp parallel for schedule(static) num_threads(host_threads(M.rows))
  for (int64_t i = 0; i < M.rows; ++i) {
    double x = 0.0;
    for (int k = M.ptr[i]; k < M.ptr[i + 1]; ++k) x += std::fabs(M.val[k]);
    r[i] = x;
  }
  return r;
}
}  // namespace

int host_threads(int64_t work) {
  if (work < 65536) return 1;
  return std::max(1, std::min(16, omp_get_max_threads()));
}

template <typename T>
void par_copy(hvec<T>& dst, const T* src, int64_t len) {
  dst.resize((size_t)len);
  const int nt = host_threads(len);
#pragma omp parallel for schedule(static) num_threads(nt)
  for (int t = 0; t < nt; ++t) {
    const int64_t a = len * t / nt, b = len * (t + 1) / nt;
    if (b > a) std::memcpy(dst.data() + a, src + a, sizeof(T) * (size_t)(b - a));
  }
}
template <typename T>
void par_copy(hvec<T>& dst, const hvec<T>& src) {
  par_copy(dst, src.data(), (int64_t)src.size());
}
template void par_copy<int>(hvec<int>&, const hvec<int>&);
template void par_copy<double>(hvec<double>&, const hvec<double>&);
template void par_copy<int>(hvec<int>&, const int*, int64_t);
template void par_copy<double>(hvec<double>&, const double*, int64_t);

HCsr transpose(const HCsr& A) {
  HCsr T;
  T.rows = A.cols;
  T.cols = A.rows;
  const int64_t nnz = A.nnz();
  T.ptr.assign(T.rows + 1, 0);
  T.col.resize(nnz);
  T.val.resize(nnz);
  for (int64_t k = 0; k < nnz; ++k) T.ptr[A.col[k] + 1]++;
  for (int64_t i = 0; i < T.rows; ++i) T.ptr[i + 1] += T.ptr[i];
  std::vector<int> pos(T.ptr.begin(), T.ptr.end() - 1);
  for (int64_t i = 0; i < A.rows; ++i)
    for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k) {
      const int c = A.col[k];
      T.col[pos[c]] = (int)i;
      T.val[pos[c]] = A.val[k];
      pos[c]++;
    }
  return T;
}

bool gram_pattern(const HCsr& A, const HCsr& AT, int64_t max_work, HCsr& G) {
  G = HCsr();
  const int64_t n = AT.rows, m = A.rows;
  if (n <= 0 || m <= 0 || A.nnz() == 0) return false;
  int64_t work = 0;
  for (int64_t r = 0; r < m; ++r) {
    const int64_t len = A.ptr[r + 1] - A.ptr[r];
    work += len * len;
  }
  if (work > max_work) return false;
  bool sorted = true;
#pragma omp parallel for schedule(static) reduction(&& : sorted) num_threads(host_threads(n))
  for (int64_t p = 0; p < n; ++p)
    for (int k = AT.ptr[p] + 1; k < AT.ptr[p + 1]; ++k) sorted = sorted && AT.col[k - 1] < AT.col[k];
  if (!sorted) return false;
  // one pass: each thread lists its contiguous range of rows p into its own
  // buffer (each row sorted, a per-thread marker array dedupes), then copies
  // the buffer to its place in G.col
  const int T = host_threads(n);
  std::vector<hvec<int>> buf(T);
  hvec<int> len;
  len.resize(n);
  std::vector<int64_t> pb(T + 1, 0);
#pragma omp parallel num_threads(T)
  {
    const int t = omp_get_thread_num(), nt = omp_get_num_threads();
    const int64_t p0 = n * t / nt, p1 = n * (t + 1) / nt;
    std::vector<int> mark(n, -1);
    hvec<int>& out = buf[t];
    size_t used = 0;
    out.resize((size_t)std::max<int64_t>(1024, (p1 - p0) * 8));
    for (int64_t p = p0; p < p1; ++p) {
      const size_t start = used;
      for (int k = AT.ptr[p]; k < AT.ptr[p + 1]; ++k) {
        const int r = AT.col[k];
        for (int q = A.ptr[r]; q < A.ptr[r + 1]; ++q) {
          const int j = A.col[q];
          if (mark[j] != (int)p) {
            mark[j] = (int)p;
            if (used == out.size()) out.resize(out.size() * 2);
            out[used++] = j;
          }
        }
      }
      std::sort(out.begin() + start, out.begin() + used);
      len[p] = (int)(used - start);
    }
    pb[t + 1] = (int64_t)used;
  }
  for (int t = 0; t < T; ++t) pb[t + 1] += pb[t];
  if (pb[T] > std::numeric_limits<int>::max()) return false;  // int row pointers
  G.rows = G.cols = n;
  G.ptr.resize(n + 1);
  G.ptr[0] = 0;
  for (int64_t p = 0; p < n; ++p) G.ptr[p + 1] = G.ptr[p] + len[p];
  G.col.resize(pb[T]);
#pragma omp parallel num_threads(T)
  {
    const int t = omp_get_thread_num();
    if (pb[t + 1] > pb[t])
      std::memcpy(G.col.data() + pb[t], buf[t].data(), sizeof(int) * (size_t)(pb[t + 1] - pb[t]));
  }
  return true;
}

void StartVectorStream::fill(double* out, int64_t count) {
  auto next = [this]() {
    uint64_t v = (s += 0x9E3779B97F4A7C15ULL);
    v = (v ^ (v >> 30)) * 0xBF58476D1CE4E5B9ULL;
    v = (v ^ (v >> 27)) * 0x94D049BB133111EBULL;
    return v ^ (v >> 31);
  };
  for (int64_t i = 0; i < count; ++i) {
    const double u1 = ((next() >> 11) + 1.0) * 0x1.0p-53;
    const double u2 = (next() >> 11) * 0x1.0p-53;
    out[i] = std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2) + 1e-8;
  }
}

std::vector<double> power_start_vector(int64_t len) {
  std::vector<double> z(len);
  StartVectorStream g;
  g.fill(z.data(), len);
  return z;
}

void load_problem(const hprqp_problem* pr, HostProblem& hp) {
  if (!pr) throw Error(HPRQP_E_ARG, "null problem");
  if (pr->n <= 0 || pr->m < 0 || pr->n > INT32_MAX || pr->m > INT32_MAX)
    throw Error(HPRQP_E_ARG, "bad problem sizes (need n >= 1, m >= 0)");
  if (pr->index_base != 0 && pr->index_base != 1) throw Error(HPRQP_E_ARG, "index_base must be 0 or 1");
  HostProblem h;
  h.n = pr->n;
  h.m = pr->m;
  const int base = pr->index_base;
  h.Q_kind = pr->Q_kind;
  if (h.m > 0) {
    h.A = csc_to_csr(h.m, h.n, pr->A_colptr, pr->A_rowval, pr->A_nzval, base, "A matrix");
    if (!csc_as_transpose(h.m, h.n, pr->A_colptr, pr->A_rowval, pr->A_nzval, base, h.AT)) h.AT = transpose(h.A);
  } else {
    h.A.rows = 0;
    h.A.cols = h.n;
    h.A.ptr.assign(1, 0);
    h.AT.rows = h.n;
    h.AT.cols = 0;
    h.AT.ptr.assign(h.n + 1, 0);
  }
  h.c = copy_vec(pr->c, h.n, "c vector", false);
  h.AL = copy_vec(pr->AL, h.m, "Constraint bounds AL", true);
  h.AU = copy_vec(pr->AU, h.m, "Constraint bounds AU", true);
  h.l = copy_vec(pr->l, h.n, "Variable bounds l", true);
  h.u = copy_vec(pr->u, h.n, "Variable bounds u", true);
  // the first offending index is reported, as by a serial scan
  int64_t bad_l = h.n, bad_A = h.m;
#pragma omp parallel for schedule(static) reduction(min : bad_l) num_threads(host_threads(h.n))
  for (int64_t i = 0; i < h.n; ++i)
    if (h.l[i] > h.u[i]) bad_l = std::min(bad_l, i);
#pragma omp parallel for schedule(static) reduction(min : bad_A) num_threads(host_threads(h.m))
  for (int64_t i = 0; i < h.m; ++i)
    if (h.AL[i] > h.AU[i]) bad_A = std::min(bad_A, i);
  if (bad_l < h.n) throw Error(HPRQP_E_ARG, "Infeasible variable bounds: l > u at index " + std::to_string(bad_l));
  if (bad_A < h.m) throw Error(HPRQP_E_ARG, "Infeasible constraint bounds: AL > AU at row " + std::to_string(bad_A));
  h.obj_constant = pr->obj_constant;
  h.lambda = pr->lambda;
  if (h.Q_kind == HPRQP_Q_SPARSE) {
    if (pr->Q_colptr) {
      h.Q = csc_to_csr(h.n, h.n, pr->Q_colptr, pr->Q_rowval, pr->Q_nzval, base, "Q matrix");
      if (!csc_as_transpose(h.n, h.n, pr->Q_colptr, pr->Q_rowval, pr->Q_nzval, base, h.QT)) h.QT = transpose(h.Q);
    } else {
      h.Q.rows = h.Q.cols = h.n;
      h.Q.ptr.assign(h.n + 1, 0);
      h.QT = h.Q;
    }
  } else if (h.Q_kind == HPRQP_Q_LASSO) {
    if (pr->lasso_m <= 0 || pr->lasso_m > INT32_MAX) throw Error(HPRQP_E_ARG, "LASSO: bad lasso_m");
    h.L = csc_to_csr(pr->lasso_m, h.n, pr->L_colptr, pr->L_rowval, pr->L_nzval, base, "LASSO data matrix");
    if (!csc_as_transpose(pr->lasso_m, h.n, pr->L_colptr, pr->L_rowval, pr->L_nzval, base, h.LT)) h.LT = transpose(h.L);
  } else if (h.Q_kind == HPRQP_Q_QAP) {
    const int64_t N = pr->qap_n;
    if (N <= 0 || N * N != h.n) throw Error(HPRQP_E_ARG, "QAP: n must equal qap_n^2");
    h.qn = N;
    h.qA = copy_vec(pr->qap_A, N * N, "QAP A", false);
    h.qB = copy_vec(pr->qap_B, N * N, "QAP B", false);
    h.qS = copy_vec(pr->qap_S, N * N, "QAP S", false);
    h.qT = copy_vec(pr->qap_T, N * N, "QAP T", false);
  } else if (h.Q_kind == HPRQP_Q_CUSTOM) {
    // the operator is bound afterwards by hprqp_set_qmap
  } else {
    throw Error(HPRQP_E_ARG, "unknown Q_kind");
  }
  h.loaded = true;
  hp = std::move(h);
}

void prepare_problem(const HostProblem& hp, const hprqp_params& p, Prepared& o) {
  const int64_t n = hp.n, m = hp.m;
  o = Prepared();
  o.ruiz = p.use_Ruiz_scaling;
  o.pc = p.use_Pock_Chambolle_scaling;
  o.A = hp.A;
  o.c = hp.c;
  o.AL = hp.AL;
  o.AU = hp.AU;
  o.l = hp.l;
  o.u = hp.u;
  o.row_norm.assign(m, 1.0);
  o.col_norm.assign(n, 1.0);
  o.norm_b_org = m > 0 ? norm_b_of(o.AL, o.AU, true) : 0.0;
  o.norm_c_org = norminf(o.c);
  if (hp.Q_kind != HPRQP_Q_SPARSE) {
    // Operator Q: no scaling at all (src/utils.jl:364-406)
    o.AT = hp.AT;
    o.norm_b = m > 0 ? norm_b_of(o.AL, o.AU, false) : 0.0;
    o.norm_c = norm2(o.c);
    o.diag_Q.assign(n, 0.0);
    o.Q_is_diag = false;
  } else {
    o.Q = hp.Q;
    o.AT = hp.AT;
    HCsr& A = o.A;
    HCsr& AT = o.AT;
    HCsr& Q = o.Q;
    HCsr QT = hp.QT;
    std::vector<double> tr(m, 1.0), tc(n, 1.0);
    auto apply = [&]() {
      for (int64_t i = 0; i < m; ++i) o.row_norm[i] *= tr[i];
      for (int64_t j = 0; j < n; ++j) o.col_norm[j] *= tc[j];
      scale_rows_cols(Q, &tc, &tc);
      scale_rows_cols_T(QT, &tc, &tc);
      if (m > 0) {
        scale_rows_cols(A, &tr, &tc);
        scale_rows_cols_T(AT, &tr, &tc);
      }
      for (int64_t j = 0; j < n; ++j) o.c[j] /= tc[j];
      for (int64_t i = 0; i < m; ++i) { o.AL[i] /= tr[i]; o.AU[i] /= tr[i]; }
      for (int64_t j = 0; j < n; ++j) { o.l[j] *= tc[j]; o.u[j] *= tc[j]; }
    };
    if (p.use_Ruiz_scaling) {
      for (int pass = 0; pass < 10; ++pass) {
        // column maxima of A and Q = row maxima of A' and Q'
        const std::vector<double> ca = row_absmax(AT), cq = row_absmax(QT), ra = row_absmax(A);
        for (int64_t j = 0; j < n; ++j) {
          tc[j] = std::sqrt(std::max(ca[j], cq[j]));
          if (tc[j] == 0.0) tc[j] = 1.0;
        }
        for (int64_t i = 0; i < m; ++i) {
          tr[i] = std::sqrt(ra[i]);
          if (tr[i] == 0.0) tr[i] = 1.0;
        }
        apply();
      }
    }
    if (p.use_Pock_Chambolle_scaling) {
      // column abs-sums in increasing row order = row sums of the transposes
      const std::vector<double> ca = row_abssum(AT), cq = row_abssum(QT), ra = row_abssum(A);
      for (int64_t j = 0; j < n; ++j) {
        tc[j] = std::sqrt(ca[j] + cq[j]);
        if (tc[j] == 0.0) tc[j] = 1.0;
      }
      for (int64_t i = 0; i < m; ++i) {
        tr[i] = std::sqrt(ra[i]);
        if (tr[i] == 0.0) tr[i] = 1.0;
      }
      apply();
    }
    // Q = (Q + Q') / 2 (src/utils.jl:771-780): row-wise merge, counted first
    {
      std::vector<int> len(n, 0);
      auto merge = [&](int64_t i, int* cols, double* vals) {
        int a = Q.ptr[i], b = QT.ptr[i], cnt = 0;
        const int ae = Q.ptr[i + 1], be = QT.ptr[i + 1];
        while (a < ae || b < be) {
          const int ca = a < ae ? Q.col[a] : INT32_MAX;
          const int cb = b < be ? QT.col[b] : INT32_MAX;
          double v;
          int cc;
          if (ca == cb) { v = Q.val[a++] + QT.val[b++]; cc = ca; }
          else if (ca < cb) { v = Q.val[a++]; cc = ca; }
          else { v = QT.val[b++]; cc = cb; }
          if (cols) {
            cols[cnt] = cc;
            vals[cnt] = v / 2.0;
          }
          ++cnt;
        }
        return cnt;
      };
#pragma omp parallel for schedule(static) num_threads(host_threads(n))
      for (int64_t i = 0; i < n; ++i) len[i] = merge(i, nullptr, nullptr);
      HCsr S;
      S.rows = S.cols = n;
      S.ptr.assign(n + 1, 0);
      for (int64_t i = 0; i < n; ++i) S.ptr[i + 1] = S.ptr[i] + len[i];
      S.col.resize(S.ptr[n]);
      S.val.resize(S.ptr[n]);
#pragma omp parallel for schedule(static) num_threads(host_threads(n))
      for (int64_t i = 0; i < n; ++i) merge(i, S.col.data() + S.ptr[i], S.val.data() + S.ptr[i]);
      Q = std::move(S);
    }
    finish_sparse(o, n);
  }
  int64_t nfree = 0;
  for (int64_t i = 0; i < n; ++i) nfree += (hp.l[i] == -kInf && hp.u[i] == kInf);
  o.noC = nfree > 0.8 * n;
}

void finish_sparse(Prepared& o, int64_t n) {
  {
    const HCsr& Q = o.Q;
    o.norm_b = norm_b_of(o.AL, o.AU, false);
    o.norm_c = norm2(o.c);
    // check_Q_diagonal on the scaled Q (src/utils.jl:827-855)
    o.diag_Q.assign(n, 0.0);
    std::vector<double> colsum(n, 0.0);
    for (int64_t i = 0; i < n; ++i)
      for (int k = Q.ptr[i]; k < Q.ptr[i + 1]; ++k) {
        colsum[Q.col[k]] += std::fabs(Q.val[k]);
        if (Q.col[k] == i) o.diag_Q[i] = Q.val[k];
      }
    const double rtol = std::sqrt(std::numeric_limits<double>::epsilon());
    o.Q_is_diag = true;
    for (int64_t j = 0; j < n && o.Q_is_diag; ++j) {
      const double x = colsum[j], y = std::fabs(o.diag_Q[j]);
      const bool ok = (x == y) || (std::isfinite(x) && std::isfinite(y) &&
                                   std::fabs(x - y) <= rtol * std::max(std::fabs(x), std::fabs(y)));
      if (!ok) o.Q_is_diag = false;
    }
    o.Q_maxval = Q.nnz() ? *std::max_element(Q.val.begin(), Q.val.end()) : 0.0;
  }
}

void finish_norms(Prepared& o) {
  o.norm_b = norm_b_of(o.AL, o.AU, false);
  o.norm_c = norm2(o.c);
}

void finish_common(const HostProblem& hp, Prepared& o) {
  int64_t nfree = 0;
  for (int64_t i = 0; i < hp.n; ++i) nfree += (hp.l[i] == -kInf && hp.u[i] == kInf);
  o.noC = nfree > 0.8 * hp.n;
}

double norm_b_inf_org(const hvec<double>& AL, const hvec<double>& AU) { return norm_b_of(AL, AU, true); }
double norm_inf(const hvec<double>& v) { return norminf(v); }

}  // namespace hprqp
