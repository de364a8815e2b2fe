// hprqp_oracle.cpp — TEST INFRASTRUCTURE, NOT PRODUCT CODE.
//
// A plain C++ FP64 restatement of the HPR-QP reference CPU path
// (`params.use_gpu = false`), used only as the checker of the CUDA engine
// (tests/, __graft_entry__.smoke()) and as the timed CPU baseline of
// bench.py.  Nothing in hprqp_b200/ links, loads or calls it.
//
// The reference is Julia (PolyU-IOR/HPR-QP); Julia is not available here, so
// this file restates its CPU arithmetic function by function.  Each function
// cites the Julia source it follows.  Summation orders of the sparse
// products follow Julia's SparseArrays `mul!` (CSC scatter for A*x, per-column
// dot for A'*y), both of which equal a CSR row dot in increasing column order,
// so the CSR loops below reproduce them exactly.  Dense dot/norm calls in the
// reference go to BLAS; here they are sequential sums (differences ~1e-16).
//
// Parity pinning: the reference's tests carry no golden vectors (they assert
// status == "OPTIMAL" and residual < tol only, test/runtests.jl:149-152), and
// the reference cannot run in this container, so iterate-level parity with
// the reference itself is unpinned.  The oracle is pinned against the
// analytic optimum of the reference's model.mps / demo_QAbc.jl example and
// against the reference tests' own status/tolerance thresholds, and checked
// against scipy's HiGHS LP solver on LP instances (tests/test_oracle.py).
//
// One documented deviation: the power iteration's start vector.  The
// reference draws randn(MersenneTwister(1), m) .+ 1e-8 (src/utils.jl:1339);
// Julia's dSFMT/ziggurat stream cannot be reproduced here, so the oracle and
// the CUDA engine both use the splitmix64 + Box-Muller stream of
// power_start_vector() below.  Tests inject lambda_max_A/Q for iterate parity.

#include "../include/hprqp.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <limits>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

using Vec = std::vector<double>;
const double INF = std::numeric_limits<double>::infinity();
thread_local std::string g_err;

struct Csr {  // row-major sparse matrix, 0-based
  int64_t rows = 0, cols = 0;
  std::vector<int64_t> ptr;
  std::vector<int32_t> col;
  Vec val;
};

int g_threads = 1;

// y = M*x  (Julia mul! on CSC == CSR row dot, increasing column order)
void spmv(const Csr& M, const double* x, double* y) {
#pragma omp parallel for schedule(static) if (g_threads > 1) num_threads(g_threads)
  for (int64_t i = 0; i < M.rows; ++i) {
    double s = 0.0;
    for (int64_t k = M.ptr[i]; k < M.ptr[i + 1]; ++k) s += M.val[k] * x[M.col[k]];
    y[i] = s;
  }
}

double dot(const Vec& a, const Vec& b) {
  double s = 0.0;
  const int64_t n = (int64_t)a.size();
#pragma omp parallel for reduction(+ : s) schedule(static) if (g_threads > 1) num_threads(g_threads)
  for (int64_t i = 0; i < n; ++i) s += a[i] * b[i];
  return s;
}
double norm2(const Vec& a) { return std::sqrt(dot(a, a)); }
double norminf(const Vec& a) {
  double s = 0.0;
  for (double v : a) s = std::max(s, std::fabs(v));
  return s;
}
double norm1(const Vec& a) {
  double s = 0.0;
  for (double v : a) s += std::fabs(v);
  return s;
}
inline double clamp_(double v, double lo, double hi) { return std::min(std::max(v, lo), hi); }
inline double muladd(double a, double b, double c) { return std::fma(a, b, c); }

// Transpose a CSC (colptr/rowval/nzval, base b) of size rows x cols into CSR.
Csr csc_to_csr(int64_t rows, int64_t cols, const int32_t* cp, const int32_t* rv, const double* nz,
               int base) {
  Csr M;
  M.rows = rows;
  M.cols = cols;
  const int64_t nnz = cols > 0 ? (int64_t)cp[cols] - base : 0;
  M.ptr.assign(rows + 1, 0);
  M.col.resize(nnz);
  M.val.resize(nnz);
  for (int64_t k = 0; k < nnz; ++k) M.ptr[rv[k] - base + 1]++;
  for (int64_t i = 0; i < rows; ++i) M.ptr[i + 1] += M.ptr[i];
  std::vector<int64_t> pos(M.ptr.begin(), M.ptr.end() - 1);
  for (int64_t j = 0; j < cols; ++j)
    for (int64_t k = cp[j] - base; k < cp[j + 1] - base; ++k) {
      const int64_t r = rv[k] - base;
      M.col[pos[r]] = (int32_t)j;
      M.val[pos[r]] = nz[k];
      pos[r]++;
    }
  return M;
}

Csr transpose(const Csr& A) {
  Csr T;
  T.rows = A.cols;
  T.cols = A.rows;
  const int64_t nnz = (int64_t)A.val.size();
  T.ptr.assign(T.rows + 1, 0);
  T.col.resize(nnz);
  T.val.resize(nnz);
  for (int64_t k = 0; k < nnz; ++k) T.ptr[A.col[k] + 1]++;
  for (int64_t i = 0; i < T.rows; ++i) T.ptr[i + 1] += T.ptr[i];
  std::vector<int64_t> pos(T.ptr.begin(), T.ptr.end() - 1);
  for (int64_t i = 0; i < A.rows; ++i)
    for (int64_t k = A.ptr[i]; k < A.ptr[i + 1]; ++k) {
      const int64_t c = A.col[k];
      T.col[pos[c]] = (int32_t)i;
      T.val[pos[c]] = A.val[k];
      pos[c]++;
    }
  return T;
}

// Start vector of the power method: z_i ~ N(0,1) from splitmix64(seed 1) and
// Box-Muller, plus 1e-8 (src/utils.jl:1339,1422).  The CUDA engine generates
// the identical stream on the host.
uint64_t splitmix64(uint64_t& s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ULL);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}
Vec power_start_vector(int64_t len) {
  Vec z(len);
  uint64_t s = 1;
  for (int64_t i = 0; i < len; ++i) {
    const double u1 = ((splitmix64(s) >> 11) + 1.0) * 0x1.0p-53;  // (0,1]
    const double u2 = (splitmix64(s) >> 11) * 0x1.0p-53;          // [0,1)
    z[i] = std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2) + 1e-8;
  }
  return z;
}

// ---------------------------------------------------------------------------
// Q operators (src/Q_operators/*.jl, CPU Qmap!)
// ---------------------------------------------------------------------------
struct QOp {
  int kind = HPRQP_Q_SPARSE;
  int64_t n = 0;
  Csr Q;            // sparse: scaled + symmetrised Q (sparse_matrix_operator.jl:45-51)
  Csr L, LT;        // LASSO: A_d and A_d' (LASSO_operator.jl:112-117)
  mutable Vec temp; // LASSO: A_d*x
  int64_t qn = 0;   // QAP
  Vec qA, qB, qS, qT;
  mutable Vec tmp;

  bool is_operator() const { return kind != HPRQP_Q_SPARSE; }
  int64_t nnz() const { return (int64_t)Q.val.size(); }

  void apply(const Vec& x, Vec& Qx) const {
    if (kind == HPRQP_Q_SPARSE) {
      spmv(Q, x.data(), Qx.data());
    } else if (kind == HPRQP_Q_LASSO) {
      spmv(L, x.data(), temp.data());   // temp = A*x
      spmv(LT, temp.data(), Qx.data()); // Qx = A'*temp
    } else {
      // QAP_operator.jl:65-75: X = reshape(x,n,n); TMP = A*X;
      // QX = 2*TMP*B; QX -= 2*S*X; QX -= 2*X*T   (column-major)
      const int64_t N = qn;
      const double* X = x.data();
      double* QX = Qx.data();
      double* T = tmp.data();
#pragma omp parallel for schedule(static) if (g_threads > 1) num_threads(g_threads)
      for (int64_t j = 0; j < N; ++j)
        for (int64_t i = 0; i < N; ++i) {
          double s = 0.0;
          for (int64_t k = 0; k < N; ++k) s += qA[i + k * N] * X[k + j * N];
          T[i + j * N] = s;
        }
#pragma omp parallel for schedule(static) if (g_threads > 1) num_threads(g_threads)
      for (int64_t j = 0; j < N; ++j)
        for (int64_t i = 0; i < N; ++i) {
          double s1 = 0.0, s2 = 0.0, s3 = 0.0;
          for (int64_t k = 0; k < N; ++k) {
            s1 += T[i + k * N] * qB[k + j * N];
            s2 += qS[i + k * N] * X[k + j * N];
            s3 += X[i + k * N] * qT[k + j * N];
          }
          double v = 2.0 * s1;
          v = -2.0 * s2 + v;
          v = -2.0 * s3 + v;
          QX[i + j * N] = v;
        }
    }
  }
};

// ---------------------------------------------------------------------------
// Problem / scaling / workspace (src/structs.jl, src/utils.jl, algorithm.jl)
// ---------------------------------------------------------------------------
struct Prob {
  int64_t n = 0, m = 0;
  QOp Q;
  Csr A, AT;  // A (m x n) and A' (n x m), CSR
  Vec c, AL, AU, l, u;
  double obj_constant = 0.0, lambda = 0.0;
};

struct Scaling {  // Scaling_info_cpu (src/structs.jl:167-192)
  Vec row_norm, col_norm;
  double b_scale = 1.0, c_scale = 1.0;
  double norm_b = 0, norm_c = 0, norm_b_org = 0, norm_c_org = 0;
};

double norm_b_of(const Vec& AL, const Vec& AU, bool inf_norm) {
  // max.(abs.(AL_nInf), abs.(AU_nInf)) with infinite bounds replaced by 0
  Vec t(AL.size());
  for (size_t i = 0; i < AL.size(); ++i) {
    const double a = AL[i] == -INF ? 0.0 : AL[i];
    const double b = AU[i] == INF ? 0.0 : AU[i];
    t[i] = std::max(std::fabs(a), std::fabs(b));
  }
  return inf_norm ? norminf(t) : norm2(t);
}

// Scale the rows of CSR M by 1/dr and its columns by 1/dc, in the order
// ((1/dr_i) * m_ij) * (1/dc_j) of `DR * M * DC` (src/utils.jl:501-535).
void scale_csr(Csr& M, const Vec* dr, const Vec* dc) {
  for (int64_t i = 0; i < M.rows; ++i)
    for (int64_t k = M.ptr[i]; k < M.ptr[i + 1]; ++k) {
      double v = M.val[k];
      if (dr) v = (1.0 / (*dr)[i]) * v;
      if (dc) v = v * (1.0 / (*dc)[M.col[k]]);
      M.val[k] = v;
    }
}

// scaling! (src/utils.jl:350-804), CPU branch.
Scaling scaling(Prob& qp, const hprqp_params& p) {
  Scaling sc;
  const int64_t m = qp.m, n = qp.n;
  if (qp.Q.is_operator()) {  // src/utils.jl:364-406: no scaling at all
    sc.row_norm.assign(m, 1.0);
    sc.col_norm.assign(n, 1.0);
    sc.norm_b_org = m > 0 ? norm_b_of(qp.AL, qp.AU, true) : 0.0;
    sc.norm_c_org = norminf(qp.c);
    sc.norm_b = m > 0 ? norm_b_of(qp.AL, qp.AU, false) : 0.0;
    sc.norm_c = norm2(qp.c);
    return sc;
  }
  sc.row_norm.assign(m, 1.0);
  sc.col_norm.assign(n, 1.0);
  sc.norm_b_org = norm_b_of(qp.AL, qp.AU, true);
  sc.norm_c_org = norminf(qp.c);
  Vec tr(m, 1.0), tc(n, 1.0);
  Csr& Q = qp.Q.Q;
  Csr& A = qp.A;
  auto apply = [&]() {
    for (int64_t i = 0; i < m; ++i) sc.row_norm[i] *= tr[i];
    for (int64_t j = 0; j < n; ++j) sc.col_norm[j] *= tc[j];
    scale_csr(Q, &tc, &tc);                 // Q = DC*Q*DC
    if (m > 0) scale_csr(A, &tr, &tc);      // A = DR*A*DC
    for (int64_t j = 0; j < n; ++j) qp.c[j] /= tc[j];
    if (m > 0)
      for (int64_t i = 0; i < m; ++i) {
        qp.AL[i] /= tr[i];
        qp.AU[i] /= tr[i];
      }
    for (int64_t j = 0; j < n; ++j) {
      qp.l[j] *= tc[j];
      qp.u[j] *= tc[j];
    }
  };
  if (p.use_Ruiz_scaling) {  // src/utils.jl:453-578, 10 passes
    for (int pass = 0; pass < 10; ++pass) {
      Vec ca(n, 0.0), cq(n, 0.0);
      for (int64_t i = 0; i < A.rows; ++i)
        for (int64_t k = A.ptr[i]; k < A.ptr[i + 1]; ++k)
          ca[A.col[k]] = std::max(ca[A.col[k]], std::fabs(A.val[k]));
      for (int64_t i = 0; i < Q.rows; ++i)
        for (int64_t k = Q.ptr[i]; k < Q.ptr[i + 1]; ++k)
          cq[Q.col[k]] = std::max(cq[Q.col[k]], std::fabs(Q.val[k]));
      for (int64_t j = 0; j < n; ++j) {
        tc[j] = std::sqrt(std::max(ca[j], cq[j]));
        if (tc[j] == 0.0) tc[j] = 1.0;
      }
      if (m > 0)
        for (int64_t i = 0; i < m; ++i) {
          double r = 0.0;
          for (int64_t k = A.ptr[i]; k < A.ptr[i + 1]; ++k) r = std::max(r, std::fabs(A.val[k]));
          tr[i] = std::sqrt(r);
          if (tr[i] == 0.0) tr[i] = 1.0;
        }
      apply();
    }
  }
  if (p.use_Pock_Chambolle_scaling) {  // src/utils.jl:580-698
    Vec ca(n, 0.0), cq(n, 0.0);
    // sum(abs, A, dims=1): CSC column sums in increasing row order
    Csr AT = transpose(A), QT = transpose(Q);
    for (int64_t j = 0; j < n; ++j) {
      double s = 0.0;
      for (int64_t k = AT.ptr[j]; k < AT.ptr[j + 1]; ++k) s += std::fabs(AT.val[k]);
      ca[j] = s;
      s = 0.0;
      for (int64_t k = QT.ptr[j]; k < QT.ptr[j + 1]; ++k) s += std::fabs(QT.val[k]);
      cq[j] = s;
    }
    for (int64_t j = 0; j < n; ++j) {
      tc[j] = std::sqrt(ca[j] + cq[j]);
      if (tc[j] == 0.0) tc[j] = 1.0;
    }
    if (m > 0)
      for (int64_t i = 0; i < m; ++i) {
        double r = 0.0;
        for (int64_t k = A.ptr[i]; k < A.ptr[i + 1]; ++k) r += std::fabs(A.val[k]);
        tr[i] = std::sqrt(r);
        if (tr[i] == 0.0) tr[i] = 1.0;
      }
    apply();
  }
  // b/c scaling is disabled (`use_bc_scaling && false`, src/utils.jl:703)
  sc.b_scale = 1.0;
  sc.c_scale = 1.0;
  qp.AT = transpose(A);  // qp.AT = qp.A' (src/utils.jl:767-769)
  // Q = (Q + transpose(Q)) / 2 (src/utils.jl:771-780)
  {
    Csr QT = transpose(Q);
    Csr S;
    S.rows = S.cols = n;
    S.ptr.assign(n + 1, 0);
    for (int64_t i = 0; i < n; ++i) {
      int64_t a = Q.ptr[i], b = QT.ptr[i];
      const int64_t ae = Q.ptr[i + 1], be = QT.ptr[i + 1];
      while (a < ae || b < be) {
        int32_t ca = a < ae ? Q.col[a] : INT32_MAX;
        int32_t cb = b < be ? QT.col[b] : INT32_MAX;
        double v;
        int32_t cc;
        if (ca == cb) { v = Q.val[a++] + QT.val[b++]; cc = ca; }
        else if (ca < cb) { v = Q.val[a++]; cc = ca; }
        else { v = QT.val[b++]; cc = cb; }
        S.col.push_back(cc);
        S.val.push_back(v / 2.0);
      }
      S.ptr[i + 1] = (int64_t)S.col.size();
    }
    Q = std::move(S);
  }
  sc.norm_b = norm_b_of(qp.AL, qp.AU, false);
  sc.norm_c = norm2(qp.c);
  return sc;
}

// check_Q_diagonal (src/utils.jl:827-855): Q is diagonal iff every column
// abs-sum ≈ |Q_jj| (isapprox with rtol = sqrt(eps)).
void check_Q_diagonal(const Prob& qp, Vec& diag_Q, bool& is_diag) {
  const int64_t n = qp.n;
  diag_Q.assign(n, 0.0);
  if (qp.Q.is_operator()) { is_diag = false; return; }
  const Csr& Q = qp.Q.Q;
  Vec colsum(n, 0.0);
  Csr QT = transpose(Q);
  for (int64_t j = 0; j < n; ++j) {
    double s = 0.0;
    for (int64_t k = QT.ptr[j]; k < QT.ptr[j + 1]; ++k) {
      s += std::fabs(QT.val[k]);
      if (QT.col[k] == j) diag_Q[j] = QT.val[k];
    }
    colsum[j] = s;
  }
  const double rtol = std::sqrt(std::numeric_limits<double>::epsilon());
  is_diag = true;
  for (int64_t j = 0; j < n; ++j) {
    const double x = colsum[j], y = std::fabs(diag_Q[j]);
    const bool ok = (x == y) || (std::isfinite(x) && std::isfinite(y) &&
                                 std::fabs(x - y) <= rtol * std::max(std::fabs(x), std::fabs(y)));
    if (!ok) { is_diag = false; break; }
  }
}

struct WS {  // HPRQP_workspace_cpu (src/structs.jl:462-523)
  int64_t n = 0, m = 0;
  Vec w, w_hat, w_bar, dw, x, x_hat, x_bar, dx, y, y_hat, y_bar, dy, z_bar;
  Vec Rp, Rd, Ax, ATy, ATy_bar, ATdy, QATdy, s, Qw, Qw_hat, Qw_bar, Qx, dQw;
  Vec last_x, last_y, last_Qw, last_w, last_ATy, tempv;
  Vec diag_Q, fact1, fact2, fact, fact_M, lambda;
  Vec c, AL, AU, l, u;  // ws.c = qp.c etc. (scaled problem data)
  bool Q_is_diag = false, noC = false, to_check = true;
  double sigma = 1.0, lambda_max_A = 0.0, lambda_max_Q = 0.0;
};

struct Res {  // HPRQP_residuals (src/structs.jl:278-289)
  double err_Rp = 0, err_Rd = 0, KKT = 0, pobj = 0, gap = 0, dobj = 0;
};

struct Restart {  // HPRQP_restart + initialize_restart (algorithm.jl:1154-1171)
  bool first_restart = true;
  double save_gap = INF, current_gap = INF, last_gap = INF, best_gap = INF;
  double best_sigma = 1.0, weighted_norm = INF;
  int64_t inner = 0, times = 0, sufficient = 0, necessary = 0, long_ = 0;
  int restart_flag = 0;
};

// power_iteration_A (src/utils.jl:1335-1385)
double power_iteration_A(const Prob& qp, int max_it = 5000, double tol = 1e-4) {
  const int64_t m = qp.m, n = qp.n;
  Vec z = power_start_vector(m), q(m), ATq(n);
  double lam = 1.0;
  for (int it = 0; it < max_it; ++it) {
    q = z;
    const double nq = norm2(q);
    for (auto& v : q) v /= nq;
    spmv(qp.AT, q.data(), ATq.data());
    spmv(qp.A, ATq.data(), z.data());
    lam = dot(q, z);
    for (int64_t i = 0; i < m; ++i) q[i] = z[i] - lam * q[i];
    const double err = norm2(q) / (norm2(z) + lam);
    if (err < tol) return lam;
  }
  std::fprintf(stderr, "Power iteration (A) did not converge within the specified tolerance.\n");
  return lam;
}

// power_iteration_Q (src/utils.jl:1419-1461)
double power_iteration_Q(const Prob& qp, int max_it = 5000, double tol = 1e-4) {
  const int64_t n = qp.n;
  Vec z = power_start_vector(n), q(n);
  double lam = 1.0;
  for (int it = 0; it < max_it; ++it) {
    q = z;
    const double nq = norm2(q);
    for (auto& v : q) v /= nq;
    qp.Q.apply(q, z);
    lam = dot(q, z);
    for (int64_t i = 0; i < n; ++i) q[i] = z[i] - lam * q[i];
    const double err = norm2(q) / (norm2(z) + lam);
    if (err < tol) return lam;
  }
  std::fprintf(stderr, "Power iteration (Q) did not converge within the specified tolerance.\n");
  return lam;
}

// unified_update_Q_factors! (src/unified_operations.jl:445-459)
void update_Q_factors(WS& ws) {
  const double s = ws.sigma, s2 = s * s;
  for (int64_t i = 0; i < ws.n; ++i) {
    ws.fact2[i] = 1.0 / (1.0 + s * ws.diag_Q[i]);
    ws.fact[i] = s * ws.fact2[i];
    ws.fact1[i] = s * ws.diag_Q[i] * ws.fact2[i];
    ws.fact_M[i] = s2 * ws.fact2[i];
  }
}

// compute_residuals! (src/algorithm.jl:37-115) + compute_Rd!/compute_Rp!
// (src/kernels.jl:114-194) + compute_bounds_violation! (algorithm.jl:127-133)
void compute_residuals(WS& ws, const Prob& qp, const Scaling& sc, Res& r, const hprqp_params& p,
                       int64_t iter) {
  const int64_t n = ws.n, m = ws.m;
  qp.Q.apply(ws.x_bar, ws.Qx);
  const double bc = sc.b_scale * sc.c_scale;
  const double xQx = dot(ws.x_bar, ws.Qx);
  r.pobj = bc * (dot(ws.c, ws.x_bar) + 0.5 * xQx) + qp.obj_constant;
  r.dobj = bc * (-0.5 * xQx + dot(ws.z_bar, ws.x_bar)) + qp.obj_constant;
  if (m > 0) r.dobj += bc * dot(ws.y_bar, ws.s);
  if (p.problem_type == HPRQP_PROBLEM_LASSO && n > 0) {
    for (int64_t i = 0; i < n; ++i) ws.tempv[i] = ws.lambda[i] * ws.x_bar[i];
    const double l1 = norm1(ws.tempv);
    r.pobj += bc * l1;
    r.dobj += bc * l1;
  }
  r.gap = std::fabs(r.pobj - r.dobj) / (1.0 + std::max(std::fabs(r.pobj), std::fabs(r.dobj)));
  // compute_Rd!
  if (m > 0) spmv(qp.AT, ws.y_bar.data(), ws.ATdy.data());
  for (int64_t i = 0; i < n; ++i) {
    const double f = sc.col_norm[i] * sc.c_scale;
    ws.Rd[i] = (ws.Qx[i] + ws.c[i] - ws.ATdy[i] - ws.z_bar[i]) * f;
    ws.Qx[i] *= f;
    ws.ATdy[i] *= f;
  }
  r.err_Rd = norminf(ws.Rd) /
             (1.0 + std::max(std::max(sc.norm_c_org, norminf(ws.ATdy)), norminf(ws.Qx)));
  if (m > 0) {  // compute_Rp!
    spmv(qp.A, ws.x_bar.data(), ws.Ax.data());
    for (int64_t i = 0; i < m; ++i) {
      const double ax = ws.Ax[i];
      const double corr = clamp_(ax, ws.AL[i], ws.AU[i]) - ax;
      const double f = sc.row_norm[i] * sc.b_scale;
      ws.Rp[i] = corr * f;
      ws.Ax[i] = ax * f;
    }
    r.err_Rp = norminf(ws.Rp) / (1.0 + std::max(sc.norm_b_org, norminf(ws.Ax)));
  } else {
    r.err_Rp = 0.0;
  }
  if (iter == 0) {
    for (int64_t i = 0; i < n; ++i) {
      const double lv = std::max(ws.l[i] - ws.x_bar[i], 0.0);
      const double uv = std::max(ws.x_bar[i] - ws.u[i], 0.0);
      ws.dx[i] = (lv + uv) * (sc.b_scale / sc.col_norm[i]);
    }
    r.err_Rp = std::max(r.err_Rp, norminf(ws.dx));
  }
  r.KKT = std::max(std::max(r.err_Rp, r.err_Rd), r.gap);
}

}  // namespace

namespace {

// ---------------------------------------------------------------------------
// Iteration updates, CPU loops (src/kernels.jl:2115-2832)
// ---------------------------------------------------------------------------

// update_zxw1_cpu! (src/kernels.jl:2301-2397): QP path step 1
void update_zxw1(WS& ws, const Prob& qp, double h1, double h2) {
  qp.Q.apply(ws.w, ws.Qw);
  const double f2s = 1.0 / (1.0 + ws.sigma * ws.lambda_max_Q), f1s = 1.0 - f2s;
  const double sigma = ws.sigma;
#pragma omp parallel for schedule(static) if (g_threads > 1) num_threads(g_threads)
  for (int64_t i = 0; i < ws.n; ++i) {
    const double x_i = ws.x[i], w_i = ws.w[i];
    const double tmp = -ws.Qw[i] + ws.ATy[i] - ws.c[i];
    const double z_raw = x_i + sigma * tmp;
    const double xb = clamp_(z_raw, ws.l[i], ws.u[i]);
    const double xh = 2.0 * xb - x_i;
    const double xn = muladd(h2, xh, h1 * ws.last_x[i]);
    const double wb = ws.Q_is_diag ? muladd(ws.fact1[i], w_i, ws.fact2[i] * xh)
                                   : muladd(f1s, w_i, f2s * xh);
    if (ws.to_check) {
      ws.dx[i] = xb - x_i;
      ws.x_bar[i] = xb;
      ws.z_bar[i] = (xb - z_raw) / sigma;
    }
    ws.x[i] = xn;
    ws.x_hat[i] = xh;
    ws.w_bar[i] = wb;
  }
}

// update_y_cpu! (src/kernels.jl:2682-2743): QP path step 2+3
void update_y(WS& ws, const Prob& qp, double h1, double h2) {
  if (ws.m == 0) return;
  qp.Q.apply(ws.w_bar, ws.Qw_bar);
  for (int64_t i = 0; i < ws.n; ++i) ws.tempv[i] = ws.x_hat[i] + ws.sigma * (ws.Qw[i] - ws.Qw_bar[i]);
  spmv(qp.A, ws.tempv.data(), ws.Ax.data());
  const double f1 = ws.lambda_max_A * ws.sigma, f2 = 1.0 / f1;
#pragma omp parallel for schedule(static) if (g_threads > 1) num_threads(g_threads)
  for (int64_t i = 0; i < ws.m; ++i) {
    const double yi = ws.y[i];
    const double s_raw = ws.Ax[i] - f1 * yi;
    const double s_proj = clamp_(s_raw, ws.AL[i], ws.AU[i]);
    const double yb = f2 * (s_proj - s_raw);
    const double yh = 2.0 * yb - yi;
    const double yn = muladd(h2, yh, h1 * ws.last_y[i]);
    if (ws.to_check) {
      ws.s[i] = s_proj;
      ws.dy[i] = yb - yi;
    }
    ws.y_bar[i] = yb;
    ws.y[i] = yn;
  }
}

// update_w2_cpu! (src/kernels.jl:2747-2832): QP path step 4
void update_w2(WS& ws, const Prob& qp, double h1, double h2) {
  spmv(qp.AT, ws.y_bar.data(), ws.ATy_bar.data());
  const double fs = ws.sigma / (1.0 + ws.sigma * ws.lambda_max_Q);
#pragma omp parallel for schedule(static) if (g_threads > 1) num_threads(g_threads)
  for (int64_t i = 0; i < ws.n; ++i) {
    const double w_i = ws.w[i], aty = ws.ATy[i], atyb = ws.ATy_bar[i];
    const double f = ws.Q_is_diag ? ws.fact[i] : fs;
    const double wbn = ws.w_bar[i] + f * (atyb - aty);
    const double wn = h1 * ws.last_w[i] + h2 * (2.0 * wbn - w_i);
    const double atyn = h1 * ws.last_ATy[i] + h2 * (2.0 * atyb - aty);
    ws.w[i] = wn;
    ws.ATy[i] = atyn;
    if (ws.to_check) {
      ws.w_bar[i] = wbn;
      ws.dw[i] = wbn - w_i;
      ws.ATdy[i] = atyb - aty;
    }
  }
}

// unified_update_zxw_cpu! (src/kernels.jl:2117-2238): QP-noC path
void update_zxw_noC(WS& ws, const Prob& qp, double h1, double h2) {
  spmv(qp.AT, ws.y.data(), ws.ATy.data());
  const double f2s = 1.0 / (1.0 + ws.sigma * ws.lambda_max_Q), f1s = 1.0 - f2s;
  const double sigma = ws.sigma;
#pragma omp parallel for schedule(static) if (g_threads > 1) num_threads(g_threads)
  for (int64_t i = 0; i < ws.n; ++i) {
    const double x_i = ws.x[i], w_i = ws.w[i];
    const double tmp = -ws.Qw[i] + ws.ATy[i] - ws.c[i];
    const double z_raw = x_i + sigma * tmp;
    const double xb = clamp_(z_raw, ws.l[i], ws.u[i]);
    const double xh = 2.0 * xb - x_i;
    const double xn = muladd(h2, xh, h1 * ws.last_x[i]);
    const double wb = ws.Q_is_diag ? muladd(ws.fact1[i], w_i, ws.fact2[i] * xh)
                                   : muladd(f1s, w_i, f2s * xh);
    const double wh = 2.0 * wb - w_i;
    const double wn = muladd(h2, wh, h1 * ws.last_w[i]);
    if (ws.to_check) {
      ws.dx[i] = xb - x_i;
      ws.x_bar[i] = xb;
      ws.z_bar[i] = (xb - z_raw) / sigma;
      ws.dw[i] = wb - w_i;
    }
    ws.x[i] = xn;
    ws.x_hat[i] = xh;
    ws.w_bar[i] = wb;
    ws.w[i] = wn;
  }
  qp.Q.apply(ws.w_bar, ws.Qw_bar);
  for (int64_t i = 0; i < ws.n; ++i) {
    const double qw = ws.Qw[i], qwb = ws.Qw_bar[i];
    const double qwh = 2.0 * qwb - qw;
    ws.Qw[i] = muladd(h2, qwh, h1 * ws.last_Qw[i]);
    ws.tempv[i] = ws.x_hat[i] + sigma * (qw - qwb);
  }
}

// unified_update_y_cpu! (src/kernels.jl:2242-2298): QP-noC path y step
void update_y_noC(WS& ws, const Prob& qp, double h1, double h2) {
  if (ws.m == 0) return;
  spmv(qp.A, ws.tempv.data(), ws.Ax.data());
  const double f1 = ws.lambda_max_A * ws.sigma, f2 = 1.0 / f1;
  for (int64_t i = 0; i < ws.m; ++i) {
    const double yi = ws.y[i];
    const double s_raw = ws.Ax[i] - f1 * yi;
    const double s_proj = clamp_(s_raw, ws.AL[i], ws.AU[i]);
    const double yb = f2 * (s_proj - s_raw);
    const double yh = 2.0 * yb - yi;
    const double yn = muladd(h2, yh, h1 * ws.last_y[i]);
    if (ws.to_check) {
      ws.s[i] = s_proj;
      ws.dy[i] = yb - yi;
    }
    ws.y_bar[i] = yb;
    ws.y[i] = yn;
  }
}

// unified_update_zx_cpu! (src/kernels.jl:2504-2578): LP path
void update_zx_LP(WS& ws, const Prob& qp, double h1, double h2) {
  spmv(qp.AT, ws.y.data(), ws.ATy.data());
  const double sigma = ws.sigma;
  for (int64_t i = 0; i < ws.n; ++i) {
    const double x_i = ws.x[i];
    const double z_raw = x_i + sigma * (ws.ATy[i] - ws.c[i]);
    const double xb = clamp_(z_raw, ws.l[i], ws.u[i]);
    const double xh = 2.0 * xb - x_i;
    const double xn = muladd(h2, xh, h1 * ws.last_x[i]);
    if (ws.to_check) {
      ws.dx[i] = xb - x_i;
      ws.x_bar[i] = xb;
      ws.z_bar[i] = (xb - z_raw) / sigma;
    }
    ws.x[i] = xn;
    ws.x_hat[i] = xh;
  }
}

// unified_update_y_noQ_cpu! (src/kernels.jl:2582-2658): LP path.  The
// partial variant writes y only (not y_bar), as in the reference CPU loop.
void update_y_LP(WS& ws, const Prob& qp, double h1, double h2) {
  if (ws.m == 0) return;
  spmv(qp.A, ws.x_hat.data(), ws.Ax.data());
  const double f1 = ws.lambda_max_A * ws.sigma, f2 = 1.0 / f1;
  for (int64_t i = 0; i < ws.m; ++i) {
    const double yi = ws.y[i];
    const double s_raw = ws.Ax[i] - f1 * yi;
    const double s_proj = clamp_(s_raw, ws.AL[i], ws.AU[i]);
    const double yb = f2 * (s_proj - s_raw);
    const double yh = 2.0 * yb - yi;
    const double yn = muladd(h2, yh, h1 * ws.last_y[i]);
    if (ws.to_check) {
      ws.s[i] = s_proj;
      ws.dy[i] = yb - yi;
      ws.y_bar[i] = yb;
    }
    ws.y[i] = yn;
  }
}

// update_zxw_LASSO_cpu! (src/kernels.jl:2400-2496)
void update_zxw_LASSO(WS& ws, const Prob& qp, double h1, double h2) {
  const double f2s = 1.0 / (1.0 + ws.sigma * ws.lambda_max_Q), f1s = 1.0 - f2s;
  qp.Q.apply(ws.w, ws.Qw);
  const double sigma = ws.sigma;
#pragma omp parallel for schedule(static) if (g_threads > 1) num_threads(g_threads)
  for (int64_t i = 0; i < ws.n; ++i) {
    const double x_i = ws.x[i], w_i = ws.w[i];
    const double tmp = -ws.Qw[i] + ws.ATy[i] - ws.c[i];
    const double z_raw = x_i + sigma * tmp;
    const double ls = ws.lambda[i] * sigma;
    const double shrink = std::max(std::fabs(z_raw) - ls, 0.0);
    const double xb = std::copysign(shrink, z_raw);
    const double xh = 2.0 * xb - x_i;
    const double xn = muladd(h2, xh, h1 * ws.last_x[i]);
    const double wb = muladd(f1s, w_i, f2s * xh);
    const double wn = muladd(h2, 2.0 * wb - w_i, h1 * ws.last_w[i]);
    if (ws.to_check) {
      ws.dx[i] = xb - x_i;
      ws.x_bar[i] = xb;
      ws.z_bar[i] = (xb - z_raw) / sigma;
      ws.dw[i] = wb - w_i;
    }
    ws.x[i] = xn;
    ws.x_hat[i] = xh;
    ws.w_bar[i] = wb;
    ws.w[i] = wn;
  }
}

// main_update_cpu! (src/algorithm.jl:945-972)
void main_update(WS& ws, const Prob& qp, const Restart& ri) {
  const double h1 = 1.0 / (ri.inner + 2.0), h2 = 1.0 - h1;
  if (qp.Q.kind == HPRQP_Q_LASSO) {
    update_zxw_LASSO(ws, qp, h1, h2);
    return;
  }
  if (qp.Q.kind == HPRQP_Q_QAP || qp.Q.nnz() > 0) {
    if (ws.noC) {
      update_zxw_noC(ws, qp, h1, h2);
      update_y_noC(ws, qp, h1, h2);
    } else {
      update_zxw1(ws, qp, h1, h2);
      update_y(ws, qp, h1, h2);
      update_w2(ws, qp, h1, h2);
    }
  } else {
    update_zx_LP(ws, qp, h1, h2);
    update_y_LP(ws, qp, h1, h2);
  }
}

// compute_M_norm! (src/algorithm.jl:689-739)
double compute_M_norm(WS& ws, const Prob& qp) {
  double M1 = 0.0, M2 = (1.0 / ws.sigma) * dot(ws.dx, ws.dx), M3 = 0.0;
  qp.Q.apply(ws.dw, ws.dQw);
  M2 -= 2.0 * dot(ws.dQw, ws.dx);
  if (ws.m > 0) {
    M1 = ws.sigma * ws.lambda_max_A * dot(ws.dy, ws.dy);
    spmv(qp.AT, ws.dy.data(), ws.ATdy.data());
    qp.Q.apply(ws.ATdy, ws.QATdy);
    M1 -= 2.0 * ws.sigma * dot(ws.dQw, ws.ATdy);
    M2 += 2.0 * dot(ws.ATdy, ws.dx);
    if (ws.Q_is_diag) {
      for (int64_t i = 0; i < ws.n; ++i) ws.ATdy[i] *= ws.fact_M[i];
      M3 = dot(ws.ATdy, ws.QATdy);
      M1 += ws.sigma * dot(ws.dQw, ws.dQw);
    } else {
      M3 = (ws.sigma * ws.sigma) / (1.0 + ws.sigma * ws.lambda_max_Q) * dot(ws.ATdy, ws.QATdy);
      M1 += ws.sigma * ws.lambda_max_Q * dot(ws.dw, ws.dQw);
    }
  } else if (!ws.Q_is_diag) {
    M1 = ws.sigma * ws.lambda_max_Q * dot(ws.dw, ws.dQw);
  }
  M2 += std::max(M1, 0.0);
  const double Mn = std::max(M2, 0.0) + std::max(M3, 0.0);
  return std::sqrt(Mn);
}

// golden (src/kernels.jl:1453-1486): minimise a x + b/x + c x^2/(1+d x)
double golden(double ap, double bp, double cp, double dp, double lo, double hi, double tol,
              int maxiter = 200) {
  auto f = [&](double x) { return ap * x + bp / x + cp * x * x / (1 + dp * x); };
  const double phi = (std::sqrt(5.0) - 1.0) / 2.0;
  double a = lo, b = hi, c = b - phi * (b - a), d = a + phi * (b - a);
  double fc = f(c), fd = f(d);
  for (int i = 0; i < maxiter; ++i) {
    if (fd < fc) {
      a = c; c = d; fc = fd;
      d = a + phi * (b - a);
      fd = f(d);
    } else {
      b = d; d = c; fd = fc;
      c = b - phi * (b - a);
      fc = f(c);
    }
    if ((b - a) < tol) break;
  }
  return 0.5 * (a + b);
}

// unified_golden_Q_diag, CPU (src/unified_operations.jl:348-386):
// minimise a x + b/x + x^2 * dot(c, d ./ (1 + x Q))
double golden_Q_diag(double a, double b, const Vec& Q, const Vec& c, const Vec& d, Vec& tempv,
                     double lo, double hi, double tol, int maxiter = 200) {
  const double phi = (std::sqrt(5.0) - 1.0) / 2.0;
  auto f = [&](double x) {
    for (size_t i = 0; i < Q.size(); ++i) tempv[i] = d[i] / (1.0 + x * Q[i]);
    return a * x + b / x + x * x * dot(c, tempv);
  };
  double x1 = hi - phi * (hi - lo), x2 = lo + phi * (hi - lo);
  double f1 = f(x1), f2 = f(x2);
  int it = 0;
  while (std::fabs(hi - lo) > tol * std::max(1.0, std::fabs(lo)) && it < maxiter) {
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
  return (f1 < f2) ? x1 : x2;
}

// update_sigma! (src/algorithm.jl:323-423)
void update_sigma(const hprqp_params& p, Restart& ri, WS& ws, const Prob& qp, const Res& r) {
  if (p.sigma_fixed || ri.restart_flag < 1) return;
  const double sigma_old = ws.sigma;
  for (int64_t i = 0; i < ws.n; ++i) {
    ws.dx[i] = ws.x_bar[i] - ws.last_x[i];
    ws.dw[i] = ws.w_bar[i] - ws.last_w[i];
  }
  qp.Q.apply(ws.dw, ws.dQw);
  double a = 0.0, b = dot(ws.dx, ws.dx), c = 0.0, d = 0.0;
  if (ws.m > 0) {
    for (int64_t i = 0; i < ws.m; ++i) ws.dy[i] = ws.y_bar[i] - ws.last_y[i];
    for (int64_t i = 0; i < ws.n; ++i) ws.ATdy[i] = ws.ATy_bar[i] - ws.last_ATy[i];
    qp.Q.apply(ws.ATdy, ws.QATdy);
    a = ws.lambda_max_A * dot(ws.dy, ws.dy) - 2 * dot(ws.dQw, ws.ATdy);
  }
  if (ws.Q_is_diag) {
    const double nq = norm2(ws.dQw);
    a += nq * nq;
  } else {
    a += ws.lambda_max_Q * dot(ws.dw, ws.dQw);
    if (ws.m > 0) {
      c = dot(ws.ATdy, ws.QATdy);
      d = ws.lambda_max_Q;
    }
  }
  a = std::max(a, 1e-12);
  b = std::max(b, 1e-12);
  double est;
  if (ws.Q_is_diag)
    est = ws.m > 0 ? golden_Q_diag(a, b, ws.diag_Q, ws.ATdy, ws.QATdy, ws.tempv, 1e-12, 1e12, 1e-13)
                   : std::sqrt(b / a);
  else
    est = ws.m > 0 ? golden(a, b, c, d, 1e-12, 1e12, 1e-13) : std::sqrt(b / a);
  const double fact = std::exp(-0.05 * (ri.current_gap / ri.best_gap));
  const double temp1 = std::max(std::min(r.err_Rd, r.err_Rp), std::min(r.gap, ri.current_gap));
  const double cand = std::exp(fact * std::log(est) + (1 - fact) * std::log(ri.best_sigma));
  double kappa;
  if (temp1 > 9e-10) kappa = 1.0;
  else if (temp1 > 5e-10) kappa = std::min(std::max(std::sqrt(r.err_Rd / r.err_Rp), 1e-2), 100.0);
  else kappa = std::min(std::max(r.err_Rd / r.err_Rp, 1e-2), 100.0);
  ws.sigma = kappa * cand;
  if (ws.Q_is_diag && std::fabs(sigma_old - ws.sigma) > 1e-15) update_Q_factors(ws);
}

// check_restart (src/algorithm.jl:441-492)
void check_restart(Restart& ri, int64_t iter, int64_t check_iter, double sigma) {
  ri.restart_flag = 0;
  if (ri.first_restart) {
    if (iter == check_iter) {
      ri.first_restart = false;
      ri.restart_flag = 1;
      ri.weighted_norm = ri.current_gap;
      ri.best_gap = ri.current_gap;
      ri.best_sigma = sigma;
    }
  } else if (iter % check_iter == 0) {
    if (ri.current_gap < 0) ri.current_gap = 1e-6;
    if (ri.current_gap <= 0.2 * ri.last_gap) { ri.sufficient++; ri.restart_flag = 1; }
    if (ri.current_gap <= 0.8 * ri.last_gap && ri.current_gap > 1.00 * ri.save_gap) {
      ri.necessary++;
      ri.restart_flag = 2;
    }
    const double fact = (ri.current_gap / ri.weighted_norm > 1e-1) ? 0.5 : 0.2;
    if (ri.inner >= fact * iter) { ri.long_++; ri.restart_flag = 3; }
    if (ri.best_gap > ri.current_gap) { ri.best_gap = ri.current_gap; ri.best_sigma = sigma; }
    ri.save_gap = ri.current_gap;
  }
}

// do_restart! (src/algorithm.jl:522-555)
void do_restart(Restart& ri, WS& ws, const Prob& qp) {
  if (ri.restart_flag <= 0) return;
  ws.x = ws.x_bar;
  ws.w = ws.w_bar;
  ws.last_x = ws.x_bar;
  ws.last_w = ws.w_bar;
  if (ws.m > 0) {
    ws.y = ws.y_bar;
    ws.last_y = ws.y_bar;
    spmv(qp.AT, ws.y_bar.data(), ws.ATy_bar.data());
    ws.last_ATy = ws.ATy_bar;
    ws.ATy = ws.ATy_bar;
  }
  if (ws.noC) {
    ws.Qw = ws.Qw_bar;
    ws.last_Qw = ws.Qw_bar;
  }
  ri.last_gap = ri.current_gap;
  ri.save_gap = INF;
  ri.times++;
  ri.inner = 0;
}

// print_step (src/algorithm.jl:1173-1175): max(10^floor(log10 iter)/10, 10)
double print_step(int64_t iter) {
  return std::max(std::pow(10.0, std::floor(std::log10((double)iter))) / 10.0, 10.0);
}
bool on_print_schedule(int64_t iter, const hprqp_params& p) {
  if (p.print_frequency == -1) return std::fmod((double)iter, print_step(iter)) == 0.0;
  return iter % p.print_frequency == 0;
}

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

// Build the internal problem from the C description (QP_info_cpu fields).
int build(const hprqp_problem* pr, Prob& qp) {
  if (!pr || pr->n < 0 || pr->m < 0) return fail(HPRQP_E_ARG, "bad problem sizes");
  const int base = pr->index_base;
  qp.n = pr->n;
  qp.m = pr->m;
  const int64_t n = qp.n, m = qp.m;
  qp.A = (m > 0 && pr->A_colptr) ? csc_to_csr(m, n, pr->A_colptr, pr->A_rowval, pr->A_nzval, base)
                                 : Csr{m, n, std::vector<int64_t>(m + 1, 0), {}, {}};
  qp.AT = transpose(qp.A);
  qp.c.assign(pr->c, pr->c + n);
  qp.AL.assign(pr->AL ? pr->AL : pr->c, (pr->AL ? pr->AL : pr->c) + (pr->AL ? m : 0));
  qp.AU.assign(pr->AU ? pr->AU : pr->c, (pr->AU ? pr->AU : pr->c) + (pr->AU ? m : 0));
  qp.l.assign(pr->l, pr->l + n);
  qp.u.assign(pr->u, pr->u + n);
  qp.obj_constant = pr->obj_constant;
  qp.lambda = pr->lambda;
  qp.Q.kind = pr->Q_kind;
  qp.Q.n = n;
  if (pr->Q_kind == HPRQP_Q_SPARSE) {
    if (pr->Q_colptr) qp.Q.Q = csc_to_csr(n, n, pr->Q_colptr, pr->Q_rowval, pr->Q_nzval, base);
    else qp.Q.Q = Csr{n, n, std::vector<int64_t>(n + 1, 0), {}, {}};
  } else if (pr->Q_kind == HPRQP_Q_LASSO) {
    qp.Q.L = csc_to_csr(pr->lasso_m, n, pr->L_colptr, pr->L_rowval, pr->L_nzval, base);
    qp.Q.LT = transpose(qp.Q.L);
    qp.Q.temp.assign(pr->lasso_m, 0.0);
  } else if (pr->Q_kind == HPRQP_Q_QAP) {
    const int64_t N = pr->qap_n;
    if (N * N != n) return fail(HPRQP_E_ARG, "QAP: n must equal qap_n^2");
    qp.Q.qn = N;
    qp.Q.qA.assign(pr->qap_A, pr->qap_A + N * N);
    qp.Q.qB.assign(pr->qap_B, pr->qap_B + N * N);
    qp.Q.qS.assign(pr->qap_S, pr->qap_S + N * N);
    qp.Q.qT.assign(pr->qap_T, pr->qap_T + N * N);
    qp.Q.tmp.assign(N * N, 0.0);
  } else {
    return fail(HPRQP_E_ARG, "unknown Q_kind");
  }
  return HPRQP_OK;
}

void alloc_ws(WS& ws, int64_t n, int64_t m) {
  ws.n = n;
  ws.m = m;
  for (Vec* v : {&ws.w, &ws.w_hat, &ws.w_bar, &ws.dw, &ws.x, &ws.x_hat, &ws.x_bar, &ws.dx, &ws.z_bar,
                 &ws.Rd, &ws.ATy, &ws.ATy_bar, &ws.ATdy, &ws.QATdy, &ws.Qw, &ws.Qw_hat, &ws.Qw_bar,
                 &ws.Qx, &ws.dQw, &ws.last_x, &ws.last_Qw, &ws.last_w, &ws.last_ATy, &ws.tempv,
                 &ws.fact1, &ws.fact2, &ws.fact, &ws.fact_M})
    v->assign(n, 0.0);
  for (Vec* v : {&ws.y, &ws.y_hat, &ws.y_bar, &ws.dy, &ws.Rp, &ws.Ax, &ws.s, &ws.last_y})
    v->assign(m, 0.0);
}

}  // namespace

extern "C" {

const char* oracle_last_error(void) { return g_err.c_str(); }

// Scalar trace of the next oracle_solve (then cleared): per traced iteration
// the sigma of the step and its Halpern inner counter (0 after a restart).
static double* g_sig_trace = nullptr;
static int64_t* g_inner_trace = nullptr;
void oracle_set_scalar_trace(double* sigma_trace, int64_t* inner_trace) {
  g_sig_trace = sigma_trace;
  g_inner_trace = inner_trace;
}

// solve (src/algorithm.jl:1904-2039), CPU path, with optional iterate trace.
// `threads` = 1 reproduces the reference's single-threaded CPU loops;
// > 1 parallelises SpMV and the update loops with OpenMP (timing only).
int oracle_solve(const hprqp_problem* pr, const hprqp_params* params, const double* x0,
                 const double* y0, hprqp_result* res, double* xo, double* yo, double* zo,
                 double* wo, int64_t trace_iters, double* xt, double* yt, double* wt,
                 int32_t threads) {
  g_err.clear();
  g_threads = threads < 1 ? 1 : threads;
  double* const sig_t = g_sig_trace;
  int64_t* const inner_t = g_inner_trace;
  g_sig_trace = nullptr;
  g_inner_trace = nullptr;
  if (!params || !res) return fail(HPRQP_E_ARG, "null params/result");
  const hprqp_params& p = *params;
  const double setup_start = now_s();
  Prob qp;
  int rc = build(pr, qp);
  if (rc) return rc;
  const int64_t n = qp.n, m = qp.m;
  Scaling sc = scaling(qp, p);
  WS ws;
  alloc_ws(ws, n, m);
  check_Q_diagonal(qp, ws.diag_Q, ws.Q_is_diag);
  ws.c = qp.c; ws.AL = qp.AL; ws.AU = qp.AU; ws.l = qp.l; ws.u = qp.u;
  ws.lambda.assign(n, qp.lambda);
  // allocate_workspace sigma rule (src/algorithm.jl:838-851)
  if (p.sigma == -1) {
    ws.sigma = (sc.norm_c > 1e-16 && sc.norm_b > 1e-16 && sc.norm_b < 1e16 && sc.norm_c < 1e16)
                   ? sc.norm_b / sc.norm_c : 1.0;
  } else if (p.sigma > 0) {
    ws.sigma = p.sigma;
  } else {
    return fail(HPRQP_E_ARG, "Invalid sigma value");
  }
  const double setup_time = now_s() - setup_start;
  const double t0 = now_s();
  // estimate_eigenvalues (src/algorithm.jl:1407-1440)
  if (m > 0)
    ws.lambda_max_A = p.lambda_max_A_override > 0 ? p.lambda_max_A_override
                                                  : power_iteration_A(qp) * p.eig_factor;
  if (qp.Q.is_operator()) {
    ws.lambda_max_Q = p.lambda_max_Q_override > 0 ? p.lambda_max_Q_override
                                                  : power_iteration_Q(qp) * p.eig_factor;
  } else if (qp.Q.nnz() > 0) {
    if (!ws.Q_is_diag)
      ws.lambda_max_Q = p.lambda_max_Q_override > 0 ? p.lambda_max_Q_override
                                                    : power_iteration_Q(qp) * p.eig_factor;
    else
      ws.lambda_max_Q = *std::max_element(qp.Q.Q.val.begin(), qp.Q.Q.val.end());
  }
  const double power_time = now_s() - t0;
  // process_initial_points! (src/algorithm.jl:1783-1836)
  if (x0) {
    for (int64_t i = 0; i < n; ++i) {
      const double v = x0[i] * sc.col_norm[i] / sc.b_scale;
      ws.x[i] = ws.x_bar[i] = ws.last_x[i] = ws.w[i] = ws.w_bar[i] = ws.last_w[i] = v;
    }
  }
  if (y0) {
    for (int64_t i = 0; i < m; ++i) {
      const double v = y0[i] * sc.row_norm[i] / sc.c_scale;
      ws.y[i] = ws.y_bar[i] = ws.last_y[i] = v;
    }
    if (m > 0) {
      spmv(qp.AT, ws.y_bar.data(), ws.ATy_bar.data());
      ws.ATy = ws.ATy_bar;
      ws.last_ATy = ws.ATy_bar;
    }
    qp.Q.apply(ws.x_bar, ws.Qx);
    for (int64_t i = 0; i < n; ++i) {
      const double tmp = -ws.Qx[i] + ws.ATy_bar[i] - ws.c[i];
      const double z_raw = ws.x_bar[i] + ws.sigma * tmp;
      ws.z_bar[i] = (ws.x_bar[i] - z_raw) / ws.sigma;
    }
    if (m > 0) {
      spmv(qp.A, ws.x_bar.data(), ws.Ax.data());
      const double f1 = ws.lambda_max_A * ws.sigma;
      for (int64_t i = 0; i < m; ++i) ws.s[i] = clamp_(ws.Ax[i] - f1 * ws.y[i], ws.AL[i], ws.AU[i]);
    }
  }
  Restart ri;
  ri.best_sigma = ws.sigma;
  if (ws.Q_is_diag) update_Q_factors(ws);
  int64_t nfree = 0;
  for (int64_t i = 0; i < n; ++i) nfree += (pr->l[i] == -INF && pr->u[i] == INF);
  ws.noC = nfree > 0.8 * n;
  const int64_t check_iter = p.check_iter;
  Res r;
  int64_t iter_4 = 0, iter_6 = 0;
  double time_4 = 0, time_6 = 0;
  bool first_4 = true, first_6 = true;
  if (p.verbose)
    std::printf(" iter     errRp        errRd         p_obj           d_obj          gap        sigma       time\n");
  for (int64_t iter = 0; iter <= p.max_iter; ++iter) {
    const bool time_up = now_s() - t0 > p.time_limit;
    const bool print_yes = on_print_schedule(iter, p) || iter == p.max_iter || time_up;
    if (iter % check_iter == 0 || print_yes) compute_residuals(ws, qp, sc, r, p, iter);
    int status = -1;
    if (r.KKT < p.stoptol) status = HPRQP_STATUS_OPTIMAL;
    else if (iter == p.max_iter) status = HPRQP_STATUS_MAX_ITER;
    else if (now_s() - t0 > p.time_limit) status = HPRQP_STATUS_TIME_LIMIT;
    check_restart(ri, iter, check_iter, ws.sigma);
    update_sigma(p, ri, ws, qp, r);
    do_restart(ri, ws, qp);
    if ((print_yes || status >= 0) && p.verbose)
      std::printf("%5lld    %3.2e    %3.2e    %+7.6e    %+7.6e    %3.2e    %3.2e    %6.2f\n",
                  (long long)iter, r.err_Rp, r.err_Rd, r.pobj, r.dobj, r.gap, ws.sigma, now_s() - t0);
    if (r.KKT < 1e-4 && first_4) { time_4 = now_s() - t0; iter_4 = iter; first_4 = false; }
    if (r.KKT < 1e-6 && first_6) { time_6 = now_s() - t0; iter_6 = iter; first_6 = false; }
    if (status >= 0) {
      // handle_termination + collect_results! (src/algorithm.jl:1039-1097, 611-643)
      std::memset(res, 0, sizeof(*res));
      res->iter = iter;
      res->time = now_s() - t0;
      res->power_time = power_time;
      res->setup_time = setup_time;
      res->residuals = r.KKT;
      res->primal_obj = r.pobj;
      res->dual_obj = r.dobj;
      res->gap = r.gap;
      res->err_Rp = r.err_Rp;
      res->err_Rd = r.err_Rd;
      res->status = status;
      res->Q_is_diag = ws.Q_is_diag;
      res->sigma = ws.sigma;
      res->lambda_max_A = ws.lambda_max_A;
      res->lambda_max_Q = ws.lambda_max_Q;
      res->restarts = ri.times;
      res->time_4 = time_4 == 0.0 ? res->time : time_4;
      res->iter_4 = iter_4 == 0 ? iter : iter_4;
      res->time_6 = time_6 == 0.0 ? res->time : time_6;
      res->iter_6 = iter_6 == 0 ? iter : iter_6;
      for (int64_t i = 0; i < n; ++i) {
        if (xo) xo[i] = sc.b_scale * (ws.x_bar[i] / sc.col_norm[i]);
        if (wo) wo[i] = sc.b_scale * (ws.w_bar[i] / sc.col_norm[i]);
        if (zo) zo[i] = sc.c_scale * (ws.z_bar[i] * sc.col_norm[i]);
      }
      if (yo)
        for (int64_t i = 0; i < m; ++i) yo[i] = sc.c_scale * (ws.y_bar[i] / sc.row_norm[i]);
      return HPRQP_OK;
    }
    const int64_t next = iter + 1;
    ws.to_check = (next % check_iter == 0) || (ri.restart_flag > 0) || on_print_schedule(next, p);
    // perform_iteration_step! (src/algorithm.jl:1881-1900)
    const int64_t inner_used = ri.inner;
    main_update(ws, qp, ri);
    if (ri.restart_flag > 0) ri.last_gap = compute_M_norm(ws, qp);
    if ((iter + 1) % check_iter == 0) ri.current_gap = compute_M_norm(ws, qp);
    ri.inner++;
    if (next <= trace_iters) {
      if (xt) std::memcpy(xt + (next - 1) * n, ws.x.data(), n * sizeof(double));
      if (yt && m) std::memcpy(yt + (next - 1) * m, ws.y.data(), m * sizeof(double));
      if (wt) std::memcpy(wt + (next - 1) * n, ws.w.data(), n * sizeof(double));
      if (sig_t) sig_t[next - 1] = ws.sigma;
      if (inner_t) inner_t[next - 1] = inner_used;
    }
  }
  return fail(HPRQP_E_STATE, "loop exited without status");
}

}  // extern "C"
