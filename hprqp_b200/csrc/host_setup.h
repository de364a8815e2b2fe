// host_setup.h — host-side problem intake and scaling for libhprqp.
//
// Loading converts the caller's CSC arrays (QP_info_cpu, src/structs.jl:98-149)
// into CSR and validates them.  Scaling restates the reference's scaling!
// (src/utils.jl:350-804, CPU branch): 10 Ruiz passes on [Q; A], one
// Pock-Chambolle pass, b/c scaling disabled, Q symmetrised afterwards, and
// check_Q_diagonal (src/utils.jl:827-855).  It runs on the host once per
// prepare, row-parallel (OpenMP): A and A', Q and Q' are scaled side by
// side with the same arithmetic, so column maxima and sums are row sweeps
// of the transposes and every result is bitwise the sequential one.  The
// scaled arrays are then uploaded to HBM.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <memory>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#include "../../include/hprqp.h"
#include "pool.h"

namespace hprqp {

// Allocator whose value-initialisation of trivial elements is default-
// initialisation: resize leaves them uninitialised.  The host arrays of a
// problem (hundreds of MB for the large configurations) are filled in full
// right after they are sized, mostly by parallel loops; std::allocator's
// zero-fill would first touch every page on one thread (38 ms per 100 MB
// on the B200 host, against 4 ms for the parallel first touch).  Arrays of
// 4 MiB and more come from the process's host block cache (host_take), so
// that the next problem's arrays of similar sizes reuse pages that are
// already mapped and faulted in.
template <typename T, typename A = std::allocator<T>>
struct NoInitAlloc : A {
  template <typename U>
  struct rebind {
    using other = NoInitAlloc<U, typename std::allocator_traits<A>::template rebind_alloc<U>>;
  };
  using A::A;
  NoInitAlloc() = default;
  static constexpr size_t kLarge = size_t(4) << 20;
  T* allocate(size_t n) {
    if (n * sizeof(T) < kLarge) return A::allocate(n);
    return static_cast<T*>(host_take(n * sizeof(T)));
  }
  void deallocate(T* p, size_t n) {
    if (n * sizeof(T) < kLarge) return A::deallocate(p, n);
    host_give(p);
  }
  template <typename U>
  void construct(U* p) noexcept(std::is_nothrow_default_constructible<U>::value) {
    ::new (static_cast<void*>(p)) U;
  }
  template <typename U, typename... Args>
  void construct(U* p, Args&&... args) {
    std::allocator_traits<A>::construct(static_cast<A&>(*this), p, std::forward<Args>(args)...);
  }
};
template <typename T>
using hvec = std::vector<T, NoInitAlloc<T>>;

struct HCsr {
  int64_t rows = 0, cols = 0;
  hvec<int> ptr, col;
  hvec<double> val;
  int64_t nnz() const { return (int64_t)col.size(); }
};

struct HostProblem {  // the loaded, unscaled problem
  int64_t n = 0, m = 0;
  int Q_kind = HPRQP_Q_SPARSE;
  HCsr A;   // m x n
  HCsr AT;  // n x m: the caller's CSC of A read as CSR of A'
  HCsr QT;  // n x n: the caller's CSC of Q read as CSR of Q' (sparse kind)
  hvec<double> c, AL, AU, l, u;
  double obj_constant = 0.0, lambda = 0.0;
  HCsr Q;  // n x n (sparse kind)
  HCsr L;   // lasso data, lasso_m x n
  HCsr LT;  // its transpose (the caller's CSC read as CSR)
  int64_t qn = 0;
  hvec<double> qA, qB, qS, qT;  // column-major qn x qn
  bool loaded = false;
};

// Device copies of the scaled problem left by the GPU scaling: the engines
// copy from them on the device (FP64) or cast them there (FP32) instead of
// uploading the host arrays a second time.
struct DevCsrView {
  const int* ptr = nullptr;
  const int* col = nullptr;
  const double* val = nullptr;
};
struct DevScaled {
  PoolBlocks mem;  // owns every array below
  DevCsrView A, AT, Q;
  const double *c = nullptr, *l = nullptr, *u = nullptr, *AL = nullptr, *AU = nullptr;
  const double *row_norm = nullptr, *col_norm = nullptr;
};

struct Prepared {  // scaled problem + scaling info (Scaling_info_cpu)
  std::shared_ptr<DevScaled> dev;  // set by the GPU scaling, null after host scaling
  HCsr A, AT, Q;  // with `dev`, A and A' carry their patterns only (values on the device)
  // With `dev`, the patterns of A, A' and (when Q's pattern is symmetric,
  // so that it is S's) Q are the loaded problem's, not copied: these point
  // to its records, and A, AT, Q above stay empty.  Apat() etc. give the
  // pattern in either case.
  const HCsr* A_pat = nullptr;
  const HCsr* AT_pat = nullptr;
  const HCsr* Q_pat = nullptr;
  const HCsr& Apat() const { return A_pat ? *A_pat : A; }
  const HCsr& ATpat() const { return AT_pat ? *AT_pat : AT; }
  const HCsr& Qpat() const { return Q_pat ? *Q_pat : Q; }
  hvec<double> c, AL, AU, l, u, row_norm, col_norm, diag_Q;
  double norm_b = 0, norm_c = 0, norm_b_org = 0, norm_c_org = 0;
  double b_scale = 1.0, c_scale = 1.0;
  bool Q_is_diag = false;
  double Q_maxval = 0.0;  // maximum(Q.nzval), lambda_max_Q of a diagonal Q
  bool noC = false;
  int ruiz = -1, pc = -1;
};

// Validate and copy; throws Error(HPRQP_E_ARG) on bad input.
void load_problem(const hprqp_problem* pr, HostProblem& hp);
// scaling! + check_Q_diagonal + the noC rule (src/algorithm.jl:1969-1974).
void prepare_problem(const HostProblem& hp, const hprqp_params& p, Prepared& out);
// The same for a sparse Q with the matrix scaling on the GPU (scale.cu):
// bitwise the host result, with the scaled arrays copied back into `out`.
// h2d / d2h: byte counters of the handle, incremented by every host<->device
// copy the scaling makes
void prepare_problem_gpu(const HostProblem& hp, const hprqp_params& p, Prepared& out, cudaStream_t st,
                         int64_t* h2d, int64_t* d2h);
// the tails shared by both: norms, check_Q_diagonal and Q_maxval on the
// scaled sparse Q; the noC rule
void finish_sparse(Prepared& o, int64_t n);
// the vector norms of finish_sparse alone (the GPU scaling checks Q's
// diagonal on the device)
void finish_norms(Prepared& o);
void finish_common(const HostProblem& hp, Prepared& o);
double norm_b_inf_org(const hvec<double>& AL, const hvec<double>& AU);
double norm_inf(const hvec<double>& v);
HCsr transpose(const HCsr& A);
// Pattern of the Gram matrix G = A'A (n x n) from A (CSR) and A' (CSR of
// the transpose): row p holds the columns of every row of A that has an
// entry in column p, sorted and without repeats.  Only ptr and col are
// filled (the values are formed on the device).  Returns false, leaving G
// empty, when A' has a row that is not strictly increasing (the device
// merge needs sorted rows) or when the product's work, sum over the rows of
// A of their length squared, exceeds max_work.
bool gram_pattern(const HCsr& A, const HCsr& AT, int64_t max_work, HCsr& G);
// dst = src with the copy split over host threads, which also first-touch
// dst's pages (the preparation copies ~100 MB of patterns and vectors).
template <typename T>
void par_copy(hvec<T>& dst, const hvec<T>& src);
// dst = src[0, len) likewise, from a caller's array
template <typename T>
void par_copy(hvec<T>& dst, const T* src, int64_t len);
// Host threads for a row-parallel loop over `work` items: 1 below ~64k
// items (a parallel region costs more than it saves there), else at most
// 16 (the loops are memory-bound; more threads only add wake-up cost).
int host_threads(int64_t work);
// splitmix64 + Box-Muller start vector of the power method (+1e-8).
std::vector<double> power_start_vector(int64_t len);
// The same stream, produced incrementally into a caller buffer.
struct StartVectorStream {
  uint64_t s = 1;
  void fill(double* out, int64_t count);
};

}  // namespace hprqp
