// engine.cuh — device state and kernel launch layer of the HPR-QP engine.
//
// Engine<V> owns the scaled problem and every iterate in HBM (V = double
// for the FP64 path, float for the FP32 phase; Halpern anchors stay double)
// and exposes the steps of the reference loop as stream-ordered launches:
// step() = main_update (src/algorithm.jl:945-972), residuals() =
// compute_residuals!, mnorm() = compute_M_norm!, sigma_stats() = the
// reductions of update_sigma!, restart() = do_restart!, power_*() =
// power_iteration_A/Q.  Scalars from reductions land in a device slot array
// that the host reads once per residual check.
#pragma once


#include <memory>
#include <vector>

#include "pool.h"
#include "host_setup.h"
#include "kernels.cuh"

namespace hprqp {

enum Path { PATH_QP = 0, PATH_NOC = 1, PATH_LP = 2, PATH_LASSO = 3 };

// Device scalar slot layout
enum Slot {
  S_RES_N = 0,     // 8 slots: EpiResN
  S_RES_M = 8,     // 3 slots: EpiResM
  S_MN_CUR = 16,   // 8 + 1 slots: M-norm for current_gap
  S_MN_LAST = 32,  // 8 + 1 slots: M-norm for last_gap
  S_SIG = 48,      // 5 + 1 slots: sigma statistics
  S_GOLD = 56,     // golden-section result (diagonal Q)
  S_POW = 64,      // power method (A A') working scalars (4)
  S_POW_Q = 72,    // power method (Q) working scalars (4)
  S_POWLOG = 128,  // power method log A A': (lambda, err) per iteration
  kPowChunk = 32,
  S_POWLOG_Q = S_POWLOG + 2 * kPowChunk,  // power method log Q
  kNumSlots = S_POWLOG_Q + 2 * kPowChunk,
};

struct DeviceMem : PoolBlocks {  // owns blocks of the library's device memory pool
  template <typename T>
  T* alloc(int64_t count) { return (T*)get(sizeof(T) * (size_t)(count > 0 ? count : 1)); }
};

struct Common {  // per-handle resources shared by the engines
  cudaStream_t stream = nullptr;
  cudaStream_t stream2 = nullptr;  // second chain of the power method
  double* d_scal = nullptr;
  double* h_scal = nullptr;  // pinned mirror
  ReduceWs rws{}, rws2{};
  int64_t launches = 0;
  int64_t h2d = 0, d2h = 0;  // bytes copied host<->device
  int num_sms = 148;
  bool pdl = true;           // programmatic dependent launch between kernels
  // persistent power method: partials [2][2][grid][3], barrier counter +
  // status word; CTAs per SM (0 = as many as fit, capped at 2)
  double* pow_part = nullptr;
  unsigned* pow_bar = nullptr;
  int pow_ctas_per_sm = 0;
  // the graph-captured chains measured faster than the persistent kernel on
  // the 700x700 grid (99 vs 112 ms); HPRQP_POWER_PERSISTENT=1 selects it
  bool pow_persistent = false;
  int reduce_cap = kMaxReduceGrid;  // CTAs of a grid-stride reduction (HPRQP_REDUCE_CAP)
  bool pow_prefer_ell = false;  // HPRQP_POWER_ELL=1: power sweeps on ELL copies
  bool pow_split = false;       // HPRQP_POWER_SPLIT=1: product pass + separate dot reduction
  // A A' chain on the Gram matrix A'A (HPRQP_POWER_GRAM): -1 = when A'A has
  // at most 3 nnz(A) entries, 0 = never, 1 = whenever its product work
  // (sum of squared row lengths of A) stays within 64 nnz(A)
  int pow_gram = -1;
  // pass epilogues prefetch their row operands before the product
  // (HPRQP_EPI_PREFETCH: 0 off, 1 into L1, 2 into L2); measured no faster
  // on the 700x700 grid (FP32 iteration 40.3 vs 40.3 us, FP64 50.3 vs
  // 48.4 us), so off by default
  int epi_prefetch = 0;
  // ELL passes load their constant data before waiting on the previous kernel
  // (HPRQP_ELL_PROLOGUE: 0 off = k_row_pass, 1 the matrix rows, 2 the matrix
  // rows and the epilogue's problem data).  Measured on the 700x700 grid, ELL
  // for Q, A, A': FP32 plain iteration 43.4 / 28.6 / 29.5 us, FP64 48.3 /
  // 45.1 / 46.4 us for 0 / 1 / 2
  int ell_prologue = 1;
  int pow_rows_preloaded = 2;  // rows per thread whose power-step matrix entries load before the wait (1 or 2)
  // power chains folded once per chunk (HPRQP_POWER_CHUNK_FOLD=0: per step)
  bool pow_chunk_fold = true;
  // row-schedule autotuner (timed); HPRQP_AUTOTUNE=0 applies a fixed rule
  // instead, e.g. under a profiler, whose serialisation makes the timings
  // meaningless
  bool autotune = true;
  // timed schedule choices are kept per process by sparsity signature and
  // reused for a matrix of the same pattern (HPRQP_SCHED_CACHE=0: time always)
  bool sched_cache = true;
  hprqp_qmap_fn qmap = nullptr;  // a custom Q operator's callback (HPRQP_Q_CUSTOM)
  void* qmap_user = nullptr;
  bool tc_qap = true;  // FP32 QAP products on the 3xTF32 tensor-core GEMM (else the CUDA-core k_qap_gemm)
  DeviceMem mem;
  void init();
  ~Common();
  void sync_read(int first, int count);
  void to_dev(void* d, const void* h, size_t bytes) {
    if (!bytes) return;
    h2d_staged(d, h, bytes, stream);
    h2d += (int64_t)bytes;
  }
  void to_host(void* h, const void* d, size_t bytes) {  // (1 MiB and more: synchronous, pinned chunks)
    if (!bytes) return;
    if (bytes >= (1u << 20)) d2h_staged(h, d, bytes, stream);
    else HPRQP_CUDA(cudaMemcpyAsync(h, d, bytes, cudaMemcpyDeviceToHost, stream));
    d2h += (int64_t)bytes;
  }
};

struct PendingMnorm {
  bool active = false;
  int slot = 0;
  double sigma = 0, lamA = 0, lamQ = 0;
};

template <typename V>
class Engine {
 public:
  // power_engine: this engine runs the power method (it then builds the
  // Gram matrix of the A A' chain where that applies)
  Engine(Common& cm, const HostProblem& hp, const Prepared& pp, int path, int tpr_mode_Q, int tpr_mode_A,
         bool power_engine = true);
  int64_t n, m;
  int path;
  bool Q_is_diag, has_Q_sparse, is_qap, is_lasso;
  bool is_custom = false;  // Q through the user's callback
  bool is_op = false;      // an operator Q applied as a whole product (QAP or custom)
  double b_scale, c_scale, norm_b_org, norm_c_org;
  double sigma = 1.0, lamA = 0.0, lamQ = 0.0;
  double lam_l1 = 0.0;   // lambda in the L1 objective term (problem_type LASSO)
  double lasso_lam = 0;  // soft-threshold lambda

  // iteration state (V) and anchors (double)
  V *x, *x_hat, *x_bar, *dx, *w, *w_bar, *dw, *z_bar, *Qw, *Qw_bar, *ATy, *ATy_bar, *ATdy, *QATdy,
      *dQw, *Qx, *tempv, *c, *l, *u, *col_norm, *fact1, *fact2, *fact, *fact_M, *diag_Q;
  V *y, *y_bar, *dy, *s, *Ax, *AL, *AU, *row_norm;
  // Halpern anchors: every value they take is an iterate of this engine's
  // storage type (restart and initial points copy V values), so V holds
  // them exactly
  V *last_x, *last_w, *last_ATy, *last_Qw, *last_y;
  V* ltemp = nullptr;                 // LASSO A_d w
  V* ltemp2 = nullptr;                // LASSO A_d z of the Q power chain
  double *stage_n, *stage_m;          // FP64 staging for host copies
  V *pz, *pq, *pt;                    // power method vectors

  DCsr<V> A, AT, Q, L, LT;
  // Gram matrix G = A'A (n x n) of the A A' power chain; its values are
  // formed on the device at every power method (gram_values)
  DCsr<V> G;
  bool gram = false;
  void autotune_gram(uint64_t key);  // (public: it launches device lambdas); key: schedule cache, 0 = none
  void autotune_power_Q(uint64_t key);
  template <typename Step>
  void tune_reduce(DCsr<V>& M, Step step, uint64_t key = 0);
  DCsr<V> Qp;  // Q under the schedule of its power step
  bool power_ready = false;
  ~Engine();
  cudaGraphExec_t pow_exec[4] = {nullptr, nullptr, nullptr, nullptr};  // power chunk graphs by active chains
  int64_t pow_exec_launches[4] = {0, 0, 0, 0};
  int pow_exec_key = -1;
  double *pow_cf_part = nullptr, *pow_cf_tot = nullptr;  // chunk-fold partials and totals
  int64_t pow_cf_region = 0;                              // doubles per chain in pow_cf_part
  double *gq0 = nullptr, *gq1 = nullptr;                  // the chunk-fold Q chain's FP64 state
  void power_setup(const Prepared& pp, int tpr_A, int tpr_Q);
  double *gu0 = nullptr, *gu1 = nullptr;  // the Gram chain's state u_k (FP64 in both engines)
  V *qA = nullptr, *qB = nullptr, *qS = nullptr, *qT = nullptr, *qTmp = nullptr;
  int* qap_n_d = nullptr;              // one-instance descriptor of k_qap_gemm
  int64_t* qap_off_d = nullptr;
  unsigned char* qap_on_d = nullptr;
  float* qws = nullptr;  // TF32 operand images of the tensor-core QAP products

  void reset_state();
  void set_sigma(double s);  // + diagonal factors (unified_update_Q_factors!)
  void step(bool full, double h1, double h2);
  void residuals_launch(bool with_bounds);
  void mnorm_launch(int slot);
  void sigma_stats_launch();
  void golden_diag_launch(double a, double b);
  void restart();
  void initial_points(const double* x0, const double* y0);
  void collect(double* x_out, double* y_out, double* z_out, double* w_out);
  void trace_copy(double* xt, double* yt, double* wt);
  // checkpoint helpers: a state vector to / from FP64 host memory (exact:
  // every V value is a double), and the bar iterates into FP64 device copies
  void vec_to_host(const V* src, int64_t len, double* dst);
  void vec_from_host(V* dst, const double* src, int64_t len);
  void bars_to_device(double* xb, double* yb, double* zb, double* wb);
  // Both power methods (A A' and Q) at once, on two streams; want_* select
  // which run.  Returns lambda estimates (not yet times eig_factor).
  void power_both(bool want_A, bool want_Q, double tol, int max_it, double* lamA_out, double* lamQ_out,
                  int64_t* itA, int64_t* itQ);
  bool power_persistent(bool onA, bool onQ, double tol, int max_it, double* lamA_out, double* lamQ_out,
                        int64_t* itA, int64_t* itQ);
  V *pz2 = nullptr, *pq2 = nullptr, *pt2 = nullptr;  // Q chain vectors
  template <typename W>
  void import_state(const Engine<W>& o);  // precision switch (FP32 -> FP64)

  void apply_Q(const V* xin, V* yout);  // Qmap! into a vector
  template <typename Epi>
  void mat_rows(const DCsr<V>& M, const V* xin, const Epi& e);  // fused pass on M's format
  Common& cm;

  // pass profiling: when `prof` is set, step() records an event before the
  // first pass and after every pass
  std::vector<cudaEvent_t>* prof = nullptr;
  size_t prof_k = 0;
  void mark() {
    if (prof && prof_k < prof->size()) HPRQP_CUDA(cudaEventRecord((*prof)[prof_k++], cm.stream));
  }
  int npasses() const {
    return path == PATH_QP ? (m > 0 ? 4 : 2) : path == PATH_NOC ? (m > 0 ? 3 : 2) : path == PATH_LP ? (m > 0 ? 2 : 1) : 2;
  }
  void pass_info(int k, const char** name, double* bytes, int* tpr) const;
  // algorithmic HBM bytes of one power-method step of chain `which`
  // (0 = A A', 1 = Q or the LASSO operator); 0 for the QAP operator
  double power_step_bytes(int which) const;

 private:
  DeviceMem mem;
  void upload_csr(const HCsr& h, DCsr<V>& d, int tpr_mode, const DevCsrView* dsrc = nullptr);
  V* vec_in(const hvec<double>& h, const double* dsrc, int64_t len);
  int autotune(DCsr<V>& d);
  void spmv(const DCsr<V>& M, const V* xin, V* yout, double scale = 1.0);
  void build_sell(const HCsr& h, DCsr<V>& d);
  void build_ell(const HCsr& h, DCsr<V>& d);
  void build_split(const HCsr& h, DCsr<V>& d);
  void build_stage(const HCsr& h, DCsr<V>& d);
  void qap_apply(const V* xin, V* yout);
  void build_gram(const Prepared& pp, int tpr_mode);  // tpr_mode: A's (pinned when > 0)
  void gram_values();
};

}  // namespace hprqp
