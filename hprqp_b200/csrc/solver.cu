// solver.cu — the HPR control loop and the C ABI of libhprqp.so.
//
// The loop restates solve() (src/algorithm.jl:1904-2039) on the host with
// every vector in HBM: per iteration it only enqueues the fused passes of
// Engine::step(); it synchronises with the device only on the residual
// cadence of the reference (check_iter and the print schedule), reading the
// residual, M-norm and sigma scalars in one copy.  Restart decisions, the
// sigma blend and the scalar golden-section search (src/kernels.jl:1453-1486)
// run on the host from those scalars.
#include <chrono>
#include <ctime>
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <memory>
#include <string>

#include "checkpoint.h"
#include "engine.cuh"

namespace hprqp {

namespace {
const double kInf = std::numeric_limits<double>::infinity();
thread_local std::string g_global_err;

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

double print_step(int64_t iter) {  // src/algorithm.jl:1173-1175
  return std::max(std::pow(10.0, std::floor(std::log10((double)iter))) / 10.0, 10.0);
}
bool on_print_schedule(int64_t iter, const hprqp_params& p) {
  if (p.print_frequency == -1) return std::fmod((double)iter, print_step(iter)) == 0.0;
  return iter % p.print_frequency == 0;
}

// golden (src/kernels.jl:1453-1486)
double golden(double ap, double bp, double cp, double dp, double lo, double hi, double tol, int maxiter = 200) {
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
}  // namespace

void set_global_error(const std::string& msg) { g_global_err = msg; }

struct RestartInfo {  // HPRQP_restart / initialize_restart (src/algorithm.jl:1154-1171)
  bool first_restart = true;
  double save_gap = kInf, current_gap = kInf, last_gap = kInf, best_gap = kInf;
  double best_sigma = 1.0, weighted_norm = kInf;
  int64_t inner = 0, times = 0, sufficient = 0, necessary = 0, long_ = 0;
  int restart_flag = 0;
};

struct Residuals {
  double err_Rp = 0, err_Rd = 0, KKT = kInf, pobj = 0, dobj = 0, gap = 0;
};

struct LoopState {
  int64_t iter = 0;
  RestartInfo ri;
  Residuals res;
  double t0 = 0;
  int64_t iter_4 = 0, iter_6 = 0;
  double time_4 = 0, time_6 = 0;
  bool first_4 = true, first_6 = true;
  PendingMnorm pend_cur, pend_last;
  double polish_tol = 0, best_kkt = kInf;
  int stall = 0;
  bool force_residuals = false;
  int status = -1;
  bool skip_checks_once = false;  // resume: the checkpoint's checks are done, run its step
};

constexpr int kSwitch = -100;

// The best bar iterates so far (ws.saved_state, src/algorithm.jl:97-113),
// kept on the device in FP64 while params.auto_save is set.
struct SavedBest {
  double *x = nullptr, *y = nullptr, *z = nullptr, *w = nullptr;
  int64_t cap_n = 0, cap_m = 0;
  double sigma = 0.0;
  int64_t iter = 0;
  double err_Rp = kInf, err_Rd = kInf, pobj = kInf, dobj = kInf, gap = kInf;
};

// Live per-pass timing: a pool of event sets, one set (npass + 1 marks) per
// recorded plain iteration, harvested after each residual synchronisation.
struct PassProfiler {
  bool on = false;
  int np = 0;
  static constexpr int kSets = 64;
  std::vector<cudaEvent_t> ev;
  int used = 0;  // sets recorded since the last harvest
  double ms[HPRQP_MAX_PASSES] = {0};
  int64_t count = 0;
  void init(int npass) {
    np = npass;
    if (ev.empty()) {
      ev.resize((size_t)kSets * (HPRQP_MAX_PASSES + 1));
      for (auto& e : ev) HPRQP_CUDA(cudaEventCreate(&e));
    }
    used = 0;
    count = 0;
    for (double& v : ms) v = 0;
  }
  ~PassProfiler() {
    for (auto& e : ev) cudaEventDestroy(e);
  }
  // events of the next set, or false when the pool is full
  bool begin(std::vector<cudaEvent_t>& view) {
    if (used >= kSets) return false;
    view.assign(ev.begin() + (size_t)used * (HPRQP_MAX_PASSES + 1),
                ev.begin() + (size_t)used * (HPRQP_MAX_PASSES + 1) + np + 1);
    ++used;
    return true;
  }
  void harvest() {  // call only after a stream synchronisation
    for (int s = 0; s < used; ++s) {
      for (int k = 0; k < np; ++k) {
        float t = 0;
        HPRQP_CUDA(cudaEventElapsedTime(&t, ev[(size_t)s * (HPRQP_MAX_PASSES + 1) + k],
                                        ev[(size_t)s * (HPRQP_MAX_PASSES + 1) + k + 1]));
        ms[k] += t;
      }
      ++count;
    }
    used = 0;
  }
};

static double eval_mnorm(const Common& cm, const PendingMnorm& pm, bool has_m, bool diag, bool verbose) {
  const double* s = cm.h_scal + pm.slot;
  const double sg = pm.sigma;
  double M1 = 0.0, M2 = (1.0 / sg) * s[0], M3 = 0.0;
  M2 -= 2.0 * s[1];
  if (has_m) {
    M1 = sg * pm.lamA * s[8];
    M1 -= 2.0 * sg * s[2];
    M2 += 2.0 * s[3];
    if (diag) {
      M3 = s[4];
      M1 += sg * s[6];
    } else {
      M3 = (sg * sg) / (1.0 + sg * pm.lamQ) * s[5];
      M1 += sg * pm.lamQ * s[7];
    }
  } else if (!diag) {
    M1 = sg * pm.lamQ * s[7];
  }
  M2 += std::max(M1, 0.0);
  const double Mn = std::max(M2, 0.0) + std::max(M3, 0.0);
  if (verbose && std::min(std::min(M1, M2), M3) < -1e-8)
    std::printf("M_1 = %g, M_2 = %g, M_3 = %g, negative M norm due to numerical instability, consider increasing eig_factor\n",
                M1, M2, M3);
  return std::sqrt(Mn);
}

struct Handle {
  int device = 0;
  std::unique_ptr<Common> cm;
  HostProblem hp;
  Prepared pp;
  bool prepared = false;
  int key[5] = {-1, -1, -1, -1, -1};
  int path = PATH_QP;
  std::unique_ptr<Engine<double>> e64;
  std::unique_ptr<Engine<float>> e32;
  std::string err;
  int64_t trace_iters = 0;
  double *xt = nullptr, *yt = nullptr, *wt = nullptr;
  std::string save_file = "hprqp_autosave.ckpt";  // auto-save target (hprqp_set_save_file)
  SavedBest best;
  std::vector<double> init_x, init_y;  // the call's initial points (for the checkpoint's parameters/)
  double* sig_t = nullptr;    // sigma of each traced iteration
  int64_t* inner_t = nullptr; // inner (Halpern) counter of each traced iteration
  double setup_time = 0.0;
  int64_t h2d_at_solve_start = 0;
  PassProfiler prof64, prof32;
  hprqp_pass_stats stats64{}, stats32{};
};

// A fingerprint of the loaded problem's data (FNV-1a over its arrays), so a
// checkpoint is only resumed on the problem it was written for.
static double problem_fingerprint(const HostProblem& hp) {
  uint64_t h = 1469598103934665603ULL;
  auto mix = [&](const void* p, size_t bytes) {
    const unsigned char* b = (const unsigned char*)p;
    for (size_t i = 0; i < bytes; ++i) h = (h ^ b[i]) * 1099511628211ULL;
  };
  auto vec = [&](const auto& v) { mix(v.data(), sizeof(double) * v.size()); };
  auto csr = [&](const HCsr& M) {
    mix(M.ptr.data(), sizeof(int) * M.ptr.size());
    mix(M.col.data(), sizeof(int) * M.col.size());
    vec(M.val);
  };
  mix(&hp.n, 8);
  mix(&hp.m, 8);
  mix(&hp.Q_kind, sizeof(hp.Q_kind));
  vec(hp.c); vec(hp.AL); vec(hp.AU); vec(hp.l); vec(hp.u);
  csr(hp.A); csr(hp.Q); csr(hp.L);
  vec(hp.qA); vec(hp.qB); vec(hp.qS); vec(hp.qT);
  return (double)(h >> 11);  // exact in a double
}

static const char* problem_type_name(int t) { return t == HPRQP_PROBLEM_LASSO ? "LASSO" : t == HPRQP_PROBLEM_QAP ? "QAP" : "QP"; }

// save_state_to_hdf5! (src/algorithm.jl:183-301): the current and the best
// bar iterates unscaled as collect_results! does, their residuals, sigma and
// the parameters, under the reference's dataset names (the z of the file
// keeps the reference's c_scale * z_bar / col_norm, unlike collect_results!,
// src/algorithm.jl:213 against :640), plus the resume/ section: the scaled
// state the next step reads (x, w, y, A'y and the Halpern anchors; Qw on the
// QP-noC path), sigma, the lambda_max values and the restart and loop
// records.  A failed write warns (verbose) and the solve goes on, as in the
// reference.
template <typename V>
static void save_checkpoint(Handle& H, Engine<V>& E, const hprqp_params& p, const LoopState& L, int status,
                            bool fp32_phase) {
  const int64_t n = E.n, m = E.m;
  const double bs = E.b_scale, cs = E.c_scale;
  std::vector<double> cn(n), rn(m), xb(n), zb(n), wb(n), yb(m), v(std::max(n, m));
  E.vec_to_host(E.col_norm, n, cn.data());
  if (m > 0) E.vec_to_host(E.row_norm, m, rn.data());
  E.vec_to_host(E.x_bar, n, xb.data());
  E.vec_to_host(E.z_bar, n, zb.data());
  E.vec_to_host(E.w_bar, n, wb.data());
  if (m > 0) E.vec_to_host(E.y_bar, m, yb.data());
  ck::Writer w;
  auto org = [&](const std::string& name, const std::vector<double>& s, const std::vector<double>& nrm, double sc,
                 int64_t len) {
    for (int64_t i = 0; i < len; ++i) v[i] = sc * (s[i] / nrm[i]);
    w.f64(name, v.data(), len);
  };
  char stamp[32];
  const std::time_t now = std::time(nullptr);
  std::strftime(stamp, sizeof(stamp), "%Y-%m-%dT%H:%M:%S", std::localtime(&now));
  w.i64("current/iteration", L.iter);
  w.f64("current/time_elapsed", now_s() - L.t0);
  w.str("current/timestamp", stamp);
  org("current/x_org", xb, cn, bs, n);
  org("current/w_org", wb, cn, bs, n);
  if (m > 0) org("current/y_org", yb, rn, cs, m);
  org("current/z_org", zb, cn, cs, n);
  w.f64("current/sigma", E.sigma);
  w.f64("current/err_Rp", L.res.err_Rp);
  w.f64("current/err_Rd", L.res.err_Rd);
  w.f64("current/primal_obj", L.res.pobj);
  w.f64("current/dual_obj", L.res.dobj);
  w.f64("current/rel_gap", L.res.gap);
  w.f64("current/KKTx_and_gap", L.res.KKT);
  const SavedBest& B = H.best;
  auto down = [&](const double* d, int64_t len, std::vector<double>& h) {
    if (len > 0) HPRQP_CUDA(cudaMemcpyAsync(h.data(), d, sizeof(double) * len, cudaMemcpyDeviceToHost, H.cm->stream));
  };
  down(B.x, n, xb);
  down(B.z, n, zb);
  down(B.w, n, wb);
  if (m > 0) down(B.y, m, yb);
  HPRQP_CUDA(cudaStreamSynchronize(H.cm->stream));
  H.cm->d2h += (int64_t)sizeof(double) * (3 * n + m);
  org("best/x_org", xb, cn, bs, n);
  org("best/w_org", wb, cn, bs, n);
  if (m > 0) org("best/y_org", yb, rn, cs, m);
  org("best/z_org", zb, cn, cs, n);
  w.f64("best/sigma", B.sigma);
  w.i64("best/iteration", B.iter);
  w.f64("best/err_Rp", B.err_Rp);
  w.f64("best/err_Rd", B.err_Rd);
  w.f64("best/primal_obj", B.pobj);
  w.f64("best/dual_obj", B.dobj);
  w.f64("best/rel_gap", B.gap);
  w.f64("best/KKTx_and_gap", std::max(std::max(B.err_Rp, B.err_Rd), B.gap));
  w.f64("parameters/stoptol", p.stoptol);
  w.f64("parameters/sigma", p.sigma);
  w.i64("parameters/max_iter", p.max_iter);
  w.i64("parameters/sigma_fixed", p.sigma_fixed);
  w.f64("parameters/time_limit", p.time_limit);
  w.f64("parameters/eig_factor", p.eig_factor);
  w.i64("parameters/check_iter", p.check_iter);
  w.i64("parameters/warm_up", p.warm_up);
  w.i64("parameters/spmv_mode_Q", p.spmv_mode_Q);
  w.i64("parameters/spmv_mode_A", p.spmv_mode_A);
  w.i64("parameters/print_frequency", p.print_frequency);
  w.i64("parameters/device_number", p.device_number);
  w.i64("parameters/use_Ruiz_scaling", p.use_Ruiz_scaling);
  w.i64("parameters/use_bc_scaling", p.use_bc_scaling);
  w.i64("parameters/use_l2_scaling", p.use_l2_scaling);
  w.i64("parameters/use_Pock_Chambolle_scaling", p.use_Pock_Chambolle_scaling);
  w.str("parameters/problem_type", problem_type_name(p.problem_type));
  w.f64("parameters/lambda", p.lambda);
  w.i64("parameters/auto_save", p.auto_save);
  w.i64("parameters/precision", p.precision);
  if (!H.init_x.empty()) w.f64("parameters/initial_x", H.init_x.data(), (int64_t)H.init_x.size());
  if (!H.init_y.empty()) w.f64("parameters/initial_y", H.init_y.data(), (int64_t)H.init_y.size());
  // resume/: the scaled state of the engine's storage type, exactly
  w.f64("resume/fingerprint", problem_fingerprint(H.hp));
  w.i64("resume/n", n);
  w.i64("resume/m", m);
  w.i64("resume/phase", fp32_phase ? 32 : 64);
  w.i64("resume/status", status);
  w.i64("resume/iter", L.iter);
  w.f64("resume/sigma", E.sigma);
  w.f64("resume/lambda_max_A", E.lamA);
  w.f64("resume/lambda_max_Q", E.lamQ);
  const RestartInfo& r = L.ri;
  const double rinfo[14] = {r.first_restart ? 1.0 : 0.0, r.save_gap, r.current_gap, r.last_gap, r.best_gap,
                            r.best_sigma, r.weighted_norm, (double)r.inner, (double)r.times, (double)r.sufficient,
                            (double)r.necessary, (double)r.long_, (double)r.restart_flag, 0.0};
  w.f64("resume/restart", rinfo, 14);
  const double loop[16] = {L.res.err_Rp, L.res.err_Rd, L.res.KKT, L.res.pobj, L.res.dobj, L.res.gap,
                           (double)L.iter_4, (double)L.iter_6, L.time_4, L.time_6, L.first_4 ? 1.0 : 0.0,
                           L.first_6 ? 1.0 : 0.0, L.best_kkt, (double)L.stall, L.polish_tol, 0.0};
  w.f64("resume/loop", loop, 16);
  auto st = [&](const char* name, const V* d, int64_t len) {
    if (len <= 0 || !d) return;
    E.vec_to_host(d, len, v.data());
    w.f64(std::string("resume/") + name, v.data(), len);
  };
  st("x", E.x, n);
  st("w", E.w, n);
  st("ATy", E.ATy, n);
  st("last_x", E.last_x, n);
  st("last_w", E.last_w, n);
  st("last_ATy", E.last_ATy, n);
  st("Qw", E.Qw, n);
  st("last_Qw", E.last_Qw, n);
  st("y", E.y, m);
  st("last_y", E.last_y, m);
  std::string err;
  if (!w.write(H.save_file, err)) {
    if (p.verbose) std::printf("Warning: Failed to save the checkpoint: %s\n", err.c_str());
  } else if (p.verbose) {
    std::printf("State saved to %s at iteration %lld\n", H.save_file.c_str(), (long long)L.iter);
  }
}

// One phase of the HPR loop on engine E (src/algorithm.jl:1977-2038).
// Returns a final status, or kSwitch when the FP32 phase hands over.
template <typename V>
static int run_loop(Handle& H, Engine<V>& E, const hprqp_params& p, LoopState& L, bool fp32_phase) {
  Common& cm = *H.cm;
  const int64_t n = E.n, m = E.m;
  const int64_t check_iter = p.check_iter;
  RestartInfo& ri = L.ri;
  PassProfiler& prof = sizeof(V) == 8 ? H.prof64 : H.prof32;
  std::vector<cudaEvent_t> prof_view;
  prof.on = p.profile_passes != 0;
  if (prof.on) prof.init(E.npasses());
  for (; L.iter <= p.max_iter; ++L.iter) {
    const int64_t iter = L.iter;
    const bool time_up = now_s() - L.t0 > p.time_limit;
    const bool print_yes = on_print_schedule(iter, p) || iter == p.max_iter || time_up;
    // a resumed solve enters at its checkpoint's step: the checks of that
    // iteration ran before the checkpoint was written
    const bool checks = !L.skip_checks_once;
    L.skip_checks_once = false;
    if (checks) {
    if (iter % check_iter == 0 || print_yes || L.force_residuals) {
      L.force_residuals = false;
      E.residuals_launch(iter == 0);
      cm.sync_read(0, S_GOLD);
      if (prof.on) prof.harvest();
      if (L.pend_cur.active) {
        ri.current_gap = eval_mnorm(cm, L.pend_cur, m > 0, E.Q_is_diag, p.verbose);
        L.pend_cur.active = false;
      }
      if (L.pend_last.active) {
        ri.last_gap = eval_mnorm(cm, L.pend_last, m > 0, E.Q_is_diag, p.verbose);
        L.pend_last.active = false;
      }
      // compute_residuals! (src/algorithm.jl:37-115) from the reduced slots
      const double* r = cm.h_scal;
      const double bc = E.b_scale * E.c_scale;
      Residuals& R = L.res;
      R.pobj = bc * (r[S_RES_N + 0] + 0.5 * r[S_RES_N + 1]) + H.hp.obj_constant;
      R.dobj = bc * (-0.5 * r[S_RES_N + 1] + r[S_RES_N + 2]) + H.hp.obj_constant;
      if (m > 0) R.dobj += bc * r[S_RES_M + 0];
      if (p.problem_type == HPRQP_PROBLEM_LASSO && n > 0) {
        R.pobj += bc * r[S_RES_N + 3];
        R.dobj += bc * r[S_RES_N + 3];
      }
      R.gap = std::fabs(R.pobj - R.dobj) / (1.0 + std::max(std::fabs(R.pobj), std::fabs(R.dobj)));
      R.err_Rd = r[S_RES_N + 4] / (1.0 + std::max(std::max(E.norm_c_org, r[S_RES_N + 5]), r[S_RES_N + 6]));
      R.err_Rp = m > 0 ? r[S_RES_M + 1] / (1.0 + std::max(E.norm_b_org, r[S_RES_M + 2])) : 0.0;
      if (iter == 0) R.err_Rp = std::max(R.err_Rp, r[S_RES_N + 7]);
      R.KKT = std::max(std::max(R.err_Rp, R.err_Rd), R.gap);
      if (!std::isfinite(R.KKT) || !std::isfinite(R.pobj) || !std::isfinite(R.dobj)) return HPRQP_STATUS_NUMERICAL_ERROR;
      // the best iterates so far (compute_residuals!, src/algorithm.jl:97-113)
      SavedBest& B = H.best;
      if (p.auto_save && (iter == 0 || R.KKT < std::max(std::max(B.err_Rp, B.err_Rd), B.gap))) {
        E.bars_to_device(B.x, B.y, B.z, B.w);
        B.sigma = E.sigma;
        B.iter = iter;
        B.err_Rp = R.err_Rp;
        B.err_Rd = R.err_Rd;
        B.pobj = R.pobj;
        B.dobj = R.dobj;
        B.gap = R.gap;
      }
      if (fp32_phase) {
        if (R.KKT < L.polish_tol) return kSwitch;
        if (R.KKT < 0.9 * L.best_kkt) {
          L.best_kkt = R.KKT;
          L.stall = 0;
        } else if (++L.stall >= 50 && iter >= 1000) {
          return kSwitch;
        }
      }
    }
    // check_break (src/algorithm.jl:558-576)
    int status = -1;
    if (L.res.KKT < p.stoptol) status = HPRQP_STATUS_OPTIMAL;
    else if (iter == p.max_iter) status = HPRQP_STATUS_MAX_ITER;
    else if (now_s() - L.t0 > p.time_limit) status = HPRQP_STATUS_TIME_LIMIT;
    // check_restart (src/algorithm.jl:441-492)
    ri.restart_flag = 0;
    if (ri.first_restart) {
      if (iter == check_iter) {
        ri.first_restart = false;
        ri.restart_flag = 1;
        ri.weighted_norm = ri.current_gap;
        ri.best_gap = ri.current_gap;
        ri.best_sigma = E.sigma;
      }
    } else if (iter % check_iter == 0) {
      if (ri.current_gap < 0) {
        ri.current_gap = 1e-6;
        if (p.verbose) std::printf("current_gap < 0\n");
      }
      if (ri.current_gap <= 0.2 * ri.last_gap) { ri.sufficient++; ri.restart_flag = 1; }
      if (ri.current_gap <= 0.8 * ri.last_gap && ri.current_gap > 1.00 * ri.save_gap) {
        ri.necessary++;
        ri.restart_flag = 2;
      }
      const double fact = (ri.current_gap / ri.weighted_norm > 1e-1) ? 0.5 : 0.2;
      if (ri.inner >= fact * iter) { ri.long_++; ri.restart_flag = 3; }
      if (ri.best_gap > ri.current_gap) { ri.best_gap = ri.current_gap; ri.best_sigma = E.sigma; }
      ri.save_gap = ri.current_gap;
    }
    // update_sigma! (src/algorithm.jl:323-423)
    if (!p.sigma_fixed && ri.restart_flag >= 1) {
      const double sigma_old = E.sigma;
      E.sigma_stats_launch();
      cm.sync_read(S_SIG, 6);
      const double* s = cm.h_scal + S_SIG;
      double a = 0.0, b = s[0], c = 0.0, d = 0.0;
      if (m > 0) a = E.lamA * s[5] - 2 * s[1];
      if (E.Q_is_diag) {
        const double nq = std::sqrt(s[2]);
        a += nq * nq;
      } else {
        a += E.lamQ * s[3];
        if (m > 0) { c = s[4]; d = E.lamQ; }
      }
      a = std::max(a, 1e-12);
      b = std::max(b, 1e-12);
      double est;
      if (E.Q_is_diag) {
        if (m > 0) {
          E.golden_diag_launch(a, b);
          cm.sync_read(S_GOLD, 1);
          est = cm.h_scal[S_GOLD];
        } else {
          est = std::sqrt(b / a);
        }
      } else {
        est = m > 0 ? golden(a, b, c, d, 1e-12, 1e12, 1e-13) : std::sqrt(b / a);
      }
      const double fct = std::exp(-0.05 * (ri.current_gap / ri.best_gap));
      const double temp1 = std::max(std::min(L.res.err_Rd, L.res.err_Rp), std::min(L.res.gap, ri.current_gap));
      const double cand = std::exp(fct * std::log(est) + (1 - fct) * std::log(ri.best_sigma));
      double kappa;
      if (temp1 > 9e-10) kappa = 1.0;
      else if (temp1 > 5e-10) kappa = std::min(std::max(std::sqrt(L.res.err_Rd / L.res.err_Rp), 1e-2), 100.0);
      else kappa = std::min(std::max(L.res.err_Rd / L.res.err_Rp, 1e-2), 100.0);
      const double sigma_new = kappa * cand;
      if (E.Q_is_diag && std::fabs(sigma_old - sigma_new) > 1e-15) E.set_sigma(sigma_new);
      else E.sigma = sigma_new;
    }
    // do_restart! (src/algorithm.jl:522-555)
    if (ri.restart_flag > 0) {
      E.restart();
      ri.last_gap = ri.current_gap;
      ri.save_gap = kInf;
      ri.times++;
      ri.inner = 0;
    }
    if ((print_yes || status >= 0) && p.verbose)
      std::printf("%5lld    %3.2e    %3.2e    %+7.6e    %+7.6e    %3.2e    %3.2e    %6.2f\n", (long long)iter,
                  L.res.err_Rp, L.res.err_Rd, L.res.pobj, L.res.dobj, L.res.gap, E.sigma, now_s() - L.t0);
    if (L.res.KKT < 1e-4 && L.first_4) { L.time_4 = now_s() - L.t0; L.iter_4 = iter; L.first_4 = false; }
    if ((print_yes || status >= 0) && p.auto_save) save_checkpoint(H, E, p, L, status, fp32_phase);
    if (L.res.KKT < 1e-4 && L.first_4) { L.time_4 = now_s() - L.t0; L.iter_4 = iter; L.first_4 = false; }
    if (L.res.KKT < 1e-6 && L.first_6) { L.time_6 = now_s() - L.t0; L.iter_6 = iter; L.first_6 = false; }
    if (status >= 0) return status;
    }  // checks
    const int64_t next = iter + 1;
    const bool to_check = (next % check_iter == 0) || (ri.restart_flag > 0) || on_print_schedule(next, p);
    // perform_iteration_step! (src/algorithm.jl:1881-1900)
    const double h1 = 1.0 / (ri.inner + 2.0), h2 = 1.0 - h1;
    const int64_t inner_used = ri.inner;
    if (prof.on && !to_check && prof.begin(prof_view)) {
      E.prof = &prof_view;
      E.prof_k = 0;
    }
    E.step(to_check, h1, h2);
    E.prof = nullptr;
    if (ri.restart_flag > 0) {
      E.mnorm_launch(S_MN_LAST);
      L.pend_last = PendingMnorm{true, S_MN_LAST, E.sigma, E.lamA, E.lamQ};
    }
    if ((iter + 1) % check_iter == 0) {
      E.mnorm_launch(S_MN_CUR);
      L.pend_cur = PendingMnorm{true, S_MN_CUR, E.sigma, E.lamA, E.lamQ};
    }
    ri.inner++;
    if (next <= H.trace_iters) {
      E.trace_copy(H.xt ? H.xt + (next - 1) * n : nullptr, H.yt ? H.yt + (next - 1) * m : nullptr,
                   H.wt ? H.wt + (next - 1) * n : nullptr);
      if (H.sig_t) H.sig_t[next - 1] = E.sigma;
      if (H.inner_t) H.inner_t[next - 1] = inner_used;
    }
  }
  return HPRQP_STATUS_MAX_ITER;
}

static void check_params(const hprqp_params& p) {
  if (!(p.stoptol > 0)) throw Error(HPRQP_E_ARG, "stoptol must be positive");
  if (p.check_iter <= 0) throw Error(HPRQP_E_ARG, "check_iter must be positive");
  if (p.max_iter < 0) throw Error(HPRQP_E_ARG, "max_iter must be >= 0");
  if (!(p.sigma == -1 || p.sigma > 0))
    throw Error(HPRQP_E_ARG, "Invalid sigma value. It should be a positive number or -1 for automatic.");
  if (!(p.print_frequency == -1 || p.print_frequency > 0))
    throw Error(HPRQP_E_ARG, "Invalid print_frequency. It should be a positive integer or -1 for automatic printing.");
  if (!p.use_gpu) throw Error(HPRQP_E_UNSUPPORTED, "use_gpu = false: libhprqp has no CPU path");
  if (p.precision != HPRQP_PRECISION_FP64 && p.precision != HPRQP_PRECISION_FP32_POLISH)
    throw Error(HPRQP_E_ARG, "unknown precision mode");
  if (p.spmv_mode_Q < 0 || p.spmv_mode_Q > 10 || p.spmv_mode_A < 0 || p.spmv_mode_A > 10)
    throw Error(HPRQP_E_ARG, "spmv_mode must be 0 (auto), 1..6 (CSR, 1..32 threads per row), 7 (SELL-32), 8 (ELL), "
                             "9 (row split) or 10 (staged column blocks)");
}

static void prepare(Handle& H, const hprqp_params& p) {
  if (!H.hp.loaded) throw Error(HPRQP_E_STATE, "no problem loaded");
  check_params(p);
  const int key[5] = {p.use_Ruiz_scaling, p.use_Pock_Chambolle_scaling, 0, p.spmv_mode_Q, p.spmv_mode_A};
  if (H.prepared && std::memcmp(key, H.key, sizeof(key)) == 0) {
    // same scaling and schedule: only add the FP32 engine if it is missing
    if (p.precision == HPRQP_PRECISION_FP32_POLISH && !H.e32)
      H.e32 = std::make_unique<Engine<float>>(*H.cm, H.hp, H.pp, H.path, p.spmv_mode_Q, p.spmv_mode_A, true);
    return;
  }
  const double t = now_s();
  H.e64.reset();
  H.e32.reset();
  // scaling on the GPU for large sparse problems (bitwise the host result);
  // HPRQP_HOST_SCALING=1 keeps it on the host
  const char* hs = std::getenv("HPRQP_HOST_SCALING");
  const int64_t work = H.hp.A.nnz() + H.hp.Q.nnz();
  if (H.hp.Q_kind == HPRQP_Q_SPARSE && work >= 100000 && !(hs && hs[0] == '1'))
    prepare_problem_gpu(H.hp, p, H.pp, H.cm->stream, &H.cm->h2d, &H.cm->d2h);
  else
    prepare_problem(H.hp, p, H.pp);
  if (H.hp.Q_kind == HPRQP_Q_LASSO) H.path = PATH_LASSO;
  else if (H.hp.Q_kind == HPRQP_Q_QAP || H.hp.Q_kind == HPRQP_Q_CUSTOM || H.pp.Qpat().nnz() > 0)
    H.path = H.pp.noC ? PATH_NOC : PATH_QP;
  else H.path = PATH_LP;
  // the power method runs on the first phase's engine: only that one builds
  // the Gram matrix of the A A' chain
  const bool fp32 = p.precision == HPRQP_PRECISION_FP32_POLISH;
  const double t_scaled = now_s();
  H.e64 = std::make_unique<Engine<double>>(*H.cm, H.hp, H.pp, H.path, p.spmv_mode_Q, p.spmv_mode_A, !fp32);
  const double t_e64 = now_s();
  if (fp32)
    H.e32 = std::make_unique<Engine<float>>(*H.cm, H.hp, H.pp, H.path, p.spmv_mode_Q, p.spmv_mode_A, true);
  std::memcpy(H.key, key, sizeof(key));
  H.prepared = true;
  H.setup_time = now_s() - t;
  if (const char* tv = std::getenv("HPRQP_TIMING"))
    if (tv[0] == '1')
      std::fprintf(stderr, "[hprqp] setup: scaling %.3f s, FP64 engine %.3f s, FP32 engine %.3f s\n", t_scaled - t,
                   t_e64 - t_scaled, now_s() - t_e64);
}

// estimate_eigenvalues + compute_lambda_max_Q (src/algorithm.jl:1407-1440,
// src/unified_operations.jl:703-718): the power methods for A A' and Q run
// together, in the precision of the first phase (their 1e-4 stopping test is
// far above FP32 rounding).
static void estimate_lambdas(Handle& H, const hprqp_params& p, bool fp32, double* lamA, double* lamQ,
                             int64_t* itA_out = nullptr, int64_t* itQ_out = nullptr, double* bytes_out = nullptr) {
  const Prepared& pp = H.pp;
  const bool needA = H.hp.m > 0 && !(p.lambda_max_A_override > 0);
  const bool opQ = H.hp.Q_kind != HPRQP_Q_SPARSE || (pp.Qpat().nnz() > 0 && !pp.Q_is_diag);
  const bool needQ = opQ && !(p.lambda_max_Q_override > 0);
  double a = 0.0, q = 0.0;
  int64_t ia = 0, iq = 0;
  if (needA || needQ) {
    if (fp32) {
      H.e32->power_setup(pp, p.spmv_mode_A, p.spmv_mode_Q);
      H.e32->power_both(needA, needQ, 1e-4, 5000, &a, &q, &ia, &iq);
    } else {
      H.e64->power_setup(pp, p.spmv_mode_A, p.spmv_mode_Q);
      H.e64->power_both(needA, needQ, 1e-4, 5000, &a, &q, &ia, &iq);
    }
  }
  if (!needA) ia = 0;
  if (!needQ) iq = 0;
  if (itA_out) *itA_out = ia;
  if (itQ_out) *itQ_out = iq;
  if (bytes_out) {
    if (fp32) *bytes_out = ia * H.e32->power_step_bytes(0) + iq * H.e32->power_step_bytes(1);
    else *bytes_out = ia * H.e64->power_step_bytes(0) + iq * H.e64->power_step_bytes(1);
  }
  *lamA = H.hp.m > 0 ? (needA ? a * p.eig_factor : p.lambda_max_A_override) : 0.0;
  if (opQ) *lamQ = needQ ? q * p.eig_factor : p.lambda_max_Q_override;
  else *lamQ = pp.Qpat().nnz() > 0 ? pp.Q_maxval : 0.0;
}

template <typename V>
static void start_engine(Handle& H, Engine<V>& E, const hprqp_params& p, double lamA, double lamQ, double sigma0,
                         const double* x0, const double* y0) {
  E.reset_state();
  E.lamA = lamA;
  E.lamQ = lamQ;
  E.lam_l1 = p.problem_type == HPRQP_PROBLEM_LASSO ? H.hp.lambda : 0.0;
  E.sigma = sigma0;
  E.initial_points(x0, y0);
  if (E.Q_is_diag) E.set_sigma(sigma0);
}

// Continue from a checkpoint: the engine's state, sigma, lambda_max and the
// loop records as the checkpoint holds them; the loop then enters at the
// checkpoint's step (LoopState::skip_checks_once).
template <typename V>
static void resume_engine(Handle& H, Engine<V>& E, const hprqp_params& p, const ck::Reader& rs, LoopState& L) {
  auto f1 = [&](const char* name) { return rs.get(name)->f[0]; };
  E.reset_state();
  E.lamA = f1("resume/lambda_max_A");
  E.lamQ = f1("resume/lambda_max_Q");
  E.lam_l1 = p.problem_type == HPRQP_PROBLEM_LASSO ? H.hp.lambda : 0.0;
  E.sigma = f1("resume/sigma");
  auto put = [&](const char* name, V* d, int64_t len) {
    const ck::Record* r = rs.get(std::string("resume/") + name);
    if (len <= 0 || !d) return;
    if (!r || (int64_t)r->f.size() != len) throw Error(HPRQP_E_ARG, std::string("checkpoint lacks resume/") + name);
    E.vec_from_host(d, r->f.data(), len);
  };
  const int64_t n = E.n, m = E.m;
  put("x", E.x, n);
  put("w", E.w, n);
  put("ATy", E.ATy, n);
  put("last_x", E.last_x, n);
  put("last_w", E.last_w, n);
  put("last_ATy", E.last_ATy, n);
  put("Qw", E.Qw, n);
  put("last_Qw", E.last_Qw, n);
  put("y", E.y, m);
  put("last_y", E.last_y, m);
  if (E.Q_is_diag) E.set_sigma(E.sigma);
  const std::vector<double>& r = rs.get("resume/restart")->f;
  RestartInfo& ri = L.ri;
  ri.first_restart = r[0] != 0.0;
  ri.save_gap = r[1];
  ri.current_gap = r[2];
  ri.last_gap = r[3];
  ri.best_gap = r[4];
  ri.best_sigma = r[5];
  ri.weighted_norm = r[6];
  ri.inner = (int64_t)r[7];
  ri.times = (int64_t)r[8];
  ri.sufficient = (int64_t)r[9];
  ri.necessary = (int64_t)r[10];
  ri.long_ = (int64_t)r[11];
  ri.restart_flag = (int)r[12];
  const std::vector<double>& q = rs.get("resume/loop")->f;
  L.res.err_Rp = q[0];
  L.res.err_Rd = q[1];
  L.res.KKT = q[2];
  L.res.pobj = q[3];
  L.res.dobj = q[4];
  L.res.gap = q[5];
  L.iter_4 = (int64_t)q[6];
  L.iter_6 = (int64_t)q[7];
  L.time_4 = q[8];
  L.time_6 = q[9];
  L.first_4 = q[10] != 0.0;
  L.first_6 = q[11] != 0.0;
  L.best_kkt = q[12];
  L.stall = (int)q[13];
  L.iter = rs.get("resume/iter")->i[0];
  L.skip_checks_once = true;
}

// The checkpoint must belong to the loaded problem and the parameters that
// shape the scaled state; it must be of a solve that stopped early.
static void check_resume(const Handle& H, const hprqp_params& p, const ck::Reader& rs) {
  static const char* need_f[] = {"resume/fingerprint", "resume/sigma", "resume/lambda_max_A", "resume/lambda_max_Q",
                                 "resume/restart", "resume/loop"};
  static const char* need_i[] = {"resume/n", "resume/m", "resume/phase", "resume/status", "resume/iter",
                                 "parameters/use_Ruiz_scaling", "parameters/use_Pock_Chambolle_scaling"};
  for (const char* k : need_f)
    if (!rs.get(k) || rs.get(k)->f.empty()) throw Error(HPRQP_E_ARG, std::string("checkpoint lacks ") + k);
  for (const char* k : need_i)
    if (!rs.get(k) || rs.get(k)->i.empty()) throw Error(HPRQP_E_ARG, std::string("checkpoint lacks ") + k);
  if (rs.get("resume/restart")->f.size() < 13 || rs.get("resume/loop")->f.size() < 14)
    throw Error(HPRQP_E_ARG, "checkpoint: short restart or loop record");
  if (rs.get("resume/n")->i[0] != H.hp.n || rs.get("resume/m")->i[0] != H.hp.m ||
      rs.get("resume/fingerprint")->f[0] != problem_fingerprint(H.hp))
    throw Error(HPRQP_E_ARG, "checkpoint is of another problem than the loaded one");
  if (rs.get("parameters/use_Ruiz_scaling")->i[0] != p.use_Ruiz_scaling ||
      rs.get("parameters/use_Pock_Chambolle_scaling")->i[0] != p.use_Pock_Chambolle_scaling)
    throw Error(HPRQP_E_ARG, "checkpoint was written with other scaling parameters");
  const int64_t st = rs.get("resume/status")->i[0];
  if (st == HPRQP_STATUS_OPTIMAL || st == HPRQP_STATUS_NUMERICAL_ERROR)
    throw Error(HPRQP_E_ARG, "checkpoint is of a finished solve (status " + std::to_string(st) + ")");
  if (rs.get("resume/phase")->i[0] == 32 && p.precision != HPRQP_PRECISION_FP32_POLISH)
    throw Error(HPRQP_E_ARG, "checkpoint is of the FP32 phase: resume it with precision FP32_POLISH");
}

static int solve(Handle& H, const hprqp_params& p, const double* x0, const double* y0, hprqp_result* res,
                 double* xo, double* yo, double* zo, double* wo, const ck::Reader* rs = nullptr) {
  const double setup_start = now_s();
  // host<->device bytes of this call, set-up (scaling, uploads) included
  H.h2d_at_solve_start = H.cm->h2d;
  const int64_t d2h0 = H.cm->d2h;
  prepare(H, p);
  if (rs) check_resume(H, p, *rs);
  const double setup_time = now_s() - setup_start;
  Common& cm = *H.cm;
  const int64_t launches0 = cm.launches;
  if (p.auto_save) {  // the best-iterate copies (FP64, on the device)
    SavedBest& B = H.best;
    if (B.cap_n < H.hp.n || B.cap_m < H.hp.m) {
      B.x = cm.mem.alloc<double>(H.hp.n);
      B.z = cm.mem.alloc<double>(H.hp.n);
      B.w = cm.mem.alloc<double>(H.hp.n);
      B.y = cm.mem.alloc<double>(std::max<int64_t>(H.hp.m, 1));
      B.cap_n = H.hp.n;
      B.cap_m = H.hp.m;
    }
    B.sigma = 0.0;
    B.iter = 0;
    B.err_Rp = B.err_Rd = B.pobj = B.dobj = B.gap = kInf;
    H.init_x.assign(x0 ? x0 : nullptr, x0 ? x0 + H.hp.n : nullptr);
    H.init_y.assign(y0 ? y0 : nullptr, y0 ? y0 + H.hp.m : nullptr);
  }
  const Prepared& pp = H.pp;
  const int64_t m = H.hp.m;
  Engine<double>& E64 = *H.e64;
  cudaEvent_t ev0, ev1;
  HPRQP_CUDA(cudaEventCreate(&ev0));
  HPRQP_CUDA(cudaEventCreate(&ev1));
  HPRQP_CUDA(cudaEventRecord(ev0, cm.stream));
  LoopState L;
  L.t0 = now_s();
  // estimate_eigenvalues (src/algorithm.jl:1407-1440)
  double lamA = 0.0, lamQ = 0.0;
  int64_t pit = 0;
  // The power method runs in the precision of the first phase: its 1e-4
  // stopping test is far above FP32 rounding.
  const bool fp32 = p.precision == HPRQP_PRECISION_FP32_POLISH;
  int64_t pitA = 0, pitQ = 0;
  double pbytes = 0.0;
  if (rs) {  // the checkpoint's lambda_max values
    lamA = rs->get("resume/lambda_max_A")->f[0];
    lamQ = rs->get("resume/lambda_max_Q")->f[0];
  } else {
    estimate_lambdas(H, p, fp32, &lamA, &lamQ, &pitA, &pitQ, &pbytes);
  }
  const double power_time = now_s() - L.t0;
  // sigma of allocate_workspace (src/algorithm.jl:838-851)
  double sigma0 = p.sigma > 0 ? p.sigma : 1.0;
  if (p.sigma == -1)
    sigma0 = (pp.norm_c > 1e-16 && pp.norm_b > 1e-16 && pp.norm_b < 1e16 && pp.norm_c < 1e16) ? pp.norm_b / pp.norm_c : 1.0;
  L.ri.best_sigma = sigma0;
  L.polish_tol = p.polish_tol > 0 ? p.polish_tol : 10.0 * p.stoptol;
  int status;
  int64_t iter_fp32 = 0;
  bool final64 = true;
  if (rs && rs->get("resume/phase")->i[0] == 64) {  // resumed in the FP64 phase (plain FP64 or the polish)
    resume_engine(H, E64, p, *rs, L);
    status = run_loop(H, E64, p, L, false);
  } else if (p.precision == HPRQP_PRECISION_FP32_POLISH) {
    Engine<float>& E32 = *H.e32;
    if (rs) resume_engine(H, E32, p, *rs, L);
    else start_engine(H, E32, p, lamA, lamQ, sigma0, x0, y0);
    status = run_loop(H, E32, p, L, true);
    iter_fp32 = L.iter;
    if (status == kSwitch) {
      E64.import_state(E32);
      L.force_residuals = true;
      status = run_loop(H, E64, p, L, false);
    } else {
      final64 = false;
    }
  } else {
    start_engine(H, E64, p, lamA, lamQ, sigma0, x0, y0);
    status = run_loop(H, E64, p, L, false);
  }
  // handle_termination + collect_results! (src/algorithm.jl:1039-1097, 611-643)
  HPRQP_CUDA(cudaEventRecord(ev1, cm.stream));
  HPRQP_CUDA(cudaEventSynchronize(ev1));
  float dev_ms = 0.0f;
  HPRQP_CUDA(cudaEventElapsedTime(&dev_ms, ev0, ev1));
  cudaEventDestroy(ev0);
  cudaEventDestroy(ev1);
  auto fill = [&](auto& E, PassProfiler& pr, hprqp_pass_stats& st) {
    std::memset(&st, 0, sizeof(st));
    if (!p.profile_passes || pr.count == 0) return;
    pr.harvest();
    st.npass = pr.np;
    st.path = E.path;
    st.iters = pr.count;
    for (int k = 0; k < pr.np; ++k) {
      const char* name;
      double bytes;
      int tpr;
      E.pass_info(k, &name, &bytes, &tpr);
      std::snprintf(st.name[k], sizeof(st.name[k]), "%s", name);
      st.ms_per_launch[k] = pr.ms[k] / (double)pr.count;
      st.bytes_per_launch[k] = bytes;
      st.threads_per_row[k] = tpr;
      st.ms_per_iter += st.ms_per_launch[k];
      st.bytes_per_iter += bytes;
    }
  };
  fill(E64, H.prof64, H.stats64);
  if (H.e32) fill(*H.e32, H.prof32, H.stats32);
  else std::memset(&H.stats32, 0, sizeof(H.stats32));
  if (final64) E64.collect(xo, yo, zo, wo);
  else H.e32->collect(xo, yo, zo, wo);
  const double t_end = now_s() - L.t0;
  std::memset(res, 0, sizeof(*res));
  res->iter = L.iter;
  res->time = t_end;
  res->power_time = power_time;
  res->setup_time = setup_time > 0 ? std::max(setup_time, 0.0) : 0.0;
  if (setup_time < 1e-9) res->setup_time = 0.0;
  res->primal_obj = L.res.pobj;
  res->dual_obj = L.res.dobj;
  res->residuals = L.res.KKT;
  res->gap = L.res.gap;
  res->err_Rp = L.res.err_Rp;
  res->err_Rd = L.res.err_Rd;
  res->status = status;
  res->Q_is_diag = pp.Q_is_diag;
  res->sigma = final64 ? E64.sigma : H.e32->sigma;
  res->lambda_max_A = lamA;
  res->lambda_max_Q = lamQ;
  res->restarts = L.ri.times;
  res->time_4 = L.time_4 == 0.0 ? t_end : L.time_4;
  res->iter_4 = L.iter_4 == 0 ? L.iter : L.iter_4;
  res->time_6 = L.time_6 == 0.0 ? t_end : L.time_6;
  res->iter_6 = L.iter_6 == 0 ? L.iter : L.iter_6;
  res->iter_fp32 = iter_fp32;
  res->gpu_launches = cm.launches - launches0;
  res->device_time = dev_ms * 1e-3;
  res->power_iter_A = pitA;
  res->power_iter_Q = pitQ;
  res->power_bytes = pbytes;
  res->h2d_bytes = cm.h2d - H.h2d_at_solve_start;
  res->d2h_bytes = cm.d2h - d2h0;
  if (p.verbose) {
    static const char* names[] = {"OPTIMAL", "MAX_ITER", "TIME_LIMIT", "NUMERICAL_ERROR"};
    std::printf("Status: %s  Iterations: %lld  Time: %.3f s  Primal Objective: %.12e  KKT: %.3e\n",
                names[status], (long long)L.iter, t_end, L.res.pobj, L.res.KKT);
  }
  return HPRQP_OK;
}

// Time `iters` HPR iterations pass by pass (CUDA events) from the zero state.
// Per-kernel time of each pass without the launch gap that an event between
// passes adds: one iteration is captured into a CUDA graph, its kernel nodes
// are ordered along the graph's edges, and each node's kernel is launched
// alone kReps times back to back with programmatic dependent launch (as in
// the loop); the CUDA-event time / kReps goes to ms[k].  Skipped (ms stays 0)
// when the iteration is not exactly one kernel per pass (e.g. the QAP
// operator's GEMMs).  The repeated launches overwrite iterates: profiling
// only.
template <typename F>
static void back_to_back(Common& cm, int np, F one_iteration, double* ms) {
  constexpr int kReps = 50;
  cudaGraph_t g = nullptr;
  HPRQP_CUDA(cudaStreamBeginCapture(cm.stream, cudaStreamCaptureModeThreadLocal));
  const int64_t l0 = cm.launches;
  one_iteration();
  cm.launches = l0;
  HPRQP_CUDA(cudaStreamEndCapture(cm.stream, &g));
  size_t nn = 0, ne = 0;
  HPRQP_CUDA(cudaGraphGetNodes(g, nullptr, &nn));
  std::vector<cudaGraphNode_t> nodes(nn);
  HPRQP_CUDA(cudaGraphGetNodes(g, nodes.data(), &nn));
  // programmatic (PDL) edges carry edge data: the _v2 query returns them
  HPRQP_CUDA(cudaGraphGetEdges_v2(g, nullptr, nullptr, nullptr, &ne));
  std::vector<cudaGraphNode_t> from(ne), to(ne);
  std::vector<cudaGraphEdgeData> edata(ne);
  if (ne) HPRQP_CUDA(cudaGraphGetEdges_v2(g, from.data(), to.data(), edata.data(), &ne));
  // topological order (Kahn), kernel nodes only
  std::vector<int> indeg(nn, 0);
  auto idx = [&](cudaGraphNode_t x) { return (int)(std::find(nodes.begin(), nodes.end(), x) - nodes.begin()); };
  for (size_t e = 0; e < ne; ++e) indeg[idx(to[e])]++;
  std::vector<int> order, ready;
  for (size_t i = 0; i < nn; ++i)
    if (!indeg[i]) ready.push_back((int)i);
  while (!ready.empty()) {
    const int i = ready.front();
    ready.erase(ready.begin());
    order.push_back(i);
    for (size_t e = 0; e < ne; ++e)
      if (from[e] == nodes[i] && --indeg[idx(to[e])] == 0) ready.push_back(idx(to[e]));
  }
  std::vector<cudaGraphNode_t> kern;
  for (int i : order) {
    cudaGraphNodeType t;
    HPRQP_CUDA(cudaGraphNodeGetType(nodes[i], &t));
    if (t == cudaGraphNodeTypeKernel) kern.push_back(nodes[i]);
  }
  if ((int)kern.size() == np && np <= HPRQP_MAX_PASSES) {
    cudaEvent_t a, b;
    HPRQP_CUDA(cudaEventCreate(&a));
    HPRQP_CUDA(cudaEventCreate(&b));
    for (int k = 0; k < np; ++k) {
      cudaKernelNodeParams kp{};
      HPRQP_CUDA(cudaGraphKernelNodeGetParams(kern[k], &kp));
      cudaLaunchConfig_t cfg{};
      cfg.gridDim = kp.gridDim;
      cfg.blockDim = kp.blockDim;
      cfg.dynamicSmemBytes = kp.sharedMemBytes;
      cfg.stream = cm.stream;
      cudaLaunchAttribute attr[1];
      attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
      attr[0].val.programmaticStreamSerializationAllowed = 1;
      cfg.attrs = attr;
      cfg.numAttrs = cm.pdl ? 1 : 0;
      for (int r = 0; r < 3; ++r) HPRQP_CUDA(cudaLaunchKernelExC(&cfg, kp.func, kp.kernelParams));
      HPRQP_CUDA(cudaEventRecord(a, cm.stream));
      for (int r = 0; r < kReps; ++r) HPRQP_CUDA(cudaLaunchKernelExC(&cfg, kp.func, kp.kernelParams));
      HPRQP_CUDA(cudaEventRecord(b, cm.stream));
      HPRQP_CUDA(cudaEventSynchronize(b));
      float t = 0;
      HPRQP_CUDA(cudaEventElapsedTime(&t, a, b));
      ms[k] = t / kReps;
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
  }
  cudaGraphDestroy(g);
}

static void profile(Handle& H, const hprqp_params& p, int64_t iters, bool full, hprqp_pass_stats* out) {
  prepare(H, p);
  Common& cm = *H.cm;
  const Prepared& pp = H.pp;
  Engine<double>& E64 = *H.e64;
  double lamA = 0.0, lamQ = 0.0;
  estimate_lambdas(H, p, p.precision == HPRQP_PRECISION_FP32_POLISH, &lamA, &lamQ);
  double sigma0 = p.sigma > 0 ? p.sigma : 1.0;
  if (p.sigma == -1)
    sigma0 = (pp.norm_c > 1e-16 && pp.norm_b > 1e-16 && pp.norm_b < 1e16 && pp.norm_c < 1e16) ? pp.norm_b / pp.norm_c : 1.0;
  auto run = [&](auto& E) {
    start_engine(H, E, p, lamA, lamQ, sigma0, nullptr, nullptr);
    const int np = E.npasses();
    for (int w = 0; w < 5; ++w) E.step(full, 0.5, 0.5);
    // whole iterations, no per-pass events
    cudaEvent_t a, b;
    HPRQP_CUDA(cudaEventCreate(&a));
    HPRQP_CUDA(cudaEventCreate(&b));
    HPRQP_CUDA(cudaEventRecord(a, cm.stream));
    for (int64_t k = 0; k < iters; ++k) E.step(full, 1.0 / (k + 2.0), 1.0 - 1.0 / (k + 2.0));
    HPRQP_CUDA(cudaEventRecord(b, cm.stream));
    HPRQP_CUDA(cudaEventSynchronize(b));
    float ms = 0;
    HPRQP_CUDA(cudaEventElapsedTime(&ms, a, b));
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    // per pass: np + 1 marks per iteration
    std::vector<cudaEvent_t> ev((size_t)iters * (np + 1));
    for (auto& e : ev) HPRQP_CUDA(cudaEventCreate(&e));
    E.prof = &ev;
    E.prof_k = 0;
    for (int64_t k = 0; k < iters; ++k) E.step(full, 1.0 / (k + 2.0), 1.0 - 1.0 / (k + 2.0));
    E.prof = nullptr;
    HPRQP_CUDA(cudaStreamSynchronize(cm.stream));
    std::memset(out, 0, sizeof(*out));
    out->npass = np;
    out->path = E.path;
    out->iters = iters;
    out->ms_per_iter = ms / (double)iters;
    for (int k = 0; k < np && k < HPRQP_MAX_PASSES; ++k) {
      double tot = 0.0;
      for (int64_t it = 0; it < iters; ++it) {
        float t = 0;
        HPRQP_CUDA(cudaEventElapsedTime(&t, ev[it * (np + 1) + k], ev[it * (np + 1) + k + 1]));
        tot += t;
      }
      const char* name;
      double bytes;
      int tpr;
      E.pass_info(k, &name, &bytes, &tpr);
      std::snprintf(out->name[k], sizeof(out->name[k]), "%s", name);
      out->ms_per_launch[k] = tot / (double)iters;
      out->bytes_per_launch[k] = bytes;
      out->threads_per_row[k] = tpr;
      out->bytes_per_iter += bytes;
    }
    for (auto& e : ev) cudaEventDestroy(e);
    back_to_back(cm, np, [&] { E.step(full, 0.5, 0.5); }, out->ms_back_to_back);
  };
  if (p.precision == HPRQP_PRECISION_FP32_POLISH) run(*H.e32);
  else run(E64);
}

}  // namespace hprqp

using hprqp::Error;
using hprqp::Handle;

struct hprqp_ctx : hprqp::Handle {};

#define HPRQP_GUARD(h, body)                                        \
  try {                                                             \
    if (h) cudaSetDevice(h->device);                                \
    body;                                                           \
    return HPRQP_OK;                                                \
  } catch (const Error& e) {                                        \
    (h ? h->err : hprqp::g_global_err) = e.what();                  \
    return e.code;                                                  \
  } catch (const std::exception& e) {                               \
    (h ? h->err : hprqp::g_global_err) = e.what();                  \
    return HPRQP_E_CUDA;                                            \
  }

extern "C" {

void hprqp_default_params(hprqp_params* p) {
  if (!p) return;
  std::memset(p, 0, sizeof(*p));
  p->stoptol = 1e-6;
  p->sigma = -1;
  p->max_iter = 2147483647;
  p->sigma_fixed = 0;
  p->time_limit = 3600.0;
  p->eig_factor = 1.05;
  p->check_iter = 100;
  p->warm_up = 0;
  p->spmv_mode_Q = 0;
  p->spmv_mode_A = 0;
  p->print_frequency = -1;
  p->device_number = 0;
  p->use_Ruiz_scaling = 1;
  p->use_bc_scaling = 0;
  p->use_l2_scaling = 0;
  p->use_Pock_Chambolle_scaling = 1;
  p->problem_type = HPRQP_PROBLEM_QP;
  p->lambda = 0.0;
  p->auto_save = 0;
  p->verbose = 1;
  p->use_gpu = 1;
  p->precision = HPRQP_PRECISION_FP64;
  p->polish_tol = -1.0;
  p->lambda_max_A_override = -1.0;
  p->lambda_max_Q_override = -1.0;
  p->profile_passes = 0;
}

int hprqp_abi_info(int64_t* out) {
  if (!out) return HPRQP_E_ARG;
  out[0] = HPRQP_ABI_VERSION;
  out[1] = (int64_t)sizeof(hprqp_problem);
  out[2] = (int64_t)sizeof(hprqp_params);
  out[3] = (int64_t)sizeof(hprqp_result);
  return HPRQP_OK;
}

int hprqp_create(hprqp_handle* out, int32_t device) {
  hprqp_ctx* h = nullptr;
  try {
    if (!out) throw Error(HPRQP_E_ARG, "null handle pointer");
    *out = nullptr;
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0)
      throw Error(HPRQP_E_CUDA, std::string("CUDA is not functional: ") + (e != cudaSuccess ? cudaGetErrorString(e) : "no device"));
    if (device < 0 || device >= count)
      throw Error(HPRQP_E_CUDA, "Invalid GPU device number " + std::to_string(device) + ". Valid range is [0, " +
                                    std::to_string(count - 1) + "]");
    HPRQP_CUDA(cudaSetDevice(device));
    h = new hprqp_ctx();
    h->device = device;
    h->cm = std::make_unique<hprqp::Common>();
    h->cm->init();
    *out = h;
    return HPRQP_OK;
  } catch (const Error& e) {
    hprqp::g_global_err = e.what();
    delete h;
    return e.code;
  } catch (const std::exception& e) {
    hprqp::g_global_err = e.what();
    delete h;
    return HPRQP_E_CUDA;
  }
}

int hprqp_load(hprqp_handle h, const hprqp_problem* prob) {
  if (!h) return HPRQP_E_ARG;
  HPRQP_GUARD(h, {
    h->prepared = false;
    h->e64.reset();
    h->e32.reset();
    h->cm->qmap = nullptr;  // a custom operator is bound per loaded problem
    h->cm->qmap_user = nullptr;
    hprqp::load_problem(prob, h->hp);
  })
}

int hprqp_prepare(hprqp_handle h, const hprqp_params* params) {
  if (!h || !params) return HPRQP_E_ARG;
  HPRQP_GUARD(h, { hprqp::prepare(*h, *params); })
}

int hprqp_solve(hprqp_handle h, const hprqp_params* params, const double* initial_x, const double* initial_y,
                hprqp_result* result, double* x, double* y, double* z, double* w) {
  if (!h || !params || !result) return HPRQP_E_ARG;
  HPRQP_GUARD(h, { hprqp::solve(*h, *params, initial_x, initial_y, result, x, y, z, w); })
}

int hprqp_profile_iterations(hprqp_handle h, const hprqp_params* params, int64_t iters, int32_t full,
                             hprqp_pass_stats* out) {
  if (!h || !params || !out || iters <= 0) return HPRQP_E_ARG;
  HPRQP_GUARD(h, { hprqp::profile(*h, *params, iters, full != 0, out); })
}

int hprqp_get_pass_stats(hprqp_handle h, hprqp_pass_stats* fp64, hprqp_pass_stats* fp32) {
  if (!h) return HPRQP_E_ARG;
  if (fp64) *fp64 = h->stats64;
  if (fp32) *fp32 = h->stats32;
  return HPRQP_OK;
}

int hprqp_set_trace(hprqp_handle h, int64_t iters, double* x_trace, double* y_trace, double* w_trace) {
  if (!h || iters < 0) return HPRQP_E_ARG;
  h->trace_iters = iters;
  h->xt = x_trace;
  h->yt = y_trace;
  h->wt = w_trace;
  return HPRQP_OK;
}

int hprqp_set_save_file(hprqp_handle h, const char* path) {
  if (!h || !path || !path[0]) return HPRQP_E_ARG;
  h->save_file = path;
  return HPRQP_OK;
}

int hprqp_solve_resume(hprqp_handle h, const hprqp_params* params, const char* path, hprqp_result* result,
                       double* x, double* y, double* z, double* w) {
  if (!h || !params || !path || !result) return HPRQP_E_ARG;
  HPRQP_GUARD(h, {
    if (!h->hp.loaded) throw hprqp::Error(HPRQP_E_STATE, "load a problem first");
    hprqp::check_params(*params);
    hprqp::ck::Reader rs;
    std::string err;
    if (!rs.read(path, err)) throw hprqp::Error(HPRQP_E_ARG, err);
    hprqp::solve(*h, *params, nullptr, nullptr, result, x, y, z, w, &rs);
  })
}

int hprqp_set_qmap(hprqp_handle h, hprqp_qmap_fn qmap, void* user) {
  if (!h) return HPRQP_E_ARG;
  HPRQP_GUARD(h, {
    if (!h->hp.loaded || h->hp.Q_kind != HPRQP_Q_CUSTOM)
      throw hprqp::Error(HPRQP_E_STATE, "hprqp_set_qmap: load a problem with Q_kind = HPRQP_Q_CUSTOM first");
    if (!qmap) throw hprqp::Error(HPRQP_E_ARG, "hprqp_set_qmap: null callback");
    h->cm->qmap = qmap;
    h->cm->qmap_user = user;
  })
}

int hprqp_set_trace_scalars(hprqp_handle h, double* sigma_trace, int64_t* inner_trace) {
  if (!h) return HPRQP_E_ARG;
  h->sig_t = sigma_trace;
  h->inner_t = inner_trace;
  return HPRQP_OK;
}

const char* hprqp_last_error(hprqp_handle h) { return h ? h->err.c_str() : hprqp::g_global_err.c_str(); }

int hprqp_destroy(hprqp_handle h) {
  if (!h) return HPRQP_OK;
  cudaSetDevice(h->device);
  const double t0 = hprqp::now_s();
  if (h->cm && h->cm->stream) cudaStreamSynchronize(h->cm->stream);
  h->e32.reset();
  h->e64.reset();
  const double t1 = hprqp::now_s();
  h->cm.reset();
  const double t2 = hprqp::now_s();
  h->hp = hprqp::HostProblem();
  h->pp = hprqp::Prepared();
  const double t3 = hprqp::now_s();
  delete h;
  if (const char* tv = std::getenv("HPRQP_TIMING"))
    if (tv[0] == '1')
      std::fprintf(stderr, "[hprqp] destroy: engines %.3f s, device resources %.3f s, host arrays %.3f s, rest %.3f s\n",
                   t1 - t0, t2 - t1, t3 - t2, hprqp::now_s() - t3);
  return HPRQP_OK;
}

}  // extern "C"
