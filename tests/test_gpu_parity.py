"""GPU parity tests: the CUDA engine (through the C ABI) against the oracle.

 - iterate parity: with lambda_max injected on both sides (the power method's
   start vector is the one documented deviation), the scaled iterates x, y, w
   of the first 50 HPR iterations match the oracle to 1e-10 relative;
 - solve parity: same status, objective within 1e-6 relative, KKT <= tol,
   and an independent numpy KKT check of the returned solution;
 - reference test semantics: warm start from the optimum returns iter == 0;
   an invalid device or unsupported option is an error, not a fallback.
"""
import numpy as np
import pytest

from hprqp_b200 import HPRQP_parameters, Solver
from hprqp_b200 import workloads as W
from hprqp_b200._abi import default_params
from hprqp_b200._lib import HPRQPError
from oracle import oracle as O
from tests.kkt import kkt

pytestmark = pytest.mark.gpu

ITER_RTOL = 1e-10   # first-50-iterate parity (FP64)
OBJ_RTOL = 1e-6     # objective parity of full solves

CASES = {
    "toy_diagQ": (W.toy_qp, "QP"),
    "dense_q": (W.dense_q_qp, "QP"),
    "lp": (W.small_lp, "QP"),
    "random_lp": (W.random_lp, "QP"),
    "free_var_noC": (W.free_var_qp, "QP"),
    "random_qp_n2000": (W.random_qp, "QP"),
    "lasso": (W.small_lasso, "LASSO"),
    "qap_n10": (lambda: W.qap_instance(10, 5), "QAP"),
    "grid_60x60": (lambda: W.grid_qp(N=60), "QP"),
}
_models = {}


def model(name):
    if name not in _models:
        _models[name] = CASES[name][0]()
    return _models[name]


def oracle_params(ptype, **kw):
    p = default_params()
    p.verbose = 0
    p.problem_type = {"QP": 0, "LASSO": 1, "QAP": 2}[ptype]
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def gpu_params(ptype, **kw):
    p = HPRQP_parameters(verbose=False, problem_type=ptype)
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def rel(a, b):
    return np.max(np.abs(a - b)) / max(1.0, np.max(np.abs(b))) if a.size else 0.0


@pytest.mark.parametrize("name", list(CASES))
def test_first_50_iterates_match_oracle(name):
    m = model(name)
    ptype = CASES[name][1]
    ref0 = O.solve(m, oracle_params(ptype, max_iter=1))
    lamA = ref0.lambda_max_A if m.m else -1.0
    lamQ = ref0.lambda_max_Q if (ref0.lambda_max_Q > 0 and not ref0.Q_is_diag) else -1.0
    kw = dict(max_iter=50, lambda_max_A_override=lamA, lambda_max_Q_override=lamQ)
    ref = O.solve(m, oracle_params(ptype, **kw), trace_iters=50)
    s = Solver().load(m)
    xt, yt, wt = s.set_trace(50)
    res = s.solve(gpu_params(ptype, **kw))
    s.close()
    assert res.status == ref.status_name == "MAX_ITER"
    for k in range(50):
        assert rel(xt[k], ref.x_trace[k]) < ITER_RTOL, (name, "x", k, rel(xt[k], ref.x_trace[k]))
        assert rel(wt[k], ref.w_trace[k]) < ITER_RTOL, (name, "w", k)
        if m.m:
            assert rel(yt[k], ref.y_trace[k]) < ITER_RTOL, (name, "y", k)


@pytest.mark.parametrize("name", list(CASES))
def test_full_solve_matches_oracle(name):
    m = model(name)
    ptype = CASES[name][1]
    ref = O.solve(m, oracle_params(ptype, max_iter=50000))
    s = Solver().load(m)
    res = s.solve(gpu_params(ptype, max_iter=50000))
    s.close()
    assert ref.status_name == "OPTIMAL"
    assert res.status == "OPTIMAL" and res.residuals < 1e-6
    assert abs(res.primal_obj - ref.primal_obj) / (1 + abs(ref.primal_obj)) < OBJ_RTOL
    assert res.iter == ref.iter and res.restarts == ref.restarts, (res.iter, ref.iter, res.restarts, ref.restarts)
    assert res.gpu_launches > 0
    if ptype != "LASSO":
        k = kkt(m, res.x, res.y, res.z)
        assert k["err_Rp"] < 1e-5 and k["err_Rd"] < 1e-5


@pytest.mark.parametrize("name", ["random_qp_n2000", "grid_60x60", "lp", "free_var_noC", "lasso", "qap_n10"])
def test_fp32_polish_matches_fp64(name):
    m = model(name)
    ptype = CASES[name][1]
    ref = O.solve(m, oracle_params(ptype, max_iter=50000))
    s = Solver().load(m)
    res = s.solve(gpu_params(ptype, max_iter=50000, precision="fp32_polish"))
    s.close()
    assert res.status == "OPTIMAL" and res.residuals < 1e-6
    assert res.iter_fp32 > 0
    assert abs(res.primal_obj - ref.primal_obj) / (1 + abs(ref.primal_obj)) < 1e-5


def test_warm_start_from_optimum_needs_zero_iterations():
    # test/runtests.jl:165-251
    m = model("toy_diagQ")
    s = Solver().load(m)
    cold = s.solve(gpu_params("QP", max_iter=50000))
    rx = s.solve(gpu_params("QP", max_iter=50000, initial_x=cold.x))
    assert rx.status == "OPTIMAL" and rx.iter <= cold.iter
    ry = s.solve(gpu_params("QP", max_iter=50000, initial_y=cold.y))
    assert ry.status == "OPTIMAL"
    rxy = s.solve(gpu_params("QP", max_iter=50000, initial_x=cold.x, initial_y=cold.y))
    s.close()
    assert rxy.status == "OPTIMAL" and rxy.iter == 0


def test_warm_start_matches_oracle_iterates():
    m = model("random_qp_n2000")
    ref0 = O.solve(m, oracle_params("QP", max_iter=1))
    kw = dict(max_iter=30, lambda_max_A_override=ref0.lambda_max_A, lambda_max_Q_override=ref0.lambda_max_Q)
    rng = np.random.default_rng(3)
    x0, y0 = rng.uniform(-1, 1, m.n), rng.standard_normal(m.m)
    ref = O.solve(m, oracle_params("QP", **kw), initial_x=x0, initial_y=y0, trace_iters=30)
    s = Solver().load(m)
    xt, yt, wt = s.set_trace(30)
    s.solve(gpu_params("QP", initial_x=x0, initial_y=y0, **kw))
    s.close()
    for k in range(30):
        assert rel(xt[k], ref.x_trace[k]) < ITER_RTOL
        assert rel(yt[k], ref.y_trace[k]) < ITER_RTOL


def test_max_iter_and_time_limit_status():
    m = model("random_qp_n2000")
    s = Solver().load(m)
    r = s.solve(gpu_params("QP", max_iter=7))
    assert r.status == "MAX_ITER" and r.iter == 7
    r = s.solve(gpu_params("QP", time_limit=0.0))
    s.close()
    assert r.status == "TIME_LIMIT"


def test_invalid_device_is_an_error():
    with pytest.raises(HPRQPError):
        Solver(device=999)


def test_unsupported_options_are_errors():
    s = Solver().load(model("toy_diagQ"))
    with pytest.raises(HPRQPError):
        s.solve(gpu_params("QP", use_gpu=False))
    s.close()


def test_grid_qp_full_size_properties():
    # 700 x 700 grid (n = 490,000, m = 974,408), the benchmark problem: the
    # oracle's recorded FP64 solve of it (tests/golden/grid_qp_oracle.json:
    # OPTIMAL in 570 iterations, its objective) plus size-independent
    # properties: both precision modes reach 1e-6, agree on the objective,
    # and pass the numpy KKT check.
    import json
    import os
    with open(os.path.join(os.path.dirname(__file__), "golden", "grid_qp_oracle.json")) as f:
        gold = json.load(f)["700"]
    m = W.grid_qp()
    s = Solver().load(m)
    r64 = s.solve(gpu_params("QP"))
    r32 = s.solve(gpu_params("QP", precision="fp32_polish"))
    s.close()
    assert r64.status == r32.status == gold["status"] == "OPTIMAL"
    assert r64.iter == gold["iter"], (r64.iter, gold["iter"])
    assert abs(r64.primal_obj - gold["primal_obj"]) / (1 + abs(gold["primal_obj"])) < OBJ_RTOL
    assert abs(r32.primal_obj - gold["primal_obj"]) / (1 + abs(gold["primal_obj"])) < OBJ_RTOL
    assert abs(r64.primal_obj - r32.primal_obj) / (1 + abs(r64.primal_obj)) < 1e-5
    for r in (r64, r32):
        k = kkt(m, r.x, r.y, r.z)
        assert k["err_Rp"] < 1e-5 and k["err_Rd"] < 1e-5 and k["gap"] < 1e-5


@pytest.mark.parametrize("name", list(CASES))
def test_against_committed_golden_fixtures(name):
    """The GPU path against the committed oracle fixtures (tests/golden/cases.npz)."""
    import os
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "cases.npz"))
    m = model(name)
    ptype = CASES[name][1]
    lamA, lamQ = g[name + "/lam"]
    s = Solver().load(m)
    xt, yt, wt = s.set_trace(10)
    s.solve(gpu_params(ptype, max_iter=10, lambda_max_A_override=lamA, lambda_max_Q_override=lamQ))
    s.set_trace(0)
    for k in range(10):
        assert rel(xt[k], g[name + "/x_trace"][k]) < ITER_RTOL
        if m.m:
            assert rel(yt[k], g[name + "/y_trace"][k]) < ITER_RTOL
    r = s.solve(gpu_params(ptype, max_iter=50000))
    s.close()
    assert r.status == "OPTIMAL" and int(g[name + "/status"]) == 0
    pobj = float(g[name + "/pobj"])
    assert abs(r.primal_obj - pobj) / (1 + abs(pobj)) < OBJ_RTOL
    xg = g[name + "/x"]
    assert np.max(np.abs(r.x - xg)) / max(1.0, np.max(np.abs(xg))) < 1e-3
