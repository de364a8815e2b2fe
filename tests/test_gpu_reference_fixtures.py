"""GPU tests on the reference's own test problems (tests/golden/
reference_fixtures.npz: data/AUG2D.mps, data/AUG3DCQP.mps and the QAP
data/esc64a.mat of the reference tree), through the C ABI.

 - Every pinned row schedule, as the reference runs AUG2D and AUG3DCQP under
   every SpMV mode (test/runtests.jl:704-788): status OPTIMAL, residuals
   < 1e-6 (the reference test's assertions), the oracle's objective to 1e-6
   and its iteration count.
 - esc64a as a QAP with its own S, T (test/runtests.jl:467-506), in FP64 and
   in FP32 + FP64 polish.
 - Restart and sigma parity over whole solves: with lambda_max injected, the
   engine takes the oracle's restarts at the same iterations (exactly), its
   sigma sequence to 1e-6 and its iterates x, y, w to 1e-8 on every iteration
   of solves with at least three restarts (measured on a B200: sigma 1.8e-8,
   iterates 3.2e-11 on AUG3DCQP).  Sigma is the golden-section minimiser of
   a sigma + b / sigma + c sigma^2 / (1 + d sigma) (src/kernels.jl:1449-1486),
   a function flat at its minimum, so its comparisons resolve the minimiser
   only to about sqrt(machine epsilon) relative: the rounding-level
   differences of the device reductions move sigma by up to ~1e-8.
"""
import numpy as np
import pytest

from hprqp_b200 import HPRQP_parameters, Solver
from oracle import oracle as O
from tests import reference_fixtures as RF
from tests.kkt import kkt
from tests.test_gpu_parity import oracle_params, rel

pytestmark = pytest.mark.gpu

OBJ_RTOL = 1e-6
TRACE_RTOL = 1e-8
SIGMA_RTOL = 1e-6
_models = {}


def model(name):
    if name not in _models:
        _models[name] = RF.model(name)
    return _models[name]


def gpu_params(name, **kw):
    p = HPRQP_parameters(verbose=False, problem_type=RF.PTYPE[name], max_iter=RF.MAX_ITER[name])
    for k, v in kw.items():
        setattr(p, k, v)
    return p


SCHEDULES = [("auto", "auto"), (1, 1), (2, 2), (4, 4), (8, 8), (16, 16), (32, 32), ("sell", "sell"),
             ("ell", "ell"), ("ell", 4), (1, "sell")]


@pytest.mark.parametrize("sched", SCHEDULES, ids=[f"Q{q}-A{a}" for q, a in SCHEDULES])
@pytest.mark.parametrize("name", ["AUG3DCQP", "AUG2D"])
def test_mps_fixture_every_schedule(name, sched):
    m = model(name)
    ref = RF.ref(name)
    s = Solver().load(m)
    r = s.solve(gpu_params(name, spmv_mode_Q=sched[0], spmv_mode_A=sched[1]))
    s.close()
    assert r.status == "OPTIMAL" and r.residuals < 1e-6
    assert abs(r.primal_obj - ref["primal_obj"]) / (1 + abs(ref["primal_obj"])) < OBJ_RTOL
    assert r.iter == ref["iter"], (r.iter, ref["iter"])
    assert r.restarts == ref["restarts"]
    k = kkt(m, r.x, r.y, r.z)
    assert k["err_Rp"] < 1e-5 and k["err_Rd"] < 1e-5


@pytest.mark.parametrize("name", ["AUG3DCQP", "AUG2D", "esc64a"])
def test_fixture_fp32_polish(name):
    m = model(name)
    ref = RF.ref(name)
    s = Solver().load(m)
    r = s.solve(gpu_params(name, precision="fp32_polish"))
    s.close()
    assert r.status == "OPTIMAL" and r.residuals < 1e-6
    assert r.iter_fp32 > 0
    assert abs(r.primal_obj - ref["primal_obj"]) / (1 + abs(ref["primal_obj"])) < 1e-5


def test_esc64a_qap():
    m = model("esc64a")
    ref = RF.ref("esc64a")
    s = Solver().load(m)
    r = s.solve(gpu_params("esc64a"))
    s.close()
    assert r.status == "OPTIMAL" and r.residuals < 1e-6
    assert abs(r.primal_obj - ref["primal_obj"]) / (1 + abs(ref["primal_obj"])) < OBJ_RTOL
    assert r.iter == ref["iter"] and r.restarts == ref["restarts"]
    # the relaxation's constraints: X doubly stochastic, X >= 0
    n = int(round(np.sqrt(m.n)))
    X = r.x.reshape(n, n, order="F")
    assert np.max(np.abs(X.sum(axis=0) - 1)) < 1e-5 and np.max(np.abs(X.sum(axis=1) - 1)) < 1e-5
    assert X.min() > -1e-6


@pytest.mark.parametrize("name", ["AUG3DCQP", "esc64a"])
def test_restart_and_sigma_trace_match_oracle(name):
    m = model(name)
    ref = RF.ref(name)
    iters = ref["iter"]
    restarts = RF.restart_iterations(ref["inner"])
    assert len(restarts) >= 3 and iters >= 300
    ptype = RF.PTYPE[name]
    ref0 = O.solve(m, oracle_params(ptype, max_iter=1))
    lamQ = ref0.lambda_max_Q if (ref0.lambda_max_Q > 0 and not ref0.Q_is_diag) else -1.0
    kw = dict(max_iter=iters, lambda_max_A_override=ref0.lambda_max_A, lambda_max_Q_override=lamQ)
    o = O.solve(m, oracle_params(ptype, **kw), trace_iters=iters)
    assert o.status_name == "OPTIMAL" and o.iter == iters
    s = Solver().load(m)
    xt, yt, wt = s.set_trace(iters)
    r = s.solve(gpu_params(name, **kw))
    sig, inner = s.scalar_trace()
    s.set_trace(0)
    s.close()
    assert r.status == "OPTIMAL" and r.iter == iters and r.restarts == o.restarts
    assert np.array_equal(inner, o.inner_trace), np.nonzero(inner != o.inner_trace)[0][:5]
    assert RF.restart_iterations(inner) == RF.restart_iterations(o.inner_trace)
    sig_dev = np.max(np.abs(sig - o.sigma_trace) / np.abs(o.sigma_trace))
    it_dev = max(max(rel(xt[k], o.x_trace[k]), rel(wt[k], o.w_trace[k]), rel(yt[k], o.y_trace[k]))
                 for k in range(iters))
    print(f"{name}: restarts at {RF.restart_iterations(inner)}; max sigma rel dev {sig_dev:.2e}; "
          f"max iterate rel dev {it_dev:.2e}")
    assert sig_dev < SIGMA_RTOL, sig_dev
    assert it_dev < TRACE_RTOL, it_dev
