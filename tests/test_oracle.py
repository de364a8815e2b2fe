"""CPU tests of the oracle (the FP64 restatement of the reference CPU path):
pinned against the analytic optimum of the reference's model.mps example,
the reference tests' own status/tolerance assertions, scipy's HiGHS on LPs,
sklearn on LASSO, an independent numpy KKT check, and the reference's MPS
fixtures when the reference tree is given (HPRQP_REFERENCE_DATA)."""
import os

import numpy as np
import pytest

from hprqp_b200 import workloads as W
from hprqp_b200._abi import default_params
from oracle import oracle as O
from tests.kkt import kkt

REF_DATA = os.environ.get("HPRQP_REFERENCE_DATA", "")


def params(**kw):
    p = default_params()
    p.verbose = 0
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def test_toy_analytic_optimum():
    # model.mps / demo_QAbc.jl: optimum x = (1.5, 2.5), objective -8.5
    r = O.solve(W.toy_qp(), params())
    assert r.status_name == "OPTIMAL"
    assert r.residuals < 1e-6
    assert np.allclose(r.x, [1.5, 2.5], atol=1e-5)
    assert abs(r.primal_obj + 8.5) < 1e-5


@pytest.mark.parametrize("make", [W.dense_q_qp, W.small_lp])
def test_reference_suite_problems(make):
    # test/runtests.jl:285-345: status == OPTIMAL and residuals < 1e-6
    m = make()
    r = O.solve(m, params(max_iter=10000))
    assert r.status_name == "OPTIMAL" and r.residuals < 1e-6
    k = kkt(m, r.x, r.y, r.z)
    assert k["KKT"] < 1e-5


@pytest.mark.parametrize("tol", [1e-3, 1e-5])
def test_tolerances(tol):
    # test/runtests.jl:348-380
    import scipy.sparse as sp
    n, mm = 5, 2
    model = W.build_from_QAbc(sp.identity(n, format="csc"), np.ones(n), np.ones((mm, n)), np.zeros(mm),
                              np.full(mm, n / 2), np.zeros(n), np.ones(n), verbose=False)
    r = O.solve(model, params(stoptol=tol))
    assert r.status_name == "OPTIMAL" and r.residuals < tol


def test_lp_matches_highs():
    from scipy.optimize import linprog
    m = W.random_lp()
    r = O.solve(m, params())
    assert r.status_name == "OPTIMAL"
    A = m.A.toarray()
    fin_u, fin_l = np.isfinite(m.AU), np.isfinite(m.AL)
    A_ub = np.vstack([A[fin_u], -A[fin_l]])
    b_ub = np.concatenate([m.AU[fin_u], -m.AL[fin_l]])
    h = linprog(m.c, A_ub=A_ub, b_ub=b_ub, bounds=list(zip(m.l, m.u)), method="highs")
    assert h.status == 0
    assert abs(r.primal_obj - h.fun) / (1 + abs(h.fun)) < 1e-5


def test_lasso_matches_sklearn():
    from sklearn.linear_model import Lasso
    m = W.small_lasso()
    r = O.solve(m, params(problem_type=1))
    assert r.status_name == "OPTIMAL"
    A = m.Q.A
    b = None
    # recover b from c = -A'b is not unique; rebuild the instance's b instead
    rng_model = W.small_lasso()
    mm, nn = A.shape
    # objective of the oracle solution vs sklearn's minimiser of the same problem
    lam = m.lambda_
    Ad = A.toarray()
    # b satisfies c = -A'b and obj_constant = 0.5||b||^2; regenerate deterministically
    rng = np.random.default_rng(12)
    A2 = W._sprandn(rng, 60, 200, 0.1)
    xs = np.zeros(200)
    xs[rng.choice(200, 6, replace=False)] = rng.standard_normal(6)
    b = A2 @ xs + 0.01 * rng.standard_normal(60)
    assert np.allclose(-(A2.T @ b), m.c)
    sk = Lasso(alpha=lam / mm, fit_intercept=False, tol=1e-12, max_iter=200000).fit(Ad, b)
    f = lambda x: 0.5 * np.sum((Ad @ x - b) ** 2) + lam * np.abs(x).sum()
    assert abs(f(r.x) - f(sk.coef_)) / (1 + abs(f(sk.coef_))) < 1e-6
    assert abs(r.primal_obj - f(r.x)) / (1 + abs(f(r.x))) < 1e-9


@pytest.mark.parametrize("make", [W.free_var_qp, W.random_qp, lambda: W.qap_instance(8, 3)])
def test_independent_kkt(make):
    m = make()
    pt = 2 if m.Q.kind == 2 else 0
    r = O.solve(m, params(problem_type=pt))
    assert r.status_name == "OPTIMAL" and r.residuals < 1e-6
    k = kkt(m, r.x, r.y, r.z)
    assert k["err_Rp"] < 1e-5 and k["err_Rd"] < 1e-5
    assert abs(k["pobj"] - r.primal_obj) / (1 + abs(r.primal_obj)) < 1e-8


def test_warm_start_reference_semantics():
    # test/runtests.jl:165-251
    m = W.toy_qp()
    cold = O.solve(m, params(max_iter=50000))
    rx = O.solve(m, params(max_iter=50000), initial_x=cold.x)
    assert rx.status_name == "OPTIMAL" and rx.iter <= cold.iter
    ry = O.solve(m, params(max_iter=50000), initial_y=cold.y)
    assert ry.status_name == "OPTIMAL"
    rxy = O.solve(m, params(max_iter=50000), initial_x=cold.x, initial_y=cold.y)
    assert rxy.status_name == "OPTIMAL" and rxy.iter == 0


def test_max_iter_and_trace_shapes():
    m = W.random_qp()
    r = O.solve(m, params(max_iter=30), trace_iters=30)
    assert r.status_name == "MAX_ITER" and r.iter == 30
    assert r.x_trace.shape == (30, m.n) and np.all(np.isfinite(r.x_trace))


@pytest.mark.skipif(not REF_DATA or not os.path.isdir(REF_DATA), reason="reference data files not given")
@pytest.mark.parametrize("name", ["AUG3DCQP.mps", "AUG2D.mps"])
def test_reference_mps_fixtures(name):
    # test/runtests.jl:254-280 (AUG2D) and :704-788 (AUG3DCQP): OPTIMAL, < 1e-6
    from tests.mps import read_mps
    Q, c, A, AL, AU, l, u = read_mps(os.path.join(REF_DATA, name))
    m = W.build_from_QAbc(Q, c, A, AL, AU, l, u, verbose=False)
    r = O.solve(m, params(max_iter=50000), threads=4)
    assert r.status_name == "OPTIMAL" and r.residuals < 1e-6
    k = kkt(m, r.x, r.y, r.z)
    assert k["err_Rp"] < 1e-5 and k["err_Rd"] < 1e-5


def test_oracle_reproduces_golden_fixtures():
    """Regression pin: the committed fixtures (tests/golden/make_golden.py)."""
    import os
    from tests.test_gpu_parity import CASES, oracle_params
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "cases.npz"))
    for name in ("toy_diagQ", "lp", "random_lp", "lasso", "qap_n10"):
        m = CASES[name][0]()
        r = O.solve(m, oracle_params(CASES[name][1], max_iter=50000))
        assert r.status == int(g[name + "/status"]) and r.iter == int(g[name + "/iter"])
        assert abs(r.primal_obj - float(g[name + "/pobj"])) <= 1e-12 * (1 + abs(r.primal_obj))
        lamA, lamQ = g[name + "/lam"]
        t = O.solve(m, oracle_params(CASES[name][1], max_iter=10, lambda_max_A_override=lamA,
                                     lambda_max_Q_override=lamQ), trace_iters=10)
        assert np.array_equal(t.x_trace, g[name + "/x_trace"])
