"""GPU tests of the LASSO path (implicit Q = A'A, src/Q_operators/
LASSO_operator.jl:86-117) on data with lognormal row lengths, the shape of
the 20,000 x 150,000 LASSO benchmark configuration, through the C ABI:

 - a scaled-down instance of the same generator (400 x 20,000, row lengths
   lognormal(5, 0.8): ~8e4 nonzeros, longest rows > 2,000 entries, so the
   row-split schedule cuts them into pieces): the first 50 iterates match
   the oracle to 1e-10 under the autotuned, row-split and 32-lanes-per-row
   CSR schedules; full solves give the oracle's status, iteration count and
   objective (1e-6); FP32 + polish reaches 1e-6 with the objective to 1e-5;
 - the full-size instance (20,000 x 150,000, ~1.1e7 nonzeros): both
   precision modes reach 1e-6, agree on the objective, and the solution
   passes an independent check of the LASSO optimality conditions.
"""
import numpy as np
import pytest

from hprqp_b200 import HPRQP_parameters, Solver
from hprqp_b200 import workloads as W
from oracle import oracle as O
from tests.test_gpu_parity import ITER_RTOL, OBJ_RTOL, oracle_params, rel

pytestmark = pytest.mark.gpu

_small = None


def small():
    global _small
    if _small is None:
        _small = W.lasso(m=400, n=20000, seed=31, mu=5.0)
    return _small


def params(**kw):
    p = HPRQP_parameters(verbose=False, problem_type="LASSO")
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def test_small_instance_has_long_rows():
    A = small().Q.A.tocsr()
    lens = np.diff(A.indptr)
    assert lens.max() > 2048 and lens.max() > 8 * lens.mean()


@pytest.mark.parametrize("mode", ["auto", "split", 32])
def test_first_50_iterates_match_oracle(mode):
    m = small()
    ref0 = O.solve(m, oracle_params("LASSO", max_iter=1))
    kw = dict(max_iter=50, lambda_max_Q_override=ref0.lambda_max_Q)
    ref = O.solve(m, oracle_params("LASSO", **kw), trace_iters=50)
    s = Solver().load(m)
    xt, _, wt = s.set_trace(50)
    s.solve(params(spmv_mode_Q=mode, **kw))
    s.set_trace(0)
    s.close()
    for k in range(50):
        assert rel(xt[k], ref.x_trace[k]) < ITER_RTOL, (mode, "x", k, rel(xt[k], ref.x_trace[k]))
        assert rel(wt[k], ref.w_trace[k]) < ITER_RTOL, (mode, "w", k)


@pytest.mark.parametrize("mode", ["auto", "split"])
def test_full_solve_matches_oracle(mode):
    m = small()
    ref = O.solve(m, oracle_params("LASSO", max_iter=50000))
    s = Solver().load(m)
    r = s.solve(params(max_iter=50000, spmv_mode_Q=mode))
    r32 = s.solve(params(max_iter=50000, spmv_mode_Q=mode, precision="fp32_polish"))
    s.close()
    assert ref.status_name == "OPTIMAL"
    assert r.status == "OPTIMAL" and r.residuals < 1e-6
    assert r.iter == ref.iter, (r.iter, ref.iter)
    assert abs(r.primal_obj - ref.primal_obj) / (1 + abs(ref.primal_obj)) < OBJ_RTOL
    assert r32.status == "OPTIMAL" and r32.residuals < 1e-6 and r32.iter_fp32 > 0
    assert abs(r32.primal_obj - ref.primal_obj) / (1 + abs(ref.primal_obj)) < 1e-5


def lasso_optimality(model, x):
    """Relative violation of the LASSO optimality conditions: with
    g = A'(A x - b), g_i = -lambda sign(x_i) where x_i != 0 and |g_i| <=
    lambda elsewhere (b and A from the generator)."""
    A = model.Q.A.tocsr()
    b = model.meta["b"]
    lam = model.lambda_
    g = A.T @ (A @ x - b)
    on = np.abs(x) > 1e-9 * max(1.0, np.abs(x).max())
    v_on = np.abs(g[on] + lam * np.sign(x[on])).max() if on.any() else 0.0
    v_off = max(0.0, (np.abs(g[~on]) - lam).max()) if (~on).any() else 0.0
    return max(v_on, v_off) / (lam + np.abs(A.T @ b).max())


def test_full_size_lasso_properties():
    m = W.lasso()  # 20,000 x 150,000, lognormal rows
    s = Solver().load(m)
    r64 = s.solve(params())
    r32 = s.solve(params(precision="fp32_polish"))
    s.close()
    assert r64.status == r32.status == "OPTIMAL"
    assert r64.residuals < 1e-6 and r32.residuals < 1e-6
    assert abs(r64.primal_obj - r32.primal_obj) / (1 + abs(r64.primal_obj)) < 1e-5
    for r in (r64, r32):
        assert lasso_optimality(m, r.x) < 1e-4
