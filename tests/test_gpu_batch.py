"""GPU tests of the batched LASSO-family solve: every instance of a batch
(uneven sizes) reaches the status and objective of its own single solve
(hprqp_solve), in both precision modes, and warm starts are honoured per
instance."""
import numpy as np
import pytest

from hprqp_b200 import HPRQP_parameters, Solver
from hprqp_b200 import workloads as W
from hprqp_b200.batch import solve_batch

pytestmark = pytest.mark.gpu


def family():
    ms = [W.small_lasso(m=60 + 10 * k, n=200 + 37 * k, seed=100 + k) for k in range(6)]
    ms += W.lasso_family(6, m=120, n=400, density=0.05, start=500)
    return ms


@pytest.mark.parametrize("precision", ["fp64", "fp32_polish"])
def test_batch_matches_single_solves(precision):
    ms = family()
    p = HPRQP_parameters(verbose=False, problem_type="LASSO", precision=precision)
    batch = solve_batch(ms, p)
    for m, rb in zip(ms, batch):
        s = Solver().load(m)
        rs = s.solve(HPRQP_parameters(verbose=False, problem_type="LASSO"))
        s.close()
        assert rb.status == rs.status == "OPTIMAL"
        assert rb.residuals < 1e-6
        tol = 1e-6 if precision == "fp64" else 1e-5
        assert abs(rb.primal_obj - rs.primal_obj) / (1 + abs(rs.primal_obj)) < tol
        if precision == "fp64":  # same arithmetic: the same trajectory
            assert abs(rb.iter - rs.iter) <= max(20, 0.1 * rs.iter), (rb.iter, rs.iter)
            assert np.max(np.abs(rb.x - rs.x)) / max(1.0, np.max(np.abs(rs.x))) < 1e-3


def test_batch_warm_start_from_optimum():
    ms = family()[:4]
    p = HPRQP_parameters(verbose=False, problem_type="LASSO")
    cold = solve_batch(ms, p)
    warm = solve_batch(ms, p, initial_x=[r.x for r in cold], sigma0=[r.sigma for r in cold])
    for c, w in zip(cold, warm):
        assert w.status == "OPTIMAL" and w.iter < c.iter
