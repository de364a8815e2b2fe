"""GPU tests of the batched QAP-relaxation solve (build_from_ABST models of
uneven size in one batch): every instance reaches the status and objective
of its own single solve (hprqp_solve), in FP64 (same trajectory: iteration
counts and solutions agree) and with FP32 + FP64 polish."""
import numpy as np
import pytest

from hprqp_b200 import HPRQP_parameters, Solver
from hprqp_b200 import workloads as W
from hprqp_b200.batch import solve_batch

pytestmark = pytest.mark.gpu


def family():
    return [W.qap_instance(n, 40 + n) for n in (6, 9, 12, 17, 23)]


def single(m):
    s = Solver().load(m)
    r = s.solve(HPRQP_parameters(verbose=False, problem_type="QAP"))
    s.close()
    return r


@pytest.mark.parametrize("precision", ["fp64", "fp32_polish"])
def test_qap_batch_matches_single_solves(precision):
    ms = family()
    batch = solve_batch(ms, HPRQP_parameters(verbose=False, problem_type="QAP", precision=precision))
    for m, rb in zip(ms, batch):
        rs = single(m)
        assert rs.status == "OPTIMAL"
        assert rb.status == "OPTIMAL", (rb.status, rb.iter, rb.residuals)
        assert rb.residuals < 1e-6
        tol = 1e-6 if precision == "fp64" else 1e-5
        assert abs(rb.primal_obj - rs.primal_obj) / (1 + abs(rs.primal_obj)) < tol, (rb.primal_obj, rs.primal_obj)
        assert abs(rb.lambda_max_Q - rs.lambda_max_Q) <= 1e-3 * rs.lambda_max_Q
        if precision == "fp64":  # same arithmetic up to summation order: the same trajectory
            assert abs(rb.iter - rs.iter) <= max(30, 0.1 * rs.iter), (rb.iter, rs.iter)
            assert abs(rb.lambda_max_A - rs.lambda_max_A) <= 1e-8 * rs.lambda_max_A
            assert np.max(np.abs(rb.x - rs.x)) < 1e-3, np.max(np.abs(rb.x - rs.x))


def test_qap_batch_rejects_mixed_families():
    with pytest.raises(ValueError):
        solve_batch([W.qap_instance(6, 1), W.small_lasso()])
