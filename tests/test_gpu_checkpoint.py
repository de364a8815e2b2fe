"""GPU tests of the auto-save checkpoint (params.auto_save; the reference's
save_state_to_hdf5!, src/algorithm.jl:183-301, written to the library's
container) and of hprqp_solve_resume, through the C ABI:

 - the last checkpoint of a solve holds the reference's datasets: its
   current/x_org, y_org, w_org are the returned solution, its best/ record
   is no worse than current/, its parameters/ are the call's;
 - a solve stopped by max_iter and continued from its checkpoint takes the
   same steps as the uninterrupted solve: the same iteration count and the
   same solution, bit for bit, in plain FP64 and from the FP32 phase of
   FP32 + polish;
 - a checkpoint of another problem, or of a finished solve, is refused.
"""
import numpy as np
import pytest

from hprqp_b200 import HPRQP_parameters, Solver
from hprqp_b200 import workloads as W
from hprqp_b200._lib import HPRQPError
from hprqp_b200.checkpoint import read_checkpoint

pytestmark = pytest.mark.gpu


def params(**kw):
    p = HPRQP_parameters(verbose=False)
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def test_last_checkpoint_holds_the_result(tmp_path):
    m = W.random_qp()
    path = str(tmp_path / "run.ckpt")
    rng = np.random.default_rng(5)
    x0 = rng.uniform(-1, 1, m.n)
    s = Solver().load(m)
    r = s.solve(params(auto_save=True, save_filename=path, initial_x=x0, stoptol=1e-6))
    s.close()
    ck = read_checkpoint(path)
    assert r.status == "OPTIMAL"
    assert int(ck["current/iteration"][0]) == r.iter
    assert np.array_equal(ck["current/x_org"], r.x)
    assert np.array_equal(ck["current/y_org"], r.y)
    assert np.array_equal(ck["current/w_org"], r.w)
    assert ck["current/KKTx_and_gap"][0] == r.residuals
    assert ck["best/KKTx_and_gap"][0] <= ck["current/KKTx_and_gap"][0]
    assert int(ck["best/iteration"][0]) <= r.iter
    assert ck["parameters/stoptol"][0] == 1e-6 and ck["parameters/problem_type"] == "QP"
    assert np.array_equal(ck["parameters/initial_x"], x0)
    assert int(ck["resume/status"][0]) == 0  # OPTIMAL


@pytest.mark.parametrize("precision,stop", [("fp64", 300), ("fp32_polish", 200)])
def test_resumed_solve_takes_the_same_steps(tmp_path, precision, stop):
    m = W.random_qp()
    s = Solver().load(m)
    full = s.solve(params(precision=precision))
    path = str(tmp_path / f"{precision}.ckpt")
    part = s.solve(params(precision=precision, max_iter=stop, auto_save=True, save_filename=path))
    assert part.status == "MAX_ITER" and part.iter == stop < full.iter
    ck = read_checkpoint(path)
    assert int(ck["resume/iter"][0]) == stop
    if precision == "fp32_polish":
        assert int(ck["resume/phase"][0]) == 32 and full.iter_fp32 > stop
    res = s.resume(params(precision=precision), path)
    s.close()
    assert res.status == full.status == "OPTIMAL"
    assert res.iter == full.iter, (res.iter, full.iter)
    assert res.restarts == full.restarts
    assert np.array_equal(res.x, full.x) and np.array_equal(res.y, full.y)
    assert res.primal_obj == full.primal_obj


def test_resume_refuses_foreign_or_finished_checkpoints(tmp_path):
    m = W.random_qp()
    path = str(tmp_path / "done.ckpt")
    s = Solver().load(m)
    s.solve(params(auto_save=True, save_filename=path))  # ends OPTIMAL
    with pytest.raises(HPRQPError):
        s.resume(params(), path)
    part = str(tmp_path / "part.ckpt")
    s.solve(params(max_iter=100, auto_save=True, save_filename=part))
    s.close()
    other = Solver().load(W.random_qp(seed=2))
    with pytest.raises(HPRQPError):
        other.resume(params(), part)
    with pytest.raises(HPRQPError):  # the scaling must be the checkpoint's
        s2 = Solver().load(m)
        try:
            s2.resume(params(use_Ruiz_scaling=False), part)
        finally:
            s2.close()
    other.close()
