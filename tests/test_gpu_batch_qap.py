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


C4_SIZES = (30, 64, 100, 128)  # the batch configuration's range of n_k, up to the tensor-core tile


def c4_family():
    return [W.qap_instance(n, 4 + n) for n in C4_SIZES]


def qap_numpy(m, X):
    """Qmap! (src/Q_operators/QAP_operator.jl:52-75) in FP64 numpy."""
    q = m.Q
    return 2.0 * (q.A @ X @ q.B - q.S @ X - X @ q.T)


@pytest.mark.parametrize("precision", ["fp64", "fp32_polish"])
def test_batch_qap_operator_matches_fp64_product(precision):
    """The batch's Q operator on the C4 sizes against an FP64 product: the
    FP64 engine's CUDA-core GEMMs to rounding, the FP32 phase's fused
    3xTF32 tensor-core kernel (k_qap_tc) to FP32 accuracy (one TF32 pass
    would be ~1e-3 off)."""
    from hprqp_b200.batch import BatchSolver
    ms = c4_family()
    rng = np.random.default_rng(11)
    Xs = [rng.uniform(0.0, 1.0, (int(round(np.sqrt(m.n))),) * 2) for m in ms]
    X = np.concatenate([x.ravel(order="F") for x in Xs])
    bs = BatchSolver(ms)
    Y, tc = bs.qap_apply(X, precision)
    bs.close()
    assert tc == (precision == "fp32_polish")
    off = 0
    for m, x in zip(ms, Xs):
        n = x.shape[0]
        y = Y[off:off + n * n].reshape(n, n, order="F")
        off += n * n
        ref = qap_numpy(m, x)
        err = np.max(np.abs(y - ref)) / np.max(np.abs(ref))
        assert err < (1e-13 if precision == "fp64" else 2e-6), (n, precision, err)


def test_c4_size_batch_matches_oracle():
    """Instances of the batch configuration's sizes solved together match the
    oracle's single FP64 solves: status, objective to 1e-6, iteration count
    within the residual cadence (the batch's products sum in another order)."""
    from oracle import oracle as O
    from tests.test_gpu_parity import oracle_params
    ms = c4_family()
    batch = solve_batch(ms, HPRQP_parameters(verbose=False, problem_type="QAP"))
    for m, rb in zip(ms, batch):
        ref = O.solve(m, oracle_params("QAP", max_iter=100000), threads=8)
        assert ref.status_name == "OPTIMAL" and rb.status == "OPTIMAL" and rb.residuals < 1e-6
        assert abs(rb.primal_obj - ref.primal_obj) / (1 + abs(ref.primal_obj)) < 1e-6, (rb.primal_obj, ref.primal_obj)
        assert abs(rb.iter - ref.iter) <= 100, (rb.iter, ref.iter)


def test_single_instance_qap_matches_oracle():
    """The single-instance QAP operator (FP64: the library's CUDA-core GEMM,
    no cuBLAS) gives the oracle's first 50 iterates and its full solve."""
    from oracle import oracle as O
    from tests.test_gpu_parity import ITER_RTOL, oracle_params, rel
    m = W.qap_instance(64, 68)
    ref0 = O.solve(m, oracle_params("QAP", max_iter=1))
    kw = dict(max_iter=50, lambda_max_A_override=ref0.lambda_max_A, lambda_max_Q_override=ref0.lambda_max_Q)
    ref = O.solve(m, oracle_params("QAP", **kw), trace_iters=50)
    s = Solver().load(m)
    xt, yt, wt = s.set_trace(50)
    s.solve(HPRQP_parameters(verbose=False, problem_type="QAP", **kw))
    s.set_trace(0)
    full = s.solve(HPRQP_parameters(verbose=False, problem_type="QAP", max_iter=100000))
    s.close()
    for k in range(50):
        assert rel(xt[k], ref.x_trace[k]) < ITER_RTOL and rel(yt[k], ref.y_trace[k]) < ITER_RTOL
    reff = O.solve(m, oracle_params("QAP", max_iter=100000), threads=8)
    assert full.status == reff.status_name == "OPTIMAL"
    assert full.iter == reff.iter, (full.iter, reff.iter)
    assert abs(full.primal_obj - reff.primal_obj) / (1 + abs(reff.primal_obj)) < 1e-6
