"""GPU tests of the sparse formats and the tensor-core GEMM:

 - every pinned row schedule (ELL, SELL-32, CSR with 1 and 4 threads per
   row) gives the oracle's first 50 iterates to 1e-10 (a format that cannot
   hold a matrix falls back to CSR);
 - the 3xTF32 tcgen05 GEMM of the FP32 QAP operator matches an FP64 numpy
   product to FP32 accuracy (a single TF32 pass would be ~1e-3 off), for
   sizes below, at and across its 128 x 128 tile, with alpha and beta;
 - an FP32+polish QAP solve through that GEMM reaches the FP64 optimum."""
import ctypes as C

import numpy as np
import pytest

from hprqp_b200 import HPRQP_parameters, Solver
from hprqp_b200 import workloads as W
from hprqp_b200._lib import load
from oracle import oracle as O
from tests.test_gpu_parity import ITER_RTOL, gpu_params, oracle_params, rel

pytestmark = pytest.mark.gpu

MODELS = {
    "grid_60x60": (lambda: W.grid_qp(N=60), "QP"),
    "random_qp_n2000": (W.random_qp, "QP"),
    "lasso": (W.small_lasso, "LASSO"),
}


@pytest.mark.parametrize("mode", ["ell", "sell", 1, 4])
@pytest.mark.parametrize("name", list(MODELS))
def test_pinned_schedule_iterates_match_oracle(name, mode):
    fn, ptype = MODELS[name]
    m = fn()
    ref0 = O.solve(m, oracle_params(ptype, max_iter=1))
    lamA = ref0.lambda_max_A if m.m else -1.0
    lamQ = ref0.lambda_max_Q if (ref0.lambda_max_Q > 0 and not ref0.Q_is_diag) else -1.0
    kw = dict(max_iter=50, lambda_max_A_override=lamA, lambda_max_Q_override=lamQ)
    ref = O.solve(m, oracle_params(ptype, **kw), trace_iters=50)
    s = Solver().load(m)
    xt, yt, wt = s.set_trace(50)
    s.solve(gpu_params(ptype, spmv_mode_Q=mode, spmv_mode_A=mode, **kw))
    s.close()
    for k in range(50):
        assert rel(xt[k], ref.x_trace[k]) < ITER_RTOL, (name, mode, "x", k)
        assert rel(wt[k], ref.w_trace[k]) < ITER_RTOL, (name, mode, "w", k)
        if m.m:
            assert rel(yt[k], ref.y_trace[k]) < ITER_RTOL, (name, mode, "y", k)


def _gemm(n, alpha, A, B, beta, C0):
    torch = pytest.importorskip("torch")
    dA = torch.tensor(A.astype(np.float32).ravel(order="F"), device="cuda")
    dB = torch.tensor(B.astype(np.float32).ravel(order="F"), device="cuda")
    dC = torch.tensor(C0.astype(np.float32).ravel(order="F"), device="cuda")
    L = load()
    rc = L.hprqp_gemm_3xtf32(n, C.c_float(alpha), dA.data_ptr(), dB.data_ptr(), C.c_float(beta), dC.data_ptr(),
                             C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == 0
    return dC.cpu().numpy().astype(np.float64).reshape((n, n), order="F")


@pytest.mark.parametrize("n", [10, 37, 128, 130, 257])
@pytest.mark.parametrize("alpha,beta", [(1.0, 0.0), (-2.0, 1.0)])
def test_gemm_3xtf32_fp32_accuracy(n, alpha, beta):
    rng = np.random.default_rng(n)
    A = rng.standard_normal((n, n)).astype(np.float32).astype(np.float64)
    B = rng.standard_normal((n, n)).astype(np.float32).astype(np.float64)
    C0 = rng.standard_normal((n, n)).astype(np.float32).astype(np.float64)
    got = _gemm(n, alpha, A, B, beta, C0)
    want = alpha * (A @ B) + beta * C0
    err = np.max(np.abs(got - want)) / np.max(np.abs(want))
    # FP32 accumulation over n terms; one TF32 pass (10-bit mantissa) would
    # be ~1e-3 off
    assert err < 2e-6 * max(1.0, np.sqrt(n / 16)), (n, err)


def test_qap_fp32_polish_reaches_fp64_optimum():
    m = W.qap_instance(16, 3)
    s = Solver().load(m)
    r64 = s.solve(HPRQP_parameters(verbose=False, problem_type="QAP"))
    r32 = s.solve(HPRQP_parameters(verbose=False, problem_type="QAP", precision="fp32_polish"))
    s.close()
    assert r64.status == r32.status == "OPTIMAL"
    assert r32.iter_fp32 > 0
    assert abs(r32.primal_obj - r64.primal_obj) / (1 + abs(r64.primal_obj)) < 1e-5
