"""GPU tests of the custom Q operator (a device callback bound with
hprqp_set_qmap; the reference's user-defined AbstractQOperator with its own
Qmap!, src/Q_operators/Q_operator_interface.jl:33-92), through the C ABI.

The user's operator here is sparse Q applied by torch (cuSPARSE) on the
library's stream, through raw device pointers: the kind of code a user
would bind.  With scaling off (an operator Q is never scaled,
src/utils.jl:364-406) and lambda_max injected, the custom-operator solve
reproduces the built-in sparse-Q path's first 50 iterates to 1e-10; its
own power method on the callback gives the built-in lambda_max(Q); FP32 +
polish calls it in FP32 and reaches the FP64 optimum; a callback error
stops the solve with HPRQP_E_CALLBACK, and a problem without a bound
operator is a state error.
"""
import ctypes as C

import pytest

from hprqp_b200 import HPRQP_parameters, Solver
from hprqp_b200 import workloads as W
from hprqp_b200._abi import HPRQP_E_CALLBACK, HPRQP_E_STATE, ProblemView
from hprqp_b200._lib import HPRQPError, check
from hprqp_b200.model import CustomQ, QP_info
from tests.test_gpu_parity import ITER_RTOL, rel

pytestmark = pytest.mark.gpu


class _DevArray:
    """A raw device pointer as a 1-D array (__cuda_array_interface__)."""

    def __init__(self, ptr, n, typestr):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": typestr, "data": (int(ptr), False),
                                         "version": 3, "strides": None, "stream": None}


def torch_sparse_op(Q, calls):
    """A user operator: Q x by torch's sparse CSR product, on the stream the
    library passes, in the precision it asks for."""
    torch = pytest.importorskip("torch")
    Q = Q.tocsr()
    Q.sort_indices()
    n = Q.shape[0]
    mats = {}
    for prec, dt in ((0, torch.float64), (1, torch.float32)):
        mats[prec] = torch.sparse_csr_tensor(torch.tensor(Q.indptr, dtype=torch.int64),
                                             torch.tensor(Q.indices, dtype=torch.int64),
                                             torch.tensor(Q.data, dtype=dt), size=(n, n),
                                             check_invariants=True).to("cuda")

    def device_qmap(x, qx, precision, stream):
        calls[precision] = calls.get(precision, 0) + 1
        ts = "<f8" if precision == 0 else "<f4"
        with torch.cuda.stream(torch.cuda.ExternalStream(stream)):
            xv = torch.as_tensor(_DevArray(x, n, ts), device="cuda")
            yv = torch.as_tensor(_DevArray(qx, n, ts), device="cuda")
            yv.copy_(torch.mv(mats[precision], xv))
        return 0

    return CustomQ(n_vars=n, device_qmap=device_qmap, host_qmap=lambda v: Q @ v, name="torch-sparse")


def custom_model(m, op):
    return QP_info(op, m.c, m.A, m.AL, m.AU, m.l, m.u, m.obj_constant, 0.0)


NOSCALE = dict(use_Ruiz_scaling=False, use_Pock_Chambolle_scaling=False)


def params(**kw):
    p = HPRQP_parameters(verbose=False, **NOSCALE)
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def test_custom_operator_reproduces_builtin_sparse_iterates():
    m = W.random_qp()
    s = Solver().load(m)
    ref0 = s.solve(params(max_iter=0))
    kw = dict(max_iter=50, lambda_max_A_override=ref0.lambda_max_A, lambda_max_Q_override=ref0.lambda_max_Q)
    tr = s.set_trace(50)
    s.solve(params(**kw))
    xb, yb, wb = (a.copy() for a in tr)
    s.close()
    calls = {}
    c = Solver().load(custom_model(m, torch_sparse_op(m.Q.Q, calls)))
    xt, yt, wt = c.set_trace(50)
    r = c.solve(params(**kw))
    c.set_trace(0)
    c.close()
    assert r.status == "MAX_ITER" and calls.get(0, 0) >= 100  # two products per iteration
    for k in range(50):
        assert rel(xt[k], xb[k]) < ITER_RTOL, (k, rel(xt[k], xb[k]))
        assert rel(yt[k], yb[k]) < ITER_RTOL
        assert rel(wt[k], wb[k]) < ITER_RTOL


def test_custom_operator_power_method_and_full_solves():
    m = W.random_qp()
    s = Solver().load(m)
    ref = s.solve(params(max_iter=50000))
    s.close()
    calls = {}
    c = Solver().load(custom_model(m, torch_sparse_op(m.Q.Q, calls)))
    r64 = c.solve(params(max_iter=50000))
    r32 = c.solve(params(max_iter=50000, precision="fp32_polish"))
    c.close()
    assert abs(r64.lambda_max_Q - ref.lambda_max_Q) <= 1e-8 * ref.lambda_max_Q, (r64.lambda_max_Q, ref.lambda_max_Q)
    assert ref.status == r64.status == r32.status == "OPTIMAL"
    assert abs(r64.primal_obj - ref.primal_obj) / (1 + abs(ref.primal_obj)) < 1e-6
    assert abs(r32.primal_obj - ref.primal_obj) / (1 + abs(ref.primal_obj)) < 1e-5
    assert r32.iter_fp32 > 0 and calls.get(1, 0) > 0  # the FP32 phase called it in FP32


def test_custom_operator_error_stops_the_solve():
    m = W.toy_qp()

    def failing(x, qx, precision, stream):
        return 7

    c = Solver().load(custom_model(m, CustomQ(n_vars=m.n, device_qmap=failing)))
    with pytest.raises(HPRQPError) as ei:
        c.solve(params(max_iter=10, lambda_max_Q_override=1.0))
    assert ei.value.code == HPRQP_E_CALLBACK
    c.close()


def test_custom_problem_needs_a_bound_operator():
    m = W.toy_qp()
    cm = custom_model(m, CustomQ(n_vars=m.n, device_qmap=lambda *a: 0))
    s = Solver()
    view = ProblemView(cm)
    check(s._L.hprqp_load(s.h, C.addressof(view.struct)), s.h)  # loaded, no hprqp_set_qmap
    s.model = cm
    with pytest.raises(HPRQPError) as ei:
        s.solve(params(max_iter=5))
    assert ei.value.code == HPRQP_E_STATE
    s.close()
