"""GPU test of hprqp_power_lambda_noalloc, the entry point for callers that
cannot allocate device memory where they need lambda_max(A A'): it works in
memory the caller already owns plus scratch reserved inside the library.

The test (not the entry point) allocates the device arrays with torch, then
calls the entry point twice in a row through the C ABI and checks both
results against the lambda_max_A that hprqp_solve reports for the same
matrix (scaling off, eig_factor 1, the same CSR schedule), within the 1e-10
relative tolerance of the iterate-parity tests.  This file is collected last
so that a run stopping at the first failure has run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from hprqp_b200 import HPRQP_parameters, Solver
from hprqp_b200 import workloads as W
from hprqp_b200._lib import HPRQPError, check, load

pytestmark = pytest.mark.gpu

RTOL = 1e-10


def _device_csr(M, torch):
    M = M.tocsr()
    M.sort_indices()
    return (torch.tensor(M.indptr.astype(np.int32), device="cuda"),
            torch.tensor(M.indices.astype(np.int32), device="cuda"),
            torch.tensor(M.data.astype(np.float64), device="cuda"))


def test_power_lambda_noalloc_matches_solver():
    torch = pytest.importorskip("torch")
    model = W.random_qp()
    m, n = model.m, model.n
    s = Solver(0).load(model)
    ref = s.solve(HPRQP_parameters(verbose=False, use_Ruiz_scaling=False, use_Pock_Chambolle_scaling=False,
                                   eig_factor=1.0, spmv_mode_A=1, max_iter=0))
    s.close()
    A = _device_csr(model.A, torch)
    AT = _device_csr(model.A.T, torch)
    L = load()
    stream = torch.cuda.current_stream().cuda_stream
    out = []
    for _ in range(2):
        lam, its = C.c_double(), C.c_int32()
        check(L.hprqp_power_lambda_noalloc(m, n, *[t.data_ptr() for t in A], *[t.data_ptr() for t in AT],
                                           1, 1e-4, 5000, stream, C.byref(lam), C.byref(its)))
        out.append((lam.value, its.value))
    torch.cuda.synchronize()
    for lam, its in out:
        assert 0 < its <= 5000
        assert abs(lam - ref.lambda_max_A) <= RTOL * abs(ref.lambda_max_A), (lam, ref.lambda_max_A)
    assert out[0] == out[1]


def test_power_lambda_noalloc_rejects_oversize():
    L = load()
    lam, its = C.c_double(), C.c_int32()
    m = n = 1 << 20
    dummy = C.c_void_p(8)  # never dereferenced: the size check comes first
    rc = L.hprqp_power_lambda_noalloc(m, n, dummy, dummy, dummy, dummy, dummy, dummy, 1, 1e-4, 10, None,
                                      C.byref(lam), C.byref(its))
    assert rc == -1
    assert b"too large" in L.hprqp_last_error(None)
    with pytest.raises(HPRQPError):
        check(rc)
