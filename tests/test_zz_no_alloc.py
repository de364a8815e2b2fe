"""GPU test of hprqp_power_lambda_noalloc, the entry point for callers that
cannot allocate device memory where they need lambda_max(A A'): programs
whose device memory belongs to another framework's pool allocator, and loops
that must not allocate after start-up.  It works in memory the caller
already owns plus scratch reserved inside the library.

The test (not the entry point) allocates the device arrays with torch, then
calls the entry point twice in a row through the C ABI and checks both
results against the lambda_max_A and the power-step count that hprqp_solve
reports for the same matrix (scaling off, eig_factor 1, the same CSR
schedule), within the 1e-10 relative tolerance of the iterate-parity tests.
Two more cases check a run cut off by max_iter and a problem exactly at the
scratch capacity against a numpy power iteration of the same steps.  This
file is collected last so that a run stopping at the first failure has run
every other test.
"""
import ctypes as C

import numpy as np
import pytest
import scipy.sparse as sp

from hprqp_b200 import HPRQP_parameters, Solver
from hprqp_b200 import workloads as W
from hprqp_b200._lib import check, load

pytestmark = pytest.mark.gpu

RTOL = 1e-10
CAP = 1 << 20  # 2m + n limit of the library's fixed scratch


def _device_csr(M, torch):
    M = M.tocsr()
    M.sort_indices()
    return (torch.tensor(M.indptr.astype(np.int32), device="cuda"),
            torch.tensor(M.indices.astype(np.int32), device="cuda"),
            torch.tensor(M.data.astype(np.float64), device="cuda"))


def _start_vector(length):
    """The power method's start vector: element i from outputs 2i and 2i+1 of
    the splitmix64 stream seeded with 1, through Box-Muller, plus 1e-8."""
    def mix(k):
        v = np.uint64(1) + (k + np.uint64(1)) * np.uint64(0x9E3779B97F4A7C15)
        v = (v ^ (v >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        v = (v ^ (v >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return v ^ (v >> np.uint64(31))
    i = np.arange(length, dtype=np.uint64)
    with np.errstate(over="ignore"):
        u1 = ((mix(2 * i) >> np.uint64(11)).astype(np.float64) + 1.0) * 2.0 ** -53
        u2 = (mix(2 * i + np.uint64(1)) >> np.uint64(11)).astype(np.float64) * 2.0 ** -53
    return np.sqrt(-2.0 * np.log(u1)) * np.cos(6.283185307179586 * u2) + 1e-8


def _numpy_power(A, steps, tol):
    """power_iteration_A (src/utils.jl:1335-1385) for at most `steps` steps."""
    A = A.tocsr()
    AT = A.T.tocsr()
    z = _start_vector(A.shape[0])
    lam = 1.0
    for k in range(steps):
        q = z / np.linalg.norm(z)
        z = A @ (AT @ q)
        lam = q @ z
        if np.linalg.norm(z - lam * q) / (np.linalg.norm(z) + lam) < tol:
            return lam, k + 1
    return lam, steps


def _call(L, A, AT, m, n, tpr, tol, max_iter, stream):
    lam, its = C.c_double(), C.c_int32()
    check(L.hprqp_power_lambda_noalloc(m, n, *[t.data_ptr() for t in A], *[t.data_ptr() for t in AT],
                                       tpr, tol, max_iter, stream, C.byref(lam), C.byref(its)))
    return lam.value, its.value


@pytest.mark.parametrize("tpr", [1, 4, 32])
def test_power_lambda_noalloc_matches_solver(tpr):
    torch = pytest.importorskip("torch")
    model = W.random_qp()
    m, n = model.m, model.n
    s = Solver(0).load(model)
    ref = s.solve(HPRQP_parameters(verbose=False, use_Ruiz_scaling=False, use_Pock_Chambolle_scaling=False,
                                   eig_factor=1.0, spmv_mode_A=tpr, max_iter=0))
    s.close()
    A = _device_csr(model.A, torch)
    AT = _device_csr(model.A.T, torch)
    L = load()
    stream = torch.cuda.current_stream().cuda_stream
    out = [_call(L, A, AT, m, n, tpr, 1e-4, 5000, stream) for _ in range(2)]
    torch.cuda.synchronize()
    for lam, its in out:
        assert its == ref.power_iter_A, (its, ref.power_iter_A)
        assert abs(lam - ref.lambda_max_A) <= RTOL * abs(ref.lambda_max_A), (lam, ref.lambda_max_A)
    assert out[0] == out[1]


def test_power_lambda_noalloc_stops_at_max_iter():
    torch = pytest.importorskip("torch")
    model = W.random_qp()
    A = _device_csr(model.A, torch)
    AT = _device_csr(model.A.T, torch)
    lam_ref, its_ref = _numpy_power(model.A, 7, 1e-14)
    assert its_ref == 7
    L = load()
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(2):
        lam, its = _call(L, A, AT, model.m, model.n, 1, 1e-14, 7, stream)
        assert its == 7
        assert abs(lam - lam_ref) <= RTOL * abs(lam_ref), (lam, lam_ref)


def test_power_lambda_noalloc_at_capacity():
    torch = pytest.importorskip("torch")
    m, n = CAP // 4, CAP // 2  # 2m + n == CAP exactly
    rng = np.random.default_rng(7)
    A = sp.random(m, n, density=4.0 / n, random_state=rng, format="csr")
    A.data = rng.standard_normal(A.nnz)
    lam_ref, its_ref = _numpy_power(A, 40, 1e-4)
    dA = _device_csr(A, torch)
    dAT = _device_csr(A.T, torch)
    L = load()
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(2):
        lam, its = _call(L, dA, dAT, m, n, 2, 1e-4, 40, stream)
        assert its == its_ref
        assert abs(lam - lam_ref) <= RTOL * abs(lam_ref), (lam, lam_ref)
