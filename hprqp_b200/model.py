"""Problem model and builders: the Python mirror of the reference's
QP_info_cpu (src/structs.jl:98-149), its Q-operator plug-ins
(src/Q_operators/*.jl) and the build_from_* entry points (src/utils.jl).

These run on the host in front of the C-ABI boundary, as the Julia builders
do in front of `solve`; the solver itself is libhprqp.so (see api.py).
"""
from __future__ import annotations

import warnings
from dataclasses import dataclass, field

import numpy as np
import scipy.sparse as sp

from ._abi import Q_CUSTOM, Q_LASSO, Q_QAP, Q_SPARSE


# ---------------------------------------------------------------------------
# Q operators (src/Q_operators/Q_operator_interface.jl:1-140)
# ---------------------------------------------------------------------------
class AbstractQOperatorCPU:
    """Plug-in contract of src/Q_operators/Q_operator_interface.jl.  The
    library implements the built-in operators natively; a Python-side Qmap
    is provided for checks and for users of the reference interface."""

    kind: int = -1

    def get_problem_size(self) -> int:
        raise NotImplementedError

    def get_temp_size(self) -> int:
        raise NotImplementedError

    @classmethod
    def get_operator_name(cls) -> str:
        raise NotImplementedError

    def Qmap(self, x: np.ndarray) -> np.ndarray:
        raise NotImplementedError


@dataclass
class CustomQ(AbstractQOperatorCPU):
    """A user's Q operator on the GPU: the Python side of the library's
    device-callback operator (hprqp_set_qmap; the reference's custom
    AbstractQOperator with its own Qmap!, src/Q_operators/
    Q_operator_interface.jl:33-92).

    `device_qmap(x_ptr, qx_ptr, precision, stream_ptr)` computes Qx = Q x
    for n-vectors in device memory (float64 when precision == 0, float32
    when 1) and enqueues its work on the CUDA stream `stream_ptr`; it must
    not change x, and it returns 0 (or raises / returns nonzero to stop the
    solve).  `host_qmap(x)` (optional) is the same product on numpy arrays,
    for checks on the host."""
    n_vars: int
    device_qmap: object
    host_qmap: object = None
    name: str = "Custom"
    kind: int = Q_CUSTOM

    def get_problem_size(self):
        return self.n_vars

    def get_temp_size(self):
        return 0

    def get_operator_name(self):
        return self.name

    def Qmap(self, x):
        if self.host_qmap is None:
            raise NotImplementedError("this custom operator has no host Qmap")
        return self.host_qmap(x)


@dataclass
class SparseQ(AbstractQOperatorCPU):
    """Explicit sparse Q (src/Q_operators/sparse_matrix_operator.jl)."""
    Q: sp.csc_matrix
    kind: int = Q_SPARSE

    def get_problem_size(self):
        return self.Q.shape[0]

    def get_temp_size(self):
        return 0

    @classmethod
    def get_operator_name(cls):
        return "SparseMatrix"

    def Qmap(self, x):
        return self.Q @ x


@dataclass
class LASSO_Q_operator_cpu(AbstractQOperatorCPU):
    """Q(x) = A'(A x) (src/Q_operators/LASSO_operator.jl:46-52,112-117)."""
    A: sp.csc_matrix
    kind: int = Q_LASSO

    def get_problem_size(self):
        return self.A.shape[1]

    def get_temp_size(self):
        return self.A.shape[0]

    @classmethod
    def get_operator_name(cls):
        return "LASSO"

    def Qmap(self, x):
        return self.A.T @ (self.A @ x)


@dataclass
class QAP_Q_operator_cpu(AbstractQOperatorCPU):
    """Q(X) = 2(A X B - S X - X T) on vec(X), column-major
    (src/Q_operators/QAP_operator.jl:12-20,65-75)."""
    A: np.ndarray
    B: np.ndarray
    S: np.ndarray
    T: np.ndarray
    kind: int = Q_QAP

    @property
    def n(self):
        return self.A.shape[0]

    def get_problem_size(self):
        return self.n ** 2

    def get_temp_size(self):
        return self.n ** 2

    @classmethod
    def get_operator_name(cls):
        return "QAP"

    def Qmap(self, x):
        n = self.n
        X = x.reshape(n, n, order="F")
        QX = 2.0 * (self.A @ X @ self.B) - 2.0 * (self.S @ X) - 2.0 * (X @ self.T)
        return QX.reshape(-1, order="F")


@dataclass
class QP_info:
    """QP_info_cpu (src/structs.jl:98-149)."""
    Q: AbstractQOperatorCPU
    c: np.ndarray
    A: sp.csc_matrix
    AL: np.ndarray
    AU: np.ndarray
    l: np.ndarray
    u: np.ndarray
    obj_constant: float = 0.0
    lambda_: float = 0.0
    meta: dict = field(default_factory=dict)

    @property
    def n(self):
        return len(self.c)

    @property
    def m(self):
        return self.A.shape[0]

    @property
    def AT(self):
        return self.A.T.tocsc()


# ---------------------------------------------------------------------------
# qp_formulation (src/utils.jl:67-188)
# ---------------------------------------------------------------------------
def qp_formulation(Q, c, A, AL, AU, l, u, c0=0.0, verbose=True) -> QP_info:
    """Validate and preprocess a QP like the reference qp_formulation:
    dimension/bound/NaN checks (errors), Q symmetrisation with a warning,
    and deletion of rows of A that are all zero or free on both sides."""
    Q = sp.csc_matrix(Q, dtype=np.float64)
    A = sp.csc_matrix(A, dtype=np.float64)
    c = np.asarray(c, dtype=np.float64).ravel().copy()
    AL = np.asarray(AL, dtype=np.float64).ravel().copy()
    AU = np.asarray(AU, dtype=np.float64).ravel().copy()
    l = np.asarray(l, dtype=np.float64).ravel().copy()
    u = np.asarray(u, dtype=np.float64).ravel().copy()
    mQ, nQ = Q.shape
    if mQ != nQ:
        raise ValueError(f"Q matrix must be square. Got size ({mQ}, {nQ}).")
    n = nQ
    if Q.nnz > 0:
        diff = abs(Q - Q.T)
        dev = diff.max() if diff.nnz else 0.0
        if dev > 1e-10:
            warnings.warn(f"Q matrix is not symmetric (max deviation: {dev}). "
                          "Symmetrizing Q = 0.5*(Q + Q').")
            Q = (0.5 * (Q + Q.T)).tocsc()
            Q.eliminate_zeros()
    if len(c) != n:
        raise ValueError(f"Dimension mismatch: Q is {n}x{n} but c has length {len(c)}.")
    if len(l) != n:
        raise ValueError(f"Dimension mismatch: Q is {n}x{n} but l has length {len(l)}.")
    if len(u) != n:
        raise ValueError(f"Dimension mismatch: Q is {n}x{n} but u has length {len(u)}.")
    mA, nA = A.shape
    if nA != n:
        raise ValueError(f"Dimension mismatch: Q is {n}x{n} but A has {nA} columns.")
    if len(AL) != mA:
        raise ValueError(f"Dimension mismatch: A has {mA} rows but AL has length {len(AL)}.")
    if len(AU) != mA:
        raise ValueError(f"Dimension mismatch: A has {mA} rows but AU has length {len(AU)}.")
    bad = np.nonzero(l > u)[0]
    if len(bad):
        raise ValueError(f"Infeasible variable bounds: l > u at indices: {bad[:5].tolist()}")
    bad = np.nonzero(AL > AU)[0]
    if len(bad):
        raise ValueError(f"Infeasible constraint bounds: AL > AU at rows: {bad[:5].tolist()}")
    if not np.all(np.isfinite(Q.data)):
        raise ValueError("Q matrix contains NaN or Inf values.")
    if not np.all(np.isfinite(c)):
        raise ValueError("c vector contains NaN or Inf values.")
    if not np.all(np.isfinite(A.data)):
        raise ValueError("A matrix contains NaN or Inf values.")
    if np.any(np.isnan(AL)) or np.any(np.isnan(AU)):
        raise ValueError("Constraint bounds AL or AU contain NaN values.")
    if np.any(np.isnan(l)) or np.any(np.isnan(u)):
        raise ValueError("Variable bounds l or u contain NaN values.")
    # Remove rows of A that are all zeros, or free on both sides (utils.jl:162-172)
    if mA > 0:
        rowsum = np.asarray(abs(A).sum(axis=1)).ravel()
        drop = (rowsum == 0) | ((AL == -np.inf) & (AU == np.inf))
        if drop.any():
            keep = np.nonzero(~drop)[0]
            A = A.tocsr()[keep, :].tocsc()
            AL, AU = AL[keep], AU[keep]
            if verbose:
                print(f"Deleted {int(drop.sum())} rows of A that are all zeros.")
    A.sort_indices()
    Q.sort_indices()
    return QP_info(SparseQ(Q), c, A, AL, AU, l, u, float(c0), 0.0)


def build_from_QAbc(Q, c, A, AL, AU, l, u, obj_constant=0.0, verbose=True) -> QP_info:
    """build_from_QAbc (src/utils.jl:970-1014).  Dense or sparse Q and A."""
    if isinstance(Q, np.ndarray):
        Q = sp.csc_matrix(Q)
    if isinstance(A, np.ndarray):
        A = sp.csc_matrix(A)
    return qp_formulation(Q, c, A, AL, AU, l, u, obj_constant, verbose=verbose)


def build_from_Ab_lambda(A, b, lam, verbose=True) -> QP_info:
    """build_from_Ab_lambda (src/utils.jl:1222-1267):
    min 0.5||Ax-b||^2 + lam||x||_1 as a QP with the operator Q = A'A,
    c = -A'b, obj_constant = 0.5||b||^2, no constraints, x free."""
    A = sp.csc_matrix(A, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64).ravel()
    m, n = A.shape
    if len(b) != m:
        raise ValueError("Length of b must match number of rows in A")
    if not lam > 0:
        raise ValueError("Lambda must be positive")
    c = -(A.T @ b)
    obj_constant = 0.5 * float(np.linalg.norm(b)) ** 2
    A.sort_indices()
    return QP_info(LASSO_Q_operator_cpu(A), np.asarray(c, dtype=np.float64),
                   sp.csc_matrix((0, n)), np.zeros(0), np.zeros(0),
                   -np.inf * np.ones(n), np.inf * np.ones(n), obj_constant, float(lam))


def build_from_ABST(A, B, S, T, verbose=True) -> QP_info:
    """build_from_ABST (src/utils.jl:1133-1180): QAP relaxation with
    doubly-stochastic constraints X e = e, X' e = e, X >= 0, c = 0."""
    A, B, S, T = (np.asarray(M, dtype=np.float64) for M in (A, B, S, T))
    n = A.shape[0]
    for M in (A, B, S, T):
        if M.shape != (n, n):
            raise ValueError("A, B, S, T must be square and of the same size")
    e = np.ones((1, n))
    I = sp.identity(n, format="csc")
    Acon = sp.vstack([sp.kron(e, I), sp.kron(I, e)]).tocsc()
    Acon.sort_indices()
    return QP_info(QAP_Q_operator_cpu(A, B, S, T), np.zeros(n * n), Acon,
                   np.ones(2 * n), np.ones(2 * n), np.zeros(n * n),
                   np.full(n * n, np.inf), 0.0, 0.0)
