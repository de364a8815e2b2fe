"""CPU tests of the host-side model builders (reference qp_formulation
input validation, test/runtests.jl:18-125, and build_from_* shapes)."""
import numpy as np
import pytest
import scipy.sparse as sp

from hprqp_b200 import build_from_ABST, build_from_Ab_lambda, build_from_QAbc, qp_formulation


def valid(n=3, m=2):
    Q = sp.csc_matrix(np.diag([1.0, 2.0, 1.0])[:n, :n])
    A = sp.csc_matrix(np.array([[1.0, 1.0, 0.0], [0.0, 1.0, 1.0]])[:m, :n])
    return Q, np.zeros(n), A, -np.inf * np.ones(m), np.ones(m), np.zeros(n), np.inf * np.ones(n)


def test_valid_accepted():
    assert qp_formulation(*valid(), verbose=False) is not None


def test_non_square_q_rejected():
    Q, c, A, AL, AU, l, u = valid()
    with pytest.raises(ValueError):
        qp_formulation(sp.csc_matrix(np.ones((3, 4))), c, A, AL, AU, l, u)


def test_dimension_mismatch_rejected():
    Q, c, A, AL, AU, l, u = valid()
    with pytest.raises(ValueError):
        qp_formulation(Q, np.zeros(4), A, AL, AU, l, u)


def test_infeasible_bounds_rejected():
    Q, c, A, AL, AU, l, u = valid()
    with pytest.raises(ValueError):
        qp_formulation(Q, c, A, AL, AU, np.ones(3), np.zeros(3))


def test_nan_rejected():
    Q, c, A, AL, AU, l, u = valid()
    with pytest.raises(ValueError):
        qp_formulation(Q, np.array([np.nan, 0, 0]), A, AL, AU, l, u)


def test_empty_constraints_accepted():
    Q, c, _, _, _, l, u = valid()
    m = qp_formulation(Q, c, sp.csc_matrix((0, 3)), np.zeros(0), np.zeros(0), l, u, verbose=False)
    assert m.m == 0 and m.n == 3


def test_dense_inputs_converted():
    m = build_from_QAbc(2 * np.eye(5), np.ones(5), np.ones((3, 5)), np.zeros(3), np.full(3, 2.5), np.zeros(5),
                        np.ones(5), verbose=False)
    assert sp.issparse(m.Q.Q) and sp.issparse(m.A)


def test_empty_q_is_lp():
    m = build_from_QAbc(np.zeros((5, 5)), np.ones(5), sp.csc_matrix(np.ones((3, 5))), np.zeros(3),
                        np.full(3, 2.5), np.zeros(5), np.ones(5), verbose=False)
    assert m.Q.Q.nnz == 0


def test_zero_and_free_rows_deleted():
    A = sp.csc_matrix(np.array([[1.0, 1.0], [0.0, 0.0], [1.0, -1.0]]))
    m = build_from_QAbc(np.eye(2), np.ones(2), A, np.array([0.0, 0.0, -np.inf]), np.array([1.0, 1.0, np.inf]),
                        np.zeros(2), np.ones(2), verbose=False)
    assert m.m == 1


def test_lasso_builder():
    A = sp.random(20, 30, 0.2, random_state=1, format="csc")
    b = np.arange(20.0)
    m = build_from_Ab_lambda(A, b, 0.5, verbose=False)
    assert m.m == 0 and m.n == 30 and np.allclose(m.c, -(A.T @ b))
    assert np.isclose(m.obj_constant, 0.5 * b @ b) and m.lambda_ == 0.5
    x = np.random.default_rng(0).standard_normal(30)
    assert np.allclose(m.Q.Qmap(x), A.T @ (A @ x))


def test_qap_builder():
    n = 4
    rng = np.random.default_rng(0)
    F, D = rng.random((n, n)), rng.random((n, n))
    m = build_from_ABST(F, D, np.eye(n), np.eye(n))
    assert m.n == n * n and m.m == 2 * n
    X = rng.random((n, n))
    x = X.reshape(-1, order="F")
    assert np.allclose(m.A @ x, np.concatenate([X.sum(axis=1), X.sum(axis=0)]))
    QX = 2 * (F @ X @ D - X - X)
    assert np.allclose(m.Q.Qmap(x), QX.reshape(-1, order="F"))
