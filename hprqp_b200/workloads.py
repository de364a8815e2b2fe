"""Seeded synthetic workloads with the shapes, sizes and value
distributions of the benchmark configurations, plus the small problems the
reference's own tests solve (test/runtests.jl).  No dataset is bundled: the
reference's public-benchmark inputs (Maros-Meszaros, QAPLIB, E2006) are
replaced by these generators.

  random_qp      n=2,000, m=1,000 random sparse convex QP
  grid_qp        700x700 grid QP, n=490,000, m=974,408, nnz(A)=2.92M
  lasso          20,000 x 150,000 LASSO, lognormal row lengths, nnz~1.1e7
  qap_batch      256 convexified QAP relaxations, n ~ U{30..128}
  lasso_family   2,000 x 10,000 LASSO family (fixed pattern, perturbed values)
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp

from .model import build_from_ABST, build_from_Ab_lambda, build_from_QAbc, QP_info


def _sprandn(rng, m, n, density):
    nnz = int(round(density * m * n))
    idx = rng.choice(m * n, size=nnz, replace=False)
    rows, cols = idx % m, idx // m
    vals = rng.standard_normal(nnz)
    return sp.csc_matrix((vals, (rows, cols)), shape=(m, n))


def random_qp(n=2000, m=1000, seed=1, density_A=0.005, b_rows=500, density_B=0.002,
              verbose=False) -> QP_info:
    """Random sparse convex QP: A sprandn (density 0.5%); Q = B'B + 1e-2 I with
    B 500 x n at 0.2%; c ~ N(0,1); x0 ~ U(-1,1); AL/AU = A x0 -/+ U(0,1);
    l = -10, u = 10."""
    rng = np.random.default_rng(seed)
    A = _sprandn(rng, m, n, density_A)
    B = _sprandn(rng, b_rows, n, density_B)
    Q = (B.T @ B + 1e-2 * sp.identity(n)).tocsc()
    Q = (0.5 * (Q + Q.T)).tocsc()
    c = rng.standard_normal(n)
    x0 = rng.uniform(-1, 1, n)
    Ax0 = A @ x0
    AL = Ax0 - rng.uniform(0, 1, m)
    AU = Ax0 + rng.uniform(0, 1, m)
    l = -10.0 * np.ones(n)
    u = 10.0 * np.ones(n)
    return build_from_QAbc(Q, c, A, AL, AU, l, u, verbose=verbose)


def grid_qp(N=700, seed=2, verbose=False) -> QP_info:
    """Grid QP on an N x N grid, p = i*N + j.  Q = 5-point Laplacian
    (Dirichlet) + diag U(0.1,1).  For each interior node two rows with three
    +-1 entries: x_p - x_{p+e_i} + x_{p-e_j} and x_p - x_{p+e_j} + x_{p-e_i};
    AL = -1, AU = 1; c ~ N(0,1); 0 <= x <= 5."""
    rng = np.random.default_rng(seed)
    n = N * N
    ii, jj = np.meshgrid(np.arange(N), np.arange(N), indexing="ij")
    p = (ii * N + jj).ravel()
    i, j = ii.ravel(), jj.ravel()
    rows = [p]
    cols = [p]
    vals = [4.0 + rng.uniform(0.1, 1.0, n)]
    for di, dj in ((1, 0), (-1, 0), (0, 1), (0, -1)):
        ok = (i + di >= 0) & (i + di < N) & (j + dj >= 0) & (j + dj < N)
        rows.append(p[ok])
        cols.append(((i + di) * N + (j + dj))[ok])
        vals.append(-np.ones(ok.sum()))
    Q = sp.csc_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                      shape=(n, n))
    inter = (i >= 1) & (i <= N - 2) & (j >= 1) & (j <= N - 2)
    pi, ii_, jj_ = p[inter], i[inter], j[inter]
    k = len(pi)
    r = np.arange(2 * k)
    c1 = np.stack([pi, (ii_ + 1) * N + jj_, ii_ * N + (jj_ - 1)], axis=1)
    c2 = np.stack([pi, ii_ * N + (jj_ + 1), (ii_ - 1) * N + jj_], axis=1)
    acols = np.concatenate([c1, c2], axis=0)          # rows 0..k-1 then k..2k-1
    order = np.empty(2 * k, dtype=np.int64)
    order[0::2] = np.arange(k)                         # interleave r1, r2 per node
    order[1::2] = np.arange(k, 2 * k)
    acols = acols[order]
    arows = np.repeat(r, 3)
    avals = np.tile([1.0, -1.0, 1.0], 2 * k)
    A = sp.csc_matrix((avals, (arows, acols.ravel())), shape=(2 * k, n))
    c = rng.standard_normal(n)
    m = 2 * k
    return build_from_QAbc(Q, c, A, -np.ones(m), np.ones(m), np.zeros(n), 5.0 * np.ones(n),
                           verbose=verbose)


def lasso(m=20000, n=150000, seed=3, mu=6.0, sig=0.8, lam_frac=1e-3, xstar_density=0.005,
          verbose=False) -> QP_info:
    """LASSO with lognormal(mu, sig) row lengths, uniform columns (duplicates
    merged), lognormal(0,1) values, rows scaled to unit l2 norm;
    b = A x* + 0.01 N(0,1) with x* 0.5% sparse N(0,1); lambda = 1e-3 ||A'b||_inf."""
    rng = np.random.default_rng(seed)
    lens = np.clip(np.round(rng.lognormal(mu, sig, m)), 1, n).astype(np.int64)
    rows = np.repeat(np.arange(m), lens)
    cols = rng.integers(0, n, size=lens.sum())
    vals = rng.lognormal(0.0, 1.0, size=lens.sum())
    A = sp.csr_matrix((vals, (rows, cols)), shape=(m, n))
    A.sum_duplicates()
    rn = np.sqrt(np.asarray(A.multiply(A).sum(axis=1)).ravel())
    rn[rn == 0] = 1.0
    A = sp.diags(1.0 / rn) @ A
    xs = np.zeros(n)
    k = max(1, int(round(xstar_density * n)))
    xs[rng.choice(n, k, replace=False)] = rng.standard_normal(k)
    b = A @ xs + 0.01 * rng.standard_normal(m)
    lam = lam_frac * np.abs(A.T @ b).max()
    model = build_from_Ab_lambda(A.tocsc(), b, lam, verbose=verbose)
    model.meta.update(b=b, x_star=xs)
    return model


def qap_instance(n, seed) -> QP_info:
    """Convexified QAP relaxation: F, D symmetric, zero diagonal, integers
    U{0..10}; A := F, B := D; S = T = (mu/2) I with mu the smallest product of
    extreme eigenvalues of F and D (<= 0), so Q = 2(D kron F - mu I) is PSD."""
    rng = np.random.default_rng(seed)

    def symint():
        M = rng.integers(0, 11, size=(n, n)).astype(np.float64)
        M = np.triu(M, 1)
        return M + M.T

    F, D = symint(), symint()
    ef, ed = np.linalg.eigvalsh(F), np.linalg.eigvalsh(D)
    mu = min(ef[0] * ed[0], ef[0] * ed[-1], ef[-1] * ed[0], ef[-1] * ed[-1], 0.0)
    S = T = (mu / 2.0) * np.eye(n)
    return build_from_ABST(F, D, S, T)


def qap_batch(count=256, nmin=30, nmax=128, seed=4):
    sizes = np.random.default_rng(seed).integers(nmin, nmax + 1, size=count)
    return [qap_instance(int(sizes[k]), seed + k) for k in range(count)]


def lasso_family(count, m=2000, n=10000, density=0.01, start=0, pattern_seed=5):
    """LASSO family on a fixed sparsity pattern (seed 5); instance k perturbs
    the values by (1 + 0.05 N(0,1)) (seed 5000+k), draws a 1%-sparse x*,
    b = A x* + 0.01 N(0,1) and lambda = logU(1e-4, 1e-2) ||A'b||_inf."""
    prng = np.random.default_rng(pattern_seed)
    base = _sprandn(prng, m, n, density).tocsc()
    base.sort_indices()
    out = []
    for k in range(start, start + count):
        rng = np.random.default_rng(5000 + k)
        A = base.copy()
        A.data = A.data * (1.0 + 0.05 * rng.standard_normal(A.nnz))
        xs = np.zeros(n)
        kk = max(1, int(round(0.01 * n)))
        xs[rng.choice(n, kk, replace=False)] = rng.standard_normal(kk)
        b = A @ xs + 0.01 * rng.standard_normal(m)
        lam = np.exp(rng.uniform(np.log(1e-4), np.log(1e-2))) * np.abs(A.T @ b).max()
        model = build_from_Ab_lambda(A, b, lam, verbose=False)
        model.meta.update(b=b, x_star=xs, index=k)
        out.append(model)
    return out


# ---- small problems of the reference test-suite (test/runtests.jl) --------
def toy_qp() -> QP_info:
    """min x1^2 + x2^2 - 3x1 - 5x2  s.t. x1 + 2x2 <= 10, 3x1 + x2 <= 12, x >= 0
    (model.mps / demo/demo_QAbc.jl).  Optimum x = (1.5, 2.5), objective -8.5."""
    Q = sp.csc_matrix(np.diag([2.0, 2.0]))
    A = sp.csc_matrix(np.array([[1.0, 2.0], [3.0, 1.0]]))
    return build_from_QAbc(Q, [-3.0, -5.0], A, [-np.inf, -np.inf], [10.0, 12.0],
                           [0.0, 0.0], [np.inf, np.inf], verbose=False)


def dense_q_qp(n=10, m=5) -> QP_info:
    """test/runtests.jl:285-314: Q = 2I, c = -1, A = ones, 0 <= Ax <= n/2, 0 <= x <= 1."""
    return build_from_QAbc(2.0 * np.eye(n), -np.ones(n), np.ones((m, n)), np.zeros(m),
                           np.full(m, n / 2), np.zeros(n), np.ones(n), verbose=False)


def small_lp(n=8, m=4) -> QP_info:
    """test/runtests.jl:316-345: Q = 0, c = -1, A = ones, 2 <= Ax <= 5, 0 <= x <= 1."""
    return build_from_QAbc(np.zeros((n, n)), -np.ones(n), np.ones((m, n)), np.full(m, 2.0),
                           np.full(m, 5.0), np.zeros(n), np.ones(n), verbose=False)


def free_var_qp(n=300, m=120, seed=7) -> QP_info:
    """QP with > 80% free variables (takes the reference's noC update path,
    src/algorithm.jl:1969-1974)."""
    rng = np.random.default_rng(seed)
    B = _sprandn(rng, n // 2, n, 0.02)
    Q = (B.T @ B + 0.1 * sp.identity(n)).tocsc()
    Q = (0.5 * (Q + Q.T)).tocsc()
    A = _sprandn(rng, m, n, 0.03)
    x0 = rng.uniform(-1, 1, n)
    Ax0 = A @ x0
    l = -np.inf * np.ones(n)
    u = np.inf * np.ones(n)
    nb = n // 10
    l[:nb] = -2.0
    u[:nb] = 2.0
    return build_from_QAbc(Q, rng.standard_normal(n), A, Ax0 - rng.uniform(0, 1, m),
                           Ax0 + rng.uniform(0, 1, m), l, u, verbose=False)


def random_lp(n=60, m=30, seed=11) -> QP_info:
    """Feasible bounded random LP (Q = 0) for cross-checks against HiGHS."""
    rng = np.random.default_rng(seed)
    A = _sprandn(rng, m, n, 0.3)
    x0 = rng.uniform(0, 1, n)
    Ax0 = A @ x0
    return build_from_QAbc(sp.csc_matrix((n, n)), rng.standard_normal(n), A,
                           Ax0 - rng.uniform(0, 1, m), Ax0 + rng.uniform(0, 1, m),
                           np.zeros(n), np.full(n, 2.0), verbose=False)


def small_lasso(m=60, n=200, seed=12) -> QP_info:
    rng = np.random.default_rng(seed)
    A = _sprandn(rng, m, n, 0.1)
    xs = np.zeros(n)
    xs[rng.choice(n, 6, replace=False)] = rng.standard_normal(6)
    b = A @ xs + 0.01 * rng.standard_normal(m)
    lam = 0.05 * np.abs(A.T @ b).max()
    return build_from_Ab_lambda(A, b, lam, verbose=False)
