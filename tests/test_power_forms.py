"""CPU check of the algebra behind the engine's power method.

The engine runs the reference's power iteration (src/utils.jl:1335-1461)
in a reordered form: the A A' chain in n-space on the Gram matrix G = A'A,
and both chains unnormalised between 32-step folds, with lambda and the
residual taken from scale-invariant sums (hprqp_b200/csrc/kernels.cuh,
EpiGramRaw / EpiPowRaw / pow_chunk_log).  This test restates those
formulas in numpy, FP64, and checks that they stop at the reference
form's step with its lambda to rounding."""
import numpy as np
import scipy.sparse as sp

from hprqp_b200 import workloads as W

TOL, MAXIT, CHUNK = 1e-4, 5000, 32


def reference_A(A, z):  # power_iteration_A as the reference writes it
    for i in range(MAXIT):
        q = z / np.linalg.norm(z)
        z = A @ (A.T @ q)
        lam = q @ z
        if np.linalg.norm(z - lam * q) / (np.linalg.norm(z) + lam) < TOL:
            return lam, i + 1
    return lam, MAXIT


def reference_Q(Q, z):  # power_iteration_Q
    for i in range(MAXIT):
        q = z / np.linalg.norm(z)
        z = Q @ q
        lam = q @ z
        if np.linalg.norm(z - lam * q) / (np.linalg.norm(z) + lam) < TOL:
            return lam, i + 1
    return lam, MAXIT


def gram_chunked(A, z):
    G = (A.T @ A).tocsr()
    u = A.T @ z / np.linalg.norm(z)  # w_0, normalised: s_0 = 1
    k = 0
    while k < MAXIT:
        tot = []
        for _ in range(CHUNK):  # steps write only their sums: a = u_k.u_{k+1}, b = u_k.u_k
            un = G @ u
            tot.append((u @ un, u @ u))
            u = un
        s2 = 1.0
        for j, (a, b) in enumerate(tot):
            lam, zz = s2 * b, s2 * a
            s2 = 1.0 / a
            if np.sqrt(max(zz - lam * lam, 0.0)) / (np.sqrt(zz) + lam) < TOL:
                return lam, k + j + 1
        u = u * np.sqrt(s2)  # renormalise: the next chunk starts at s = 1
        k += CHUNK
    return lam, MAXIT


def q_chunked(Q, z):
    y = z.copy()
    k = 0
    while k < MAXIT:
        tot = []
        for _ in range(CHUNK):  # a = y_k.y_{k+1}, b = y_k.y_k, c = y_{k+1}.y_{k+1}
            v = Q @ y
            tot.append((y @ v, y @ y, v @ v))
            y = v
        for j, (a, b, c) in enumerate(tot):
            lam, zz = a / b, c / b
            if np.sqrt(max(zz - lam * lam, 0.0)) / (np.sqrt(zz) + lam) < TOL:
                return lam, k + j + 1
        y = y / np.sqrt(tot[-1][2])
        k += CHUNK
    return lam, MAXIT


def test_reordered_power_iteration_matches_the_reference_form():
    for model in (W.grid_qp(N=40), W.random_qp(n=600, m=300, seed=7)):
        A = sp.csr_matrix(model.A)
        Q = sp.csr_matrix(model.Q.Q)
        rng = np.random.default_rng(1)
        za = rng.standard_normal(A.shape[0]) + 1e-8
        zq = rng.standard_normal(Q.shape[0]) + 1e-8
        la, ia = reference_A(A, za.copy())
        lg, ig = gram_chunked(A, za.copy())
        assert ig == ia and abs(lg - la) <= 1e-10 * la, (ia, ig, la, lg)
        lq, iq = reference_Q(Q, zq.copy())
        lc, ic = q_chunked(Q, zq.copy())
        assert ic == iq and abs(lc - lq) <= 1e-10 * lq, (iq, ic, lq, lc)
