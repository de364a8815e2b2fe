"""GPU tests of the staged column-block schedule (spmv_mode 10, k_stage_pass):
the input vector's column blocks in shared memory, 16-bit block-local
columns in 8-entry chunks, warps over row windows with a segmented scan,
and, with several column blocks, per-row block sums folded in block order
by the last block to arrive.

 - a QP whose Q (40,000 columns, ~20 entries a row: two blocks in FP64,
   one in FP32) and A run staged: the first 50 iterates match the oracle to
   1e-10, and the passes report the staged schedule;
 - a wide LASSO (400 x 60,000, lognormal rows with some longer than 256
   entries per block, i.e. single-row windows; three column blocks in FP64,
   two in FP32): the first 50 iterates match the oracle to 1e-10; full
   solves in FP64 and FP32 + polish give the oracle's status, iteration
   count (FP64) and objective;
 - two solves give bit-identical solutions (the fold does not depend on
   which block arrives last);
 - a QP built for the layout's edge cases (rows whose entries all sit in
   the first or in the last column block, so that they are empty in the
   others; rows of more than 32 chunks in every block; a last block
   narrower than the others): the first 50 iterates match the oracle to
   1e-10 with A pinned to the staged schedule.
"""
import numpy as np
import pytest

import scipy.sparse as sp

from hprqp_b200 import Solver, build_from_QAbc
from hprqp_b200 import workloads as W
from oracle import oracle as O
from tests.test_gpu_parity import ITER_RTOL, OBJ_RTOL, gpu_params, oracle_params, rel

pytestmark = pytest.mark.gpu

STAGED = -4  # the schedule code the pass statistics report
_cache = {}


def qp():
    if "qp" not in _cache:
        _cache["qp"] = W.random_qp(n=40000, m=3000, seed=21, density_A=0.002, b_rows=500, density_B=0.001)
    return _cache["qp"]


def wide_lasso():
    if "lasso" not in _cache:
        _cache["lasso"] = W.lasso(m=400, n=60000, seed=33, mu=5.0)
    return _cache["lasso"]


def _iterates(m, ptype, **pins):
    ref0 = O.solve(m, oracle_params(ptype, max_iter=1))
    lamA = ref0.lambda_max_A if m.m else -1.0
    lamQ = ref0.lambda_max_Q if (ref0.lambda_max_Q > 0 and not ref0.Q_is_diag) else -1.0
    kw = dict(max_iter=50, lambda_max_A_override=lamA, lambda_max_Q_override=lamQ)
    ref = O.solve(m, oracle_params(ptype, **kw), trace_iters=50)
    s = Solver().load(m)
    xt, yt, wt = s.set_trace(50)
    s.solve(gpu_params(ptype, **pins, **kw))
    s.set_trace(0)
    stats = s.profile_iterations(gpu_params(ptype, **pins), iters=3)
    s.close()
    return ref, xt, yt, wt, stats


def test_qp_staged_iterates_match_oracle():
    m = qp()
    ref, xt, yt, wt, stats = _iterates(m, "QP", spmv_mode_Q="staged", spmv_mode_A="staged")
    sched = {p["name"]: p["threads_per_row"] for p in stats["passes"]}
    assert sched["zxw1 Q*w"] == STAGED and sched["tempv Q*w_bar"] == STAGED, sched
    assert sched["y A*tempv"] == STAGED, sched
    for k in range(50):
        assert rel(xt[k], ref.x_trace[k]) < ITER_RTOL, ("x", k, rel(xt[k], ref.x_trace[k]))
        assert rel(yt[k], ref.y_trace[k]) < ITER_RTOL, ("y", k)
        assert rel(wt[k], ref.w_trace[k]) < ITER_RTOL, ("w", k)


def test_wide_lasso_has_long_block_rows():
    A = wide_lasso().Q.A.tocsr()
    lens = np.diff(A.indptr)
    # a row longer than 3 x 256 entries has more than 32 chunks in some block
    assert lens.max() > 3 * 256 and A.shape[1] * 8 > 2 * 200 * 1024


def test_wide_lasso_staged_iterates_match_oracle():
    ref, xt, _, wt, stats = _iterates(wide_lasso(), "LASSO", spmv_mode_Q="staged")
    sched = {p["name"]: p["threads_per_row"] for p in stats["passes"]}
    assert sched["lasso1 A_d*w"] == STAGED, sched
    for k in range(50):
        assert rel(xt[k], ref.x_trace[k]) < ITER_RTOL, ("x", k, rel(xt[k], ref.x_trace[k]))
        assert rel(wt[k], ref.w_trace[k]) < ITER_RTOL, ("w", k)


def test_wide_lasso_staged_full_solve_matches_oracle():
    m = wide_lasso()
    ref = O.solve(m, oracle_params("LASSO", max_iter=50000))
    s = Solver().load(m)
    r = s.solve(gpu_params("LASSO", max_iter=50000, spmv_mode_Q="staged"))
    r32 = s.solve(gpu_params("LASSO", max_iter=50000, spmv_mode_Q="staged", precision="fp32_polish"))
    again = s.solve(gpu_params("LASSO", max_iter=50000, spmv_mode_Q="staged"))
    s.close()
    assert ref.status_name == "OPTIMAL"
    assert r.status == "OPTIMAL" and r.residuals < 1e-6
    assert r.iter == ref.iter, (r.iter, ref.iter)
    assert abs(r.primal_obj - ref.primal_obj) / (1 + abs(ref.primal_obj)) < OBJ_RTOL
    assert r32.status == "OPTIMAL" and r32.residuals < 1e-6 and r32.iter_fp32 > 0
    assert abs(r32.primal_obj - ref.primal_obj) / (1 + abs(ref.primal_obj)) < 1e-5
    assert again.iter == r.iter and np.array_equal(again.x, r.x)


def edge_qp():
    """n = 61,001 (three FP64 column blocks of 20,336 columns, the last one
    20,329; two in FP32), m = 2,000 rows of A: 10% with every entry among
    the last 15,000 columns, 10% among the first 500, 20 rows of 800 entries
    (about 34 chunks in each block), the rest 30 entries; Q diagonal plus a
    sparse low-rank term; bounds around a point."""
    rng = np.random.default_rng(77)
    n, m = 61001, 2000
    rows, cols = [], []
    for r in range(m):
        if r % 10 == 0:
            c = n - 1 - rng.choice(15000, 30, replace=False)
        elif r % 10 == 1:
            c = rng.choice(500, 30, replace=False)
        elif r < 40 and r % 2 == 0:
            c = rng.choice(n, 800, replace=False)
        else:
            c = rng.choice(n, 30, replace=False)
        rows += [r] * len(c)
        cols += list(c)
    A = sp.csr_matrix((rng.standard_normal(len(rows)), (rows, cols)), shape=(m, n))
    A.sum_duplicates()
    Bm = sp.random(200, n, density=2e-4, random_state=5, format="csr")
    Q = (Bm.T @ Bm + sp.diags(rng.uniform(0.1, 1.0, n))).tocsc()
    Q = (0.5 * (Q + Q.T)).tocsc()
    x0 = rng.uniform(-1, 1, n)
    Ax0 = A @ x0
    return build_from_QAbc(Q, rng.standard_normal(n), A.tocsc(), Ax0 - rng.uniform(0, 1, m),
                           Ax0 + rng.uniform(0, 1, m), -5.0 * np.ones(n), 5.0 * np.ones(n), verbose=False)


def test_edge_layout_qp_staged_iterates_match_oracle():
    m = edge_qp()
    ref, xt, yt, wt, stats = _iterates(m, "QP", spmv_mode_A="staged", spmv_mode_Q=1)
    sched = {p["name"]: p["threads_per_row"] for p in stats["passes"]}
    assert sched["y A*tempv"] == STAGED, sched
    for k in range(50):
        assert rel(xt[k], ref.x_trace[k]) < ITER_RTOL, ("x", k, rel(xt[k], ref.x_trace[k]))
        assert rel(yt[k], ref.y_trace[k]) < ITER_RTOL, ("y", k)
        assert rel(wt[k], ref.w_trace[k]) < ITER_RTOL, ("w", k)
