"""GPU tests of the power method (src/utils.jl:1335-1461).

The engine runs both chains (A A' and Q, or the LASSO operator) on two
streams, 32 steps per CUDA graph: the A A' chain on the Gram matrix A'A
where that is small, both chains folded once per 32-step chunk.  Its
lambda_max estimates must agree with the oracle's power method (same start
vector, same stopping rule, FP64), with the engine's reference-form chains
(two products per step, HPRQP_POWER_GRAM=0; a fold per step,
HPRQP_POWER_CHUNK_FOLD=0), and with the opt-in persistent cooperative
kernel (HPRQP_POWER_PERSISTENT=1)."""
import json
import os
import subprocess
import sys

import pytest

from hprqp_b200 import HPRQP_parameters, Solver
from hprqp_b200 import workloads as W
from oracle import oracle as O
from tests.test_gpu_parity import oracle_params

pytestmark = pytest.mark.gpu

LAM_RTOL = 1e-8  # same iteration from the same start vector in FP64

CASES = {
    "random_qp_n2000": (W.random_qp, "QP"),
    "random_lp": (W.random_lp, "QP"),
    "lasso": (W.small_lasso, "LASSO"),
    "grid_60x60": (lambda: W.grid_qp(N=60), "QP"),
}


def gpu_lambdas(name, precision="fp64"):
    fn, ptype = CASES[name]
    s = Solver(0).load(fn())
    r = s.solve(HPRQP_parameters(verbose=False, problem_type=ptype, max_iter=0, precision=precision))
    s.close()
    return r.lambda_max_A, r.lambda_max_Q


@pytest.mark.parametrize("name", list(CASES))
def test_power_method_matches_oracle(name):
    fn, ptype = CASES[name]
    ref = O.solve(fn(), oracle_params(ptype, max_iter=0))
    lamA, lamQ = gpu_lambdas(name)
    for got, want in ((lamA, ref.lambda_max_A), (lamQ, ref.lambda_max_Q)):
        assert abs(got - want) <= LAM_RTOL * max(abs(want), 1e-300), (name, got, want)


@pytest.mark.parametrize("name", list(CASES))
def test_power_method_fp32_within_method_tolerance(name):
    fn, ptype = CASES[name]
    ref = O.solve(fn(), oracle_params(ptype, max_iter=0))
    lamA, lamQ = gpu_lambdas(name, precision="fp32_polish")
    for got, want in ((lamA, ref.lambda_max_A), (lamQ, ref.lambda_max_Q)):
        assert abs(got - want) <= 1e-3 * max(abs(want), 1e-300), (name, got, want)


def test_persistent_kernel_matches_launch_chain():
    code = ("import json; from tests.test_gpu_power import gpu_lambdas, CASES; "
            "print(json.dumps({k: gpu_lambdas(k) for k in CASES}))")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = {}
    for flag in ("1", "0"):
        env = dict(os.environ, HPRQP_POWER_PERSISTENT=flag)
        r = subprocess.run([sys.executable, "-c", code], cwd=root, env=env, capture_output=True, text=True,
                           timeout=600)
        assert r.returncode == 0, r.stderr[-2000:]
        out[flag] = json.loads(r.stdout.strip().splitlines()[-1])
    for k in CASES:
        for a, b in zip(out["1"][k], out["0"][k]):
            assert abs(a - b) <= 1e-10 * max(abs(b), 1e-300), (k, a, b)


def _lambdas_with_env(env_over, precision):
    code = ("import json; from hprqp_b200 import HPRQP_parameters, Solver; from tests.test_gpu_power import CASES\n"
            "out = {}\n"
            "for k, (fn, pt) in CASES.items():\n"
            "    s = Solver(0).load(fn())\n"
            f"    r = s.solve(HPRQP_parameters(verbose=False, problem_type=pt, max_iter=0, precision='{precision}'))\n"
            "    s.close()\n"
            "    out[k] = [r.lambda_max_A, r.power_iter_A, r.lambda_max_Q, r.power_iter_Q]\n"
            "print(json.dumps(out))")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = dict(os.environ, **env_over)
    r = subprocess.run([sys.executable, "-c", code], cwd=root, env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return json.loads(r.stdout.strip().splitlines()[-1])


@pytest.mark.parametrize("precision,rtol", [("fp64", 1e-10), ("fp32_polish", 1e-6)])
def test_gram_chain_matches_two_product_chain(precision, rtol):
    """The A A' chain on the Gram matrix A'A (forced on every case) runs the
    reference's iteration in n-space: same stopping step and the same lambda
    to rounding as the chain of two products per step."""
    on = _lambdas_with_env({"HPRQP_POWER_GRAM": "1"}, precision)
    off = _lambdas_with_env({"HPRQP_POWER_GRAM": "0"}, precision)
    for k in CASES:
        lam1, it1, lq1, iq1 = on[k]
        lam0, it0, lq0, iq0 = off[k]
        assert it1 == it0, (k, it1, it0)
        assert abs(lam1 - lam0) <= rtol * max(abs(lam0), 1e-300), (k, lam1, lam0)
        # the Q chain is the same code either way (its row schedule is
        # autotuned per process, so only to rounding)
        assert iq1 == iq0, (k, iq1, iq0)
        assert abs(lq1 - lq0) <= rtol * max(abs(lq0), 1e-300), (k, lq1, lq0)


@pytest.mark.parametrize("precision,rtol", [("fp64", 1e-10), ("fp32_polish", 1e-5)])
def test_chunk_fold_matches_per_step_fold(precision, rtol):
    """The chains folded once per 32-step chunk (unnormalised FP64 states,
    scale-invariant formulas) stop at the per-step fold's step with the same
    lambda to rounding.  In FP32 the per-step Q chain keeps an FP32 state,
    the chunk-fold one an FP64 state: the stop may move by a step or two."""
    on = _lambdas_with_env({"HPRQP_POWER_CHUNK_FOLD": "1"}, precision)
    off = _lambdas_with_env({"HPRQP_POWER_CHUNK_FOLD": "0"}, precision)
    for k in CASES:
        lam1, it1, lq1, iq1 = on[k]
        lam0, it0, lq0, iq0 = off[k]
        slack = 0 if precision == "fp64" else max(2, it0 // 100)
        assert abs(it1 - it0) <= slack and abs(iq1 - iq0) <= max(slack, 0 if precision == "fp64" else 2 + iq0 // 100), \
            (k, it1, it0, iq1, iq0)
        assert abs(lam1 - lam0) <= rtol * max(abs(lam0), 1e-300), (k, lam1, lam0)
        assert abs(lq1 - lq0) <= rtol * max(abs(lq0), 1e-300), (k, lq1, lq0)


def _huge_lambda_qp():
    """A QP whose Q has lambda_max ~ 4e11 with scaling off: an unnormalised
    chain leaves FP64 range within a 32-step chunk (4e11^32 > 1e308)."""
    import numpy as np
    import scipy.sparse as sp
    from hprqp_b200 import build_from_QAbc
    n, m = 3000, 500
    rng = np.random.default_rng(5)
    T = sp.diags([2.0 * np.ones(n), -np.ones(n - 1), -np.ones(n - 1)], [0, 1, -1])
    Q = (1e11 * T).tocsc()
    A = sp.random(m, n, density=0.002, random_state=6, format="csc")
    return build_from_QAbc(Q, rng.standard_normal(n), A, -np.ones(m), np.ones(m), -np.ones(n), np.ones(n),
                           verbose=False)


def test_chunk_fold_falls_back_when_a_state_leaves_fp64_range():
    code = ("import json; from hprqp_b200 import HPRQP_parameters, Solver; "
            "from tests.test_gpu_power import _huge_lambda_qp\n"
            "s = Solver(0).load(_huge_lambda_qp())\n"
            "r = s.solve(HPRQP_parameters(verbose=False, max_iter=0, use_Ruiz_scaling=False, "
            "use_Pock_Chambolle_scaling=False))\n"
            "s.close()\n"
            "print(json.dumps([r.lambda_max_Q, r.power_iter_Q, r.lambda_max_A, r.power_iter_A]))")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = {}
    for flag in ("1", "0"):
        env = dict(os.environ, HPRQP_POWER_CHUNK_FOLD=flag)
        r = subprocess.run([sys.executable, "-c", code], cwd=root, env=env, capture_output=True, text=True,
                           timeout=600)
        assert r.returncode == 0, r.stderr[-2000:]
        out[flag] = json.loads(r.stdout.strip().splitlines()[-1])
    lq1, iq1, la1, ia1 = out["1"]
    lq0, iq0, la0, ia0 = out["0"]
    assert lq0 > 1e11 and abs(lq1 - lq0) <= 1e-10 * lq0 and iq1 == iq0, (out["1"], out["0"])
    assert abs(la1 - la0) <= 1e-10 * abs(la0) and ia1 == ia0


def test_chunk_fold_with_a_larger_reduction_grid():
    """HPRQP_REDUCE_CAP above the default puts more CTAs, hence more per-CTA
    sums, into every chunk-fold step: the same steps and lambda to rounding."""
    big = _lambdas_with_env({"HPRQP_REDUCE_CAP": "4736"}, "fp64")
    ref = _lambdas_with_env({}, "fp64")
    for k in CASES:
        lam1, it1, lq1, iq1 = big[k]
        lam0, it0, lq0, iq0 = ref[k]
        assert it1 == it0 and iq1 == iq0, (k, big[k], ref[k])
        assert abs(lam1 - lam0) <= 1e-10 * abs(lam0) and abs(lq1 - lq0) <= 1e-10 * max(abs(lq0), 1e-300), k
