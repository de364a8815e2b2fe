"""Regenerate the golden fixtures in tests/golden/ from the oracle (the C++
FP64 restatement of the reference CPU path):

  cases.npz            per small case: status, iteration count, objective,
                       unscaled x, lambda_max values, and the scaled x/y
                       iterates of the first 10 HPR iterations (lambda_max
                       injected), for the regression and GPU parity tests
  grid_qp_oracle.json  the 700x700 grid QP solved to 1e-6 by the oracle:
                       iteration count (used by bench.py to extrapolate the
                       CPU baseline), objective, lambda_max values

    python tests/golden/make_golden.py [--skip-grid]
"""
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from hprqp_b200 import workloads as W  # noqa: E402
from hprqp_b200._abi import default_params  # noqa: E402
from oracle import oracle as O  # noqa: E402

CASES = {
    "toy_diagQ": (W.toy_qp, 0),
    "dense_q": (W.dense_q_qp, 0),
    "lp": (W.small_lp, 0),
    "random_lp": (W.random_lp, 0),
    "free_var_noC": (W.free_var_qp, 0),
    "random_qp_n2000": (W.random_qp, 0),
    "lasso": (W.small_lasso, 1),
    "qap_n10": (lambda: W.qap_instance(10, 5), 2),
    "grid_60x60": (lambda: W.grid_qp(N=60), 0),
}


def params(ptype, **kw):
    p = default_params()
    p.verbose = 0
    p.problem_type = ptype
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def main():
    out = {}
    for name, (make, ptype) in CASES.items():
        m = make()
        full = O.solve(m, params(ptype, max_iter=50000))
        lamA = full.lambda_max_A if m.m else -1.0
        lamQ = full.lambda_max_Q if (full.lambda_max_Q > 0 and not full.Q_is_diag) else -1.0
        tr = O.solve(m, params(ptype, max_iter=10, lambda_max_A_override=lamA, lambda_max_Q_override=lamQ),
                     trace_iters=10)
        out[name + "/status"] = np.array(full.status)
        out[name + "/iter"] = np.array(full.iter)
        out[name + "/pobj"] = np.array(full.primal_obj)
        out[name + "/x"] = full.x
        out[name + "/lam"] = np.array([lamA, lamQ])
        out[name + "/x_trace"] = tr.x_trace
        out[name + "/y_trace"] = tr.y_trace
        print(name, full.status_name, full.iter, full.primal_obj)
    np.savez_compressed(os.path.join(HERE, "cases.npz"), **out)
    if "--skip-grid" not in sys.argv:
        m = W.grid_qp(N=700)
        t = time.time()
        r = O.solve(m, params(0), threads=os.cpu_count() or 1)
        rec = {"700": {"status": r.status_name, "iter": int(r.iter), "iter_6": int(r.iter_6),
                       "primal_obj": r.primal_obj, "lambda_max_A": r.lambda_max_A,
                       "lambda_max_Q": r.lambda_max_Q, "restarts": int(r.restarts),
                       "oracle_power_s": r.power_time, "oracle_time_s": r.time,
                       "oracle_threads": os.cpu_count(), "wall_s": time.time() - t}}
        with open(os.path.join(HERE, "grid_qp_oracle.json"), "w") as f:
            json.dump(rec, f, indent=1)
        print(rec)


if __name__ == "__main__":
    main()
