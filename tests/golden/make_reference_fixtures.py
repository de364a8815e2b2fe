"""Regenerate tests/golden/reference_fixtures.npz from the reference's own
test data files (data/AUG2D.mps, data/AUG3DCQP.mps, data/esc64a.mat of the
reference tree) and the oracle's solves of them.

The reference's test suite solves exactly these files (test/runtests.jl:
AUG2D at :254-280 and :704-745, AUG3DCQP at :747-788 under every SpMV mode,
esc64a at :467-506 as a QAP with its own S, T).  The data files cannot travel
with this repository's tests, so this script stores what the tests need:

  <name>/...   the parsed problem: CSC arrays of Q and A and the vectors
               (MPS files, read by tests/mps.py the way the reference's
               read_mps does), or the dense A, B, S, T of the QAP file;
  <name>/ref   the oracle's FP64 solve at the reference test's parameters:
               [status, iter, primal_obj, lambda_max_A, lambda_max_Q,
                restarts, residuals];
  <name>/sigma, <name>/inner
               the oracle's sigma and Halpern inner counter of every
               iteration of that solve (restart iterations are where
               inner == 0), for the restart / sigma trace tests.

    HPRQP_REFERENCE_DATA=<reference>/data python tests/golden/make_reference_fixtures.py
"""
import os
import sys

import numpy as np
import scipy.io as sio

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from hprqp_b200._abi import default_params  # noqa: E402
from hprqp_b200.model import build_from_ABST, build_from_QAbc  # noqa: E402
from oracle import oracle as O  # noqa: E402
from tests.mps import read_mps  # noqa: E402

DATA = os.environ.get("HPRQP_REFERENCE_DATA", "/root/reference/data")
OUT = os.path.join(HERE, "reference_fixtures.npz")


def csc_parts(prefix, M, out):
    M = M.tocsc()
    M.sort_indices()
    out[prefix + "/shape"] = np.array(M.shape, dtype=np.int64)
    out[prefix + "/indptr"] = M.indptr.astype(np.int32)
    out[prefix + "/indices"] = M.indices.astype(np.int32)
    out[prefix + "/data"] = M.data.astype(np.float64)


def params(ptype, max_iter):
    p = default_params()
    p.verbose = 0
    p.problem_type = ptype
    p.max_iter = max_iter
    return p


def record(name, model, ptype, max_iter, out):
    r = O.solve(model, params(ptype, max_iter))  # 1 thread: the reference summation order
    t = O.solve(model, params(ptype, max_iter), trace_iters=int(r.iter))
    assert t.iter == r.iter and t.primal_obj == r.primal_obj
    out[name + "/ref"] = np.array([r.status, r.iter, r.primal_obj, r.lambda_max_A, r.lambda_max_Q, r.restarts,
                                   r.residuals], dtype=np.float64)
    out[name + "/sigma"] = t.sigma_trace
    out[name + "/inner"] = t.inner_trace
    print(name, r.status_name, r.iter, r.primal_obj, "restarts", r.restarts)


def main():
    out = {}
    for name in ("AUG3DCQP", "AUG2D"):
        Q, c, A, AL, AU, l, u = read_mps(os.path.join(DATA, name + ".mps"))
        csc_parts(name + "/Q", Q, out)
        csc_parts(name + "/A", A, out)
        for k, v in (("c", c), ("AL", AL), ("AU", AU), ("l", l), ("u", u)):
            out[name + "/" + k] = np.asarray(v, dtype=np.float64)
        model = build_from_QAbc(Q, c, A, AL, AU, l, u, verbose=False)
        record(name, model, 0, 50000, out)
    d = sio.loadmat(os.path.join(DATA, "esc64a.mat"))
    for k in "ABST":
        out["esc64a/" + k] = np.asarray(d[k], dtype=np.float64)
    model = build_from_ABST(d["A"], d["B"], d["S"], d["T"], verbose=False)
    record("esc64a", model, 2, 100000, out)
    np.savez_compressed(OUT, **out)
    print("wrote", OUT, os.path.getsize(OUT), "bytes")


if __name__ == "__main__":
    main()
