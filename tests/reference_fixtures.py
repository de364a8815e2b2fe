"""Loader of tests/golden/reference_fixtures.npz: the reference's own test
problems (data/AUG2D.mps, data/AUG3DCQP.mps, data/esc64a.mat of the
reference tree, stored by tests/golden/make_reference_fixtures.py) and the
oracle's solves of them."""
import os

import numpy as np
import scipy.sparse as sp

from hprqp_b200.model import build_from_ABST, build_from_QAbc

PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_fixtures.npz")
NAMES = ("AUG3DCQP", "AUG2D", "esc64a")
PTYPE = {"AUG3DCQP": "QP", "AUG2D": "QP", "esc64a": "QAP"}
MAX_ITER = {"AUG3DCQP": 50000, "AUG2D": 50000, "esc64a": 100000}  # the reference tests' settings
_g = None


def data():
    global _g
    if _g is None:
        _g = dict(np.load(PATH))
    return _g


def _csc(g, prefix):
    shape = tuple(int(v) for v in g[prefix + "/shape"])
    return sp.csc_matrix((g[prefix + "/data"], g[prefix + "/indices"], g[prefix + "/indptr"]), shape=shape)


def raw(name):
    """The parsed problem as stored: (Q, c, A, AL, AU, l, u) or (A, B, S, T)."""
    g = data()
    if name == "esc64a":
        return tuple(g["esc64a/" + k] for k in "ABST")
    return (_csc(g, name + "/Q"), g[name + "/c"], _csc(g, name + "/A"), g[name + "/AL"], g[name + "/AU"],
            g[name + "/l"], g[name + "/u"])


def model(name):
    """build_from_mps / build_from_mat of the reference for that file."""
    if name == "esc64a":
        return build_from_ABST(*raw(name), verbose=False)
    return build_from_QAbc(*raw(name), verbose=False)


def ref(name):
    """The oracle's FP64 solve: dict(status, iter, primal_obj, lambda_max_A,
    lambda_max_Q, restarts, residuals, sigma, inner)."""
    g = data()
    v = g[name + "/ref"]
    keys = ("status", "iter", "primal_obj", "lambda_max_A", "lambda_max_Q", "restarts", "residuals")
    out = {k: float(x) for k, x in zip(keys, v)}
    for k in ("status", "iter", "restarts"):
        out[k] = int(out[k])
    out["sigma"] = g[name + "/sigma"]
    out["inner"] = g[name + "/inner"]
    return out


def restart_iterations(inner):
    """Iterations (1-based) whose step ran right after a restart."""
    inner = np.asarray(inner)
    return [int(k) + 1 for k in np.nonzero(inner == 0)[0] if k > 0]
