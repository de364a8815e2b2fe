"""ctypes binding of the CPU oracle (oracle/hprqp_oracle.cpp).

TEST INFRASTRUCTURE: imported only by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg, as the checker / the timed reference-CPU-path
restatement.  The product (hprqp_b200/) never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from hprqp_b200._abi import Params, ProblemView, Result, STATUS_NAMES, default_params

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "_build", "libhprqp_oracle.so")
_lib = None


def build():
    """Compile the oracle with its Makefile (g++, OpenMP)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_SO):
            build()
        L = C.CDLL(_SO)
        L.oracle_solve.restype = C.c_int
        L.oracle_solve.argtypes = [
            C.c_void_p, C.POINTER(Params), C.c_void_p, C.c_void_p, C.POINTER(Result),
            C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
            C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32]
        L.oracle_last_error.restype = C.c_char_p
        L.oracle_set_scalar_trace.restype = None
        L.oracle_set_scalar_trace.argtypes = [C.c_void_p, C.c_void_p]
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data


class OracleResult(dict):
    __getattr__ = dict.__getitem__


def solve(model, params: Params | None = None, initial_x=None, initial_y=None,
          trace_iters: int = 0, threads: int = 1) -> OracleResult:
    """Run the oracle on a hprqp_b200.model.QP_info; returns the result
    fields, the unscaled x, y, z, w and (optionally) the scaled x/y/w trace."""
    L = lib()
    if params is None:
        params = default_params()
        params.verbose = 0
    view = ProblemView(model)
    n, m = model.n, model.m
    x = np.zeros(n)
    y = np.zeros(m)
    z = np.zeros(n)
    w = np.zeros(n)
    xt = np.zeros((trace_iters, n)) if trace_iters else None
    yt = np.zeros((trace_iters, m)) if trace_iters else None
    wt = np.zeros((trace_iters, n)) if trace_iters else None
    x0 = None if initial_x is None else np.ascontiguousarray(initial_x, dtype=np.float64)
    y0 = None if initial_y is None else np.ascontiguousarray(initial_y, dtype=np.float64)
    st = (np.zeros(trace_iters), np.zeros(trace_iters, dtype=np.int64)) if trace_iters else (None, None)
    L.oracle_set_scalar_trace(_p(st[0]), _p(st[1]))
    res = Result()
    rc = L.oracle_solve(C.addressof(view.struct), C.byref(params), _p(x0), _p(y0),
                        C.byref(res), _p(x), _p(y), _p(z), _p(w),
                        trace_iters, _p(xt), _p(yt), _p(wt), threads)
    if rc != 0:
        raise RuntimeError(f"oracle_solve failed ({rc}): {L.oracle_last_error().decode()}")
    out = OracleResult({f: getattr(res, f) for f, _ in Result._fields_})
    out["status_name"] = STATUS_NAMES[res.status]
    out.update(x=x, y=y, z=z, w=w, x_trace=xt, y_trace=yt, w_trace=wt, sigma_trace=st[0], inner_trace=st[1])
    return out
