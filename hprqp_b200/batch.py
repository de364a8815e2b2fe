"""Batched solves (include/hprqp_batch.h) of a LASSO family
(build_from_Ab_lambda models) or of QAP relaxations of uneven size
(build_from_ABST models): all instances advance together, one kernel per HPR
pass over the concatenated instances, with per-instance restarts, sigma,
stopping and (optionally) the per-instance FP32 -> FP64 polish switch.

    results = solve_batch(models, HPRQP_parameters(problem_type="LASSO"))
    results = solve_batch(qap_models, HPRQP_parameters(problem_type="QAP"))
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._abi import ProblemView, Result, STATUS_NAMES

Q_LASSO, Q_QAP = 1, 2  # hprqp_problem.Q_kind (include/hprqp.h)
from ._lib import HPRQPError, load
from .api import HPRQP_parameters, HPRQP_results

_blib = None


def _lib():
    global _blib
    if _blib is None:
        L = load()
        vp = C.c_void_p
        L.hprqp_batch_create.argtypes = [C.POINTER(vp), C.c_int32]
        L.hprqp_batch_load_lasso.argtypes = [vp, C.c_int32, vp]
        L.hprqp_batch_load_qap.argtypes = [vp, C.c_int32, vp]
        L.hprqp_batch_solve.argtypes = [vp, vp, vp, vp, vp, vp]
        L.hprqp_batch_qap_apply.argtypes = [vp, C.c_int32, vp, vp, C.POINTER(C.c_int32)]
        L.hprqp_batch_qap_apply.restype = C.c_int
        L.hprqp_batch_last_error.argtypes = [vp]
        L.hprqp_batch_last_error.restype = C.c_char_p
        L.hprqp_batch_destroy.argtypes = [vp]
        for f in ("hprqp_batch_create", "hprqp_batch_load_lasso", "hprqp_batch_load_qap", "hprqp_batch_solve",
                  "hprqp_batch_destroy"):
            getattr(L, f).restype = C.c_int
        _blib = L
    return _blib


class BatchSolver:
    def __init__(self, models, device=0):
        L = _lib()
        h = C.c_void_p()
        rc = L.hprqp_batch_create(C.byref(h), device)
        if rc:
            raise HPRQPError(rc, L.hprqp_batch_last_error(None).decode())
        self.L, self.h, self.models = L, h, list(models)
        views = [ProblemView(m) for m in self.models]
        kinds = {v.struct.Q_kind for v in views}
        if len(kinds) != 1 or kinds.pop() not in (Q_LASSO, Q_QAP):
            raise ValueError("a batch is either all LASSO models or all QAP models")
        arr = (type(views[0].struct) * len(views))(*[v.struct for v in views])
        load = L.hprqp_batch_load_qap if views[0].struct.Q_kind == Q_QAP else L.hprqp_batch_load_lasso
        self._check(load(h, len(views), C.addressof(arr)))
        del views

    def _check(self, rc):
        if rc:
            raise HPRQPError(rc, self.L.hprqp_batch_last_error(self.h).decode())

    def solve(self, params: HPRQP_parameters, initial_x=None, sigma0=None):
        B = len(self.models)
        res = (Result * B)()
        xs = [np.zeros(m.n) for m in self.models]
        xptr = (C.c_void_p * B)(*[x.ctypes.data for x in xs])
        x0ptr = None
        keep = []
        if initial_x is not None:
            x0s = [None if v is None else np.ascontiguousarray(v, dtype=np.float64) for v in initial_x]
            keep += x0s
            x0ptr = (C.c_void_p * B)(*[None if v is None else v.ctypes.data for v in x0s])
        sg = None
        if sigma0 is not None:
            sg = np.ascontiguousarray(sigma0, dtype=np.float64)
        p = params.to_struct()
        self._check(self.L.hprqp_batch_solve(self.h, C.byref(p), x0ptr, None if sg is None else sg.ctypes.data,
                                             C.addressof(res), xptr))
        out = []
        for k in range(B):
            r = HPRQP_results()
            for f, _ in Result._fields_:
                if f == "status":
                    r.status = STATUS_NAMES[res[k].status]
                elif hasattr(r, f):
                    setattr(r, f, getattr(res[k], f))
            r.x = xs[k]
            out.append(r)
        return out

    def qap_apply(self, X, precision="fp64"):
        """Q_k(X_k) for every instance (X concatenated, each block
        column-major); returns (Y, used the tensor-core operator)."""
        from ._abi import PRECISIONS
        X = np.ascontiguousarray(X, dtype=np.float64)
        Y = np.zeros_like(X)
        tc = C.c_int32()
        self._check(self.L.hprqp_batch_qap_apply(self.h, PRECISIONS[precision], X.ctypes.data, Y.ctypes.data,
                                                 C.byref(tc)))
        return Y, bool(tc.value)

    def close(self):
        if getattr(self, "h", None):
            self.L.hprqp_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def solve_batch(models, params: HPRQP_parameters | None = None, initial_x=None, sigma0=None, device=0):
    if params is None:
        qap = ProblemView(models[0]).struct.Q_kind == Q_QAP
        params = HPRQP_parameters(verbose=False, problem_type="QAP" if qap else "LASSO")
    s = BatchSolver(models, device)
    try:
        return s.solve(params, initial_x, sigma0)
    finally:
        s.close()
