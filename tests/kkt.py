"""Independent KKT check of a returned (unscaled) QP solution, in numpy.

Written from the optimality conditions of
    min 0.5 x'Qx + c'x + c0   s.t.  AL <= Ax <= AU,  l <= x <= u
with stationarity Qx + c - A'y - z = 0, the same sign convention and
relative normalisation as the reference's residuals (src/algorithm.jl:73-95),
but using the textbook dual objective (support functions of the boxes)
instead of any solver-internal quantity.
"""
import numpy as np


def _support(v, lo, hi, tol=1e-9):
    # sum_i min over s in [lo_i, hi_i] of v_i s  (the dual function's box term)
    out = 0.0
    for vi, a, b in zip(v, lo, hi):
        if vi > tol:
            out += vi * a if np.isfinite(a) else -np.inf
        elif vi < -tol:
            out += vi * b if np.isfinite(b) else -np.inf
    return out


def kkt(model, x, y, z):
    Q = model.Q.Q if hasattr(model.Q, "Q") else None
    Qx = model.Q.Qmap(x)
    A = model.A
    Ax = A @ x if model.m else np.zeros(0)
    ATy = A.T @ y if model.m else np.zeros(model.n)
    bnorm = 0.0
    if model.m:
        AL0 = np.where(np.isinf(model.AL), 0.0, model.AL)
        AU0 = np.where(np.isinf(model.AU), 0.0, model.AU)
        bnorm = np.max(np.maximum(np.abs(AL0), np.abs(AU0)))
    rp = 0.0
    if model.m:
        rp = np.max(np.abs(np.clip(Ax, model.AL, model.AU) - Ax)) / (1 + max(bnorm, np.max(np.abs(Ax))))
    bviol = np.max(np.maximum(model.l - x, 0) + np.maximum(x - model.u, 0))
    rd = np.max(np.abs(Qx + model.c - ATy - z)) / (
        1 + max(np.max(np.abs(model.c)), np.max(np.abs(ATy)), np.max(np.abs(Qx))))
    p = model.c @ x + 0.5 * x @ Qx + model.obj_constant
    d = -0.5 * x @ Qx + model.obj_constant + _support(z, model.l, model.u)
    if model.m:
        d += _support(y, model.AL, model.AU)
    gap = abs(p - d) / (1 + max(abs(p), abs(d)))
    return dict(err_Rp=max(rp, bviol), err_Rd=rd, gap=gap, pobj=p, dobj=d, KKT=max(rp, bviol, rd, gap))
