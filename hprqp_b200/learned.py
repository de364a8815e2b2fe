"""Learned warm start for a problem family (LASSO family: fixed sparsity
pattern, perturbed values, varying b and lambda).

The network (libhprqp's BF16 MLP, include/hprqp_mlp.h) maps instance
features (b, log lambda) to a proposed solution x and log sigma.  The solver
then starts from that proposal (`initial_x`, `sigma`, the reference's own
warm-start parameters, src/algorithm.jl:1783-1836, 838-851) and runs the
unmodified HPR iteration to the requested tolerance, so the final KKT
residual is certified by the method itself: a bad proposal only costs
iterations.

    pairs = generate_pairs(family_models, tol=1e-8)     # solver-made labels
    ws = WarmStart.fit(pairs, epochs=...)
    x0, sigma0 = ws.propose(model)
"""
from __future__ import annotations

import ctypes as C
import os
import time
from dataclasses import dataclass

import numpy as np

from ._lib import HPRQPError, load

_mlp_lib = None


def _lib():
    global _mlp_lib
    if _mlp_lib is None:
        L = load()
        vp = C.c_void_p
        fp = C.POINTER(C.c_float)
        L.hprqp_mlp_create.argtypes = [C.POINTER(vp), C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                                       C.c_uint64]
        L.hprqp_mlp_train_batch.argtypes = [vp, fp, fp, C.c_int32, C.c_float, C.POINTER(C.c_double)]
        L.hprqp_mlp_gradients.argtypes = [vp, fp, fp, C.c_int32, fp, C.POINTER(C.c_double)]
        L.hprqp_mlp_predict.argtypes = [vp, fp, C.c_int64, fp]
        L.hprqp_mlp_get_params.argtypes = [vp, fp, C.POINTER(C.c_int64)]
        L.hprqp_mlp_set_params.argtypes = [vp, fp]
        L.hprqp_mlp_last_error.argtypes = [vp]
        L.hprqp_mlp_last_error.restype = C.c_char_p
        L.hprqp_mlp_destroy.argtypes = [vp]
        for f in ("hprqp_mlp_create", "hprqp_mlp_train_batch", "hprqp_mlp_gradients", "hprqp_mlp_predict",
                  "hprqp_mlp_get_params", "hprqp_mlp_set_params", "hprqp_mlp_destroy"):
            getattr(L, f).restype = C.c_int
        _mlp_lib = L
    return _mlp_lib


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _fp(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


class MLP:
    """n_in -> width -> width -> n_out (ReLU), BF16 weights, FP32 accumulate,
    trained with Adam by libhprqp's kernels."""

    def __init__(self, n_in, n_out, width=512, batch=256, device=0, seed=1):
        self.L = _lib()
        h = C.c_void_p()
        self._check(self.L.hprqp_mlp_create(C.byref(h), device, n_in, width, n_out, batch, seed), None)
        self.h, self.n_in, self.n_out, self.width, self.batch = h, n_in, n_out, width, batch

    def _check(self, rc, h):
        if rc != 0:
            raise HPRQPError(rc, self.L.hprqp_mlp_last_error(h).decode())

    def train_batch(self, X, T, lr):
        X, T = _f32(X), _f32(T)
        loss = C.c_double()
        self._check(self.L.hprqp_mlp_train_batch(self.h, _fp(X), _fp(T), X.shape[0], lr, C.byref(loss)), self.h)
        return loss.value

    def gradients(self, X, T):
        X, T = _f32(X), _f32(T)
        g = np.zeros(self.num_params(), dtype=np.float32)
        loss = C.c_double()
        self._check(self.L.hprqp_mlp_gradients(self.h, _fp(X), _fp(T), X.shape[0], _fp(g), C.byref(loss)), self.h)
        return loss.value, g

    def predict(self, X):
        X = _f32(np.atleast_2d(X))
        Y = np.zeros((X.shape[0], self.n_out), dtype=np.float32)
        self._check(self.L.hprqp_mlp_predict(self.h, _fp(X), X.shape[0], _fp(Y)), self.h)
        return Y

    def num_params(self):
        n = C.c_int64()
        self._check(self.L.hprqp_mlp_get_params(self.h, None, C.byref(n)), self.h)
        return n.value

    def get_params(self):
        p = np.zeros(self.num_params(), dtype=np.float32)
        n = C.c_int64()
        self._check(self.L.hprqp_mlp_get_params(self.h, _fp(p), C.byref(n)), self.h)
        return p

    def set_params(self, p):
        p = _f32(p)
        self._check(self.L.hprqp_mlp_set_params(self.h, _fp(p)), self.h)

    def unpack(self, p):
        """[W1, b1, W2, b2, W3, b3] views of a parameter vector."""
        dims = [self.n_in, self.width, self.width, self.n_out]
        out, off = [], 0
        for k in range(3):
            W = p[off:off + dims[k + 1] * dims[k]].reshape(dims[k + 1], dims[k])
            off += dims[k + 1] * dims[k]
            b = p[off:off + dims[k + 1]]
            off += dims[k + 1]
            out += [W, b]
        return out

    def close(self):
        if getattr(self, "h", None):
            self.L.hprqp_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# Problem-family pipeline (LASSO family)
# ---------------------------------------------------------------------------
def lasso_scale(model):
    """Instance scale: ||c||_inf with c = -A'b.  Features and the solution
    target are divided by it, so the network works on scale-free data."""
    return float(max(np.abs(np.asarray(model.c)).max(), 1e-300))


def lasso_features(model):
    """Scale-free features of a LASSO instance (build_from_Ab_lambda):
    c / ||c||_inf (c = -A'b, what the solver sees) and log(lambda / ||c||_inf)."""
    s = lasso_scale(model)
    return np.concatenate([np.asarray(model.c) / s, [np.log(model.lambda_ / s)]]).astype(np.float32)


@dataclass
class Pair:
    features: np.ndarray
    x: np.ndarray       # converged solution divided by the instance scale
    sigma: float        # final sigma
    iters: int


def generate_pairs(models, tol=1e-8, precision="fp64", device=0, features=lasso_features, chunk=500):
    """Solve the instances with plain HPR to `tol` (batched, `chunk` at a
    time) and record (features -> solution / scale, sigma): the training
    labels come from the solver itself."""
    from . import HPRQP_parameters
    from .batch import solve_batch
    pairs = []
    p = HPRQP_parameters(verbose=False, stoptol=tol, problem_type="LASSO", precision=precision)
    for i in range(0, len(models), chunk):
        part = models[i:i + chunk]
        for m, r in zip(part, solve_batch(part, p, device=device)):
            if r.status == "OPTIMAL":
                pairs.append(Pair(features(m), (r.x / lasso_scale(m)).astype(np.float32), float(r.sigma),
                                  int(r.iter)))
    return pairs


class WarmStart:
    """Feature/target normalisation + the MLP; proposes (x0, sigma0)."""

    def __init__(self, mlp, fmean, fstd, tmean, tstd):
        self.mlp, self.fmean, self.fstd, self.tmean, self.tstd = mlp, fmean, fstd, tmean, tstd

    @classmethod
    def fit(cls, pairs, epochs=200, lr=1e-3, width=512, batch=256, seed=1, device=0, verbose=False):
        F = np.stack([p.features for p in pairs]).astype(np.float32)
        T = np.stack([np.concatenate([p.x, [np.log(p.sigma)]]) for p in pairs]).astype(np.float32)
        fmean, fstd = F.mean(0), F.std(0) + 1e-6
        # one scale for the (sparse) solution block, its own for log sigma:
        # per-coordinate scaling would blow up coordinates that are almost
        # always zero
        tmean = np.zeros(T.shape[1], dtype=np.float32)
        tstd = np.full(T.shape[1], T[:, :-1].std() + 1e-12, dtype=np.float32)
        tmean[-1], tstd[-1] = T[:, -1].mean(), T[:, -1].std() + 1e-6
        Fn, Tn = (F - fmean) / fstd, (T - tmean) / tstd
        mlp = MLP(F.shape[1], T.shape[1], width=width, batch=batch, device=device, seed=seed)
        rng = np.random.default_rng(seed)
        hist = []
        for ep in range(epochs):
            perm = rng.permutation(len(Fn))
            tot = 0.0
            for i in range(0, len(perm), batch):
                idx = perm[i:i + batch]
                tot += mlp.train_batch(Fn[idx], Tn[idx], lr) * len(idx)
            hist.append(tot / len(perm))
            if verbose and (ep % max(1, epochs // 10) == 0 or ep == epochs - 1):
                print(f"  epoch {ep}: loss {hist[-1]:.5f}", flush=True)
        ws = cls(mlp, fmean, fstd, tmean, tstd)
        ws.history = hist
        return ws

    def propose(self, models):
        """(x0, sigma0) for a list of instances of the family."""
        models = models if isinstance(models, (list, tuple)) else [models]
        F = np.stack([lasso_features(m) for m in models])
        y = self.mlp.predict(((F - self.fmean) / self.fstd).astype(np.float32))
        y = y * self.tstd + self.tmean
        sc = np.array([lasso_scale(m) for m in models])[:, None]
        x0 = y[:, :-1].astype(np.float64) * sc
        sigma0 = np.exp(np.clip(y[:, -1], -30, 30)).astype(np.float64)
        return x0, sigma0


def evaluate(models, ws: WarmStart | None, tol=1e-6, precision="fp64", device=0, features=lasso_features,
             use_sigma=False):
    """Solve each instance cold and warm-started from the network's x (and
    sigma when use_sigma); return per-instance iterations, time, status."""
    from . import HPRQP_parameters, Solver
    rows = []
    for m in models:
        s = Solver(device).load(m)
        base = dict(verbose=False, stoptol=tol, problem_type="LASSO", precision=precision)
        cold = s.solve(HPRQP_parameters(**base))
        rec = dict(cold_iter=cold.iter, cold_time=cold.device_time, cold_status=cold.status,
                   cold_obj=cold.primal_obj)
        if ws is not None:
            x0, sg = ws.propose(m)
            kw = dict(initial_x=x0[0])
            if use_sigma:
                kw["sigma"] = float(sg[0])
            warm = s.solve(HPRQP_parameters(**base, **kw))
            rec.update(warm_iter=warm.iter, warm_time=warm.device_time, warm_status=warm.status,
                       warm_obj=warm.primal_obj)
        s.close()
        rows.append(rec)
    return rows
