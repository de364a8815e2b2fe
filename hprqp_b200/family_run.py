"""LASSO-family measurement: plain FP64 single solves against the batched
engine (FP64, FP32 + FP64 polish) with and without the learned warm start.

The family is the fixed-pattern LASSO family of `workloads.lasso_family`
(A 2,000 x 10,000 at 1 %, values perturbed 5 % per instance, b = A x* +
0.01 N(0,1), lambda = logU(1e-4, 1e-2) ||A'b||_inf).  Training labels come
from batched plain-HPR solves to 1e-8; held-out instances are then solved to
1e-6 four ways, each timed on the wall clock around the call a user makes
(host data in, solutions out):

  seq_fp64      one `Solver.solve` per instance, plain FP64 (the baseline)
  batch_fp64    one batched solve, plain FP64
  batch_fp32    one batched solve, FP32 storage + FP64 polish
  batch_learned as batch_fp32, started from the network's x0 (proposal time
                included); batch_learned_sigma also takes its sigma0;
                batch_learned_sigma_only takes sigma0 alone

Every solve must end OPTIMAL with the objective within 1e-6 (relative) of
the sequential FP64 solve.  Prints one JSON line.

    python -m hprqp_b200.family_run --train 3000 --test 1000
"""
from __future__ import annotations

import argparse
import json
import sys
import time

import numpy as np

from . import HPRQP_parameters, Solver
from . import learned
from . import workloads as W
from .batch import solve_batch


def _rel(a, b):
    return abs(a - b) / (1.0 + abs(b))


def _learn(a, train, out, log):
    t = time.perf_counter()
    pairs = learned.generate_pairs(train, tol=a.label_tol, chunk=a.chunk)
    out["label_s"] = time.perf_counter() - t
    out["labels"] = len(pairs)
    out["label_iters_mean"] = float(np.mean([p.iters for p in pairs]))
    log(f"labels: {len(pairs)} in {out['label_s']:.1f} s")

    t = time.perf_counter()
    ws = learned.WarmStart.fit(pairs, epochs=a.epochs, lr=a.lr, width=a.width, batch=256)
    out["train_s"] = time.perf_counter() - t
    out["loss_first"], out["loss_last"] = float(ws.history[0]), float(ws.history[-1])
    log(f"trained in {out['train_s']:.1f} s, loss {ws.history[0]:.4f} -> {ws.history[-1]:.4f}")

    return ws


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--train", type=int, default=3000)
    ap.add_argument("--test", type=int, default=1000)
    ap.add_argument("--m", type=int, default=2000)
    ap.add_argument("--n", type=int, default=10000)
    ap.add_argument("--density", type=float, default=0.01)
    ap.add_argument("--epochs", type=int, default=150)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--width", type=int, default=512)
    ap.add_argument("--label-tol", type=float, default=1e-8)
    ap.add_argument("--tol", type=float, default=1e-6)
    ap.add_argument("--seq-sample", type=int, default=0,
                    help="time the sequential FP64 baseline on this many test instances and scale (0 = all)")
    ap.add_argument("--chunk", type=int, default=500)
    a = ap.parse_args(argv)
    fam = dict(m=a.m, n=a.n, density=a.density)
    out = dict(workload=f"lasso_family_{a.m}x{a.n}_d{a.density}", train=a.train, test=a.test, tol=a.tol)

    def log(*x):
        print(*x, file=sys.stderr, flush=True)

    t = time.perf_counter()
    train = W.lasso_family(a.train, start=0, **fam)
    test = W.lasso_family(a.test, start=1_000_000, **fam)
    log(f"generated {a.train}+{a.test} instances in {time.perf_counter() - t:.1f} s")

    ws = None
    if a.train > 0:
        ws = _learn(a, train, out, log)

    base = dict(verbose=False, stoptol=a.tol, problem_type="LASSO")

    # plain FP64, one instance at a time
    seq = test[:a.seq_sample] if a.seq_sample else test
    t = time.perf_counter()
    ref = []
    for mdl in seq:
        s = Solver().load(mdl)
        ref.append(s.solve(HPRQP_parameters(**base)))
        s.close()
    t_seq = (time.perf_counter() - t) * len(test) / len(seq)
    sc = len(test) / len(seq)
    out["seq_fp64"] = dict(s=t_seq, iters=float(np.mean([r.iter for r in ref])), timed=len(seq),
                           solve_s=sc * sum(r.device_time for r in ref), power_s=sc * sum(r.power_time for r in ref))
    log(f"seq fp64: {t_seq:.2f} s")

    sol = {}

    def batched(tag, precision, x0=None, sg=None, extra_s=0.0):
        res, solve_s, power_s, max_it = [], 0.0, 0.0, 0
        t0 = time.perf_counter()
        for i in range(0, len(test), a.chunk):
            part = test[i:i + a.chunk]
            xs = None if x0 is None else list(x0[i:i + a.chunk])
            ss = None if sg is None else list(sg[i:i + a.chunk])
            rr = solve_batch(part, HPRQP_parameters(**base, precision=precision), initial_x=xs, sigma0=ss)
            solve_s += rr[0].device_time
            power_s += rr[0].power_time
            max_it = max(max_it, max(r.iter for r in rr))
            res += rr
        dt = time.perf_counter() - t0 + extra_s
        ok = all(r.status == "OPTIMAL" for r in res)
        obj = max(_rel(r.primal_obj, q.primal_obj) for r, q in zip(res, ref))
        kkt = max(max(r.residuals, 0.0) for r in res)
        sol[tag] = [r.x for r in res]
        out[tag] = dict(s=dt, solve_s=solve_s, power_s=power_s, max_iter=max_it,
                        iters=float(np.mean([r.iter for r in res])), all_optimal=ok,
                        max_rel_obj_vs_seq=obj, max_kkt=kkt, speedup_vs_seq=t_seq / dt)
        log(tag, json.dumps(out[tag]))

    batched("batch_fp64", "fp64")
    batched("batch_fp32", "fp32_polish")
    if ws is None:
        print(json.dumps(out), flush=True)
        return
    t = time.perf_counter()
    x0, sg = [], []
    for i in range(0, len(test), 256):
        xp, sp = ws.propose(test[i:i + 256])
        x0.append(xp)
        sg.append(sp)
    x0, sg = np.concatenate(x0), np.concatenate(sg)
    t_prop = time.perf_counter() - t
    out["propose_s"] = t_prop
    # how close the proposals are to the solutions (the FP64 batch's)
    out["x0_rel_err_mean"] = float(np.mean([np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)
                                            for a, b in zip(x0, sol["batch_fp64"])]))
    out["x0_zero_rel_err"] = 1.0
    batched("batch_learned", "fp32_polish", x0=x0, extra_s=t_prop)
    batched("batch_learned_sigma", "fp32_polish", x0=x0, sg=sg, extra_s=t_prop)
    batched("batch_learned_sigma_only", "fp32_polish", sg=sg, extra_s=t_prop)
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
