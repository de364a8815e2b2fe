"""QAP-relaxation batch measurement: plain FP64 single solves against the
batched engine (FP64, and FP32 + FP64 polish) on the same instances.

The family is `workloads.qap_batch`: `count` convexified QAP relaxations
(build_from_ABST; flow and distance matrices symmetric, zero diagonal,
integers U{0..10}) with n ~ U{nmin..nmax}.  Each path is timed on the wall
clock around the calls a user makes (host data in, solutions out); every
solve must end OPTIMAL with the objective within 1e-6 (FP64) / 1e-5 (FP32 +
polish) of the single FP64 solve.  Prints one JSON line.

    python -m hprqp_b200.qap_run --count 256 --nmin 30 --nmax 128 --seq-sample 16
    python -m hprqp_b200.qap_run --only batch_fp32      # one batched path alone
"""
from __future__ import annotations

import argparse
import json
import sys
import time

import numpy as np

from . import HPRQP_parameters, Solver
from . import workloads as W
from .batch import solve_batch


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--count", type=int, default=256)
    ap.add_argument("--nmin", type=int, default=30)
    ap.add_argument("--nmax", type=int, default=128)
    ap.add_argument("--tol", type=float, default=1e-6)
    ap.add_argument("--seq-sample", type=int, default=16,
                    help="time the sequential FP64 baseline on this many instances and scale (0 = all)")
    ap.add_argument("--only", default="all", choices=["all", "batch_fp64", "batch_fp32"],
                    help="one batched path alone, without the sequential baseline (for profilers)")
    a = ap.parse_args(argv)

    def log(*x):
        print(*x, file=sys.stderr, flush=True)

    t = time.perf_counter()
    models = W.qap_batch(a.count, a.nmin, a.nmax)
    sizes = [int(round(np.sqrt(m.n))) for m in models]
    log(f"generated {a.count} instances (n {min(sizes)}..{max(sizes)}) in {time.perf_counter() - t:.1f} s")
    out = dict(workload=f"qap_batch_{a.count}_n{a.nmin}-{a.nmax}", count=a.count, tol=a.tol,
               n_mean=float(np.mean(sizes)))
    base = dict(verbose=False, stoptol=a.tol, problem_type="QAP")
    if a.only != "all":
        prec = "fp64" if a.only == "batch_fp64" else "fp32_polish"
        t = time.perf_counter()
        res = solve_batch(models, HPRQP_parameters(**base, precision=prec))
        out[a.only] = dict(s=time.perf_counter() - t, solve_s=res[0].device_time,
                           iters=float(np.mean([r.iter for r in res])),
                           all_optimal=all(r.status == "OPTIMAL" for r in res))
        print(json.dumps(out), flush=True)
        return
    idx = list(range(a.count)) if not a.seq_sample else list(range(0, a.count, max(1, a.count // a.seq_sample)))
    t = time.perf_counter()
    ref = {}
    for k in idx:
        s = Solver().load(models[k])
        ref[k] = s.solve(HPRQP_parameters(**base))
        s.close()
    t_seq = (time.perf_counter() - t) * a.count / len(idx)
    out["seq_fp64"] = dict(s=t_seq, iters=float(np.mean([r.iter for r in ref.values()])), timed=len(idx),
                           all_optimal=all(r.status == "OPTIMAL" for r in ref.values()))
    log("seq fp64", json.dumps(out["seq_fp64"]))
    for tag, prec, tol in (("batch_fp64", "fp64", 1e-6), ("batch_fp32", "fp32_polish", 1e-5)):
        t = time.perf_counter()
        res = solve_batch(models, HPRQP_parameters(**base, precision=prec))
        dt = time.perf_counter() - t
        obj = max(abs(res[k].primal_obj - ref[k].primal_obj) / (1 + abs(ref[k].primal_obj)) for k in idx)
        out[tag] = dict(s=dt, solve_s=res[0].device_time, power_s=res[0].power_time,
                        iters=float(np.mean([r.iter for r in res])), max_iter=int(max(r.iter for r in res)),
                        all_optimal=all(r.status == "OPTIMAL" for r in res),
                        max_kkt=float(max(r.residuals for r in res)), max_rel_obj_vs_seq=obj,
                        obj_within_tol=bool(obj < tol), speedup_vs_seq=t_seq / dt)
        log(tag, json.dumps(out[tag]))
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
