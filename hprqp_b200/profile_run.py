"""Run the iteration engine alone, for profilers (ncu) and quick timing.

    python -m hprqp_b200.profile_run --grid 700 --precision fp64 --mode iterations --iters 10
    python -m hprqp_b200.profile_run --grid 700 --precision fp32_polish --mode solve

--mode iterations: prepare, then hprqp_profile_iterations (5 warm-up + 2 x iters
                   plain HPR iterations from the zero state); lambda_max is
                   injected (--lam-A/--lam-Q, defaults for the 700x700 grid from
                   the oracle) so no power-method launches precede the passes.
--mode solve:      one full solve to 1e-6 (power method included).
--mode power:      the power method alone (max_iter = 0): both chains, the
                   A A' chain alone and the Q chain alone (the other's
                   lambda given as --lam-Q / --lam-A), median of 5 solves.
--mode gemm:       the 3xTF32 tensor-core GEMM of the FP32 QAP operator on
                   --n x --n FP32 matrices with a preallocated workspace
                   (--iters timed calls after 3 warm-up calls, each call =
                   the two TF32 image splits + the GEMM); reports time and
                   TFLOP/s (2 n^3 per product; the tensor pipe executes 3x
                   that).
Prints one JSON line with the per-pass CUDA-event times.
"""
import argparse
import json
import sys

from . import HPRQP_parameters, Solver
from . import workloads as W


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--grid", type=int, default=700)
    ap.add_argument("--workload", default="grid", choices=["grid", "random_qp", "lasso"])
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32_polish"])
    ap.add_argument("--mode", default="iterations", choices=["iterations", "solve", "gemm", "power"])
    ap.add_argument("--n", type=int, default=2048)
    ap.add_argument("--iters", type=int, default=10)
    ap.add_argument("--lam-A", type=float, default=0.44866094653915195)
    ap.add_argument("--lam-Q", type=float, default=0.8051445993716677)
    ap.add_argument("--tpr", default="0", help="CSR threads per row, 'sell', 'ell', or 0 = autotune")
    a = ap.parse_args(argv)
    if a.mode == "gemm":
        print(json.dumps(_gemm(a.n, a.iters)))
        return 0
    if a.workload == "grid":
        model, ptype = W.grid_qp(N=a.grid), "QP"
    elif a.workload == "random_qp":
        model, ptype = W.random_qp(), "QP"
    else:
        model, ptype = W.lasso(), "LASSO"
    s = Solver(0).load(model)
    if a.mode == "power":
        # the power method alone (max_iter = 0): both chains, then each chain with the other's
        # lambda given, median of 5 solves each
        out = {}
        for tag, over in (("both", {}), ("A_only", {"lambda_max_Q_override": a.lam_Q}),
                          ("Q_only", {"lambda_max_A_override": a.lam_A})):
            p = HPRQP_parameters(verbose=False, precision=a.precision, problem_type=ptype, max_iter=0, **over)
            if a.tpr != "0":
                p.spmv_mode_Q = p.spmv_mode_A = a.tpr if a.tpr in ("sell", "ell") else int(a.tpr)
            ts, r = [], None
            for _ in range(6):
                r = s.solve(p)
                ts.append(r.power_time)
            ts = sorted(ts[1:])
            out[tag] = dict(power_ms=ts[len(ts) // 2] * 1e3, steps=[r.power_iter_A, r.power_iter_Q],
                            lam=[r.lambda_max_A, r.lambda_max_Q])
        s.close()
        print(json.dumps(out))
        return 0
    if a.mode == "iterations":
        p = HPRQP_parameters(verbose=False, precision=a.precision, problem_type=ptype,
                             lambda_max_A_override=a.lam_A, lambda_max_Q_override=a.lam_Q)
        if a.tpr != "0":
            p.spmv_mode_Q = p.spmv_mode_A = a.tpr if a.tpr in ("sell", "ell") else int(a.tpr)
        out = s.profile_iterations(p, a.iters)
    else:
        p = HPRQP_parameters(verbose=False, precision=a.precision, problem_type=ptype, profile_passes=True)
        if a.tpr != "0":
            p.spmv_mode_Q = p.spmv_mode_A = a.tpr if a.tpr in ("sell", "ell") else int(a.tpr)
        r = s.solve(p)
        out = dict(status=r.status, iter=r.iter, iter_fp32=r.iter_fp32, time=r.time, device_time=r.device_time,
                   power_time=r.power_time, power_iter=[r.power_iter_A, r.power_iter_Q], kkt=r.residuals, launches=r.gpu_launches, passes=s.pass_stats())
    s.close()
    print(json.dumps(out))
    return 0


def _gemm(n, iters):
    import ctypes as C

    import torch

    from ._lib import load
    L = load()
    g = torch.Generator(device="cuda").manual_seed(0)
    A, B, Cm = (torch.randn(n * n, device="cuda", generator=g) for _ in range(3))
    ws = torch.empty(int(L.hprqp_gemm_3xtf32_ws_floats(n)), device="cuda", dtype=torch.float32)
    st = torch.cuda.current_stream()
    call = lambda: L.hprqp_gemm_3xtf32_ws(n, C.c_float(1.0), A.data_ptr(), B.data_ptr(), C.c_float(0.0),
                                          Cm.data_ptr(), ws.data_ptr(), C.c_void_p(st.cuda_stream))
    for _ in range(3):
        assert call() == 0
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ms = []
    for _ in range(iters):
        e0.record(st)
        assert call() == 0
        e1.record(st)
        torch.cuda.synchronize()
        ms.append(e0.elapsed_time(e1))
    assert L.hprqp_gemm_3xtf32(8, C.c_float(1.0), A.data_ptr(), B.data_ptr(), C.c_float(0.0), Cm.data_ptr(),
                               C.c_void_p(st.cuda_stream)) == 0  # also reports a timed-out wait of the runs above
    ms.sort()
    t = ms[len(ms) // 2] / 1e3
    return dict(n=n, ms=t * 1e3, tflops=2.0 * n ** 3 / t / 1e12, tensor_tflops=6.0 * n ** 3 / t / 1e12)


if __name__ == "__main__":
    sys.exit(main())
