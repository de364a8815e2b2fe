"""Python mirror of the reference solver API (src/algorithm.jl:1511-1554,
src/structs.jl:195-309) over libhprqp.so.

    model = build_from_QAbc(Q, c, A, AL, AU, l, u)
    params = HPRQP_parameters(); params.stoptol = 1e-6
    result = optimize(model, params)        # HPRQP_results

Parameter names, defaults, status strings and result fields are the
reference's.  Additions: params.precision ("fp64" | "fp32_polish"),
params.polish_tol, params.lambda_max_A_override/_Q_override.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _abi
from ._abi import Params, ProblemView, Result, STATUS_NAMES
from ._lib import check, load


@dataclass
class HPRQP_parameters:
    """HPRQP_parameters (src/structs.jl:195-275) with the reference defaults."""
    stoptol: float = 1e-6
    sigma: float = -1.0
    max_iter: int = 2**31 - 1
    sigma_fixed: bool = False
    time_limit: float = 3600.0
    eig_factor: float = 1.05
    check_iter: int = 100
    warm_up: bool = False
    spmv_mode_Q: str = "auto"
    spmv_mode_A: str = "auto"
    print_frequency: int = -1
    device_number: int = 0
    use_Ruiz_scaling: bool = True
    use_bc_scaling: bool = False
    use_l2_scaling: bool = False
    use_Pock_Chambolle_scaling: bool = True
    problem_type: str = "QP"
    lambda_: float = 0.0
    initial_x: np.ndarray | None = None
    initial_y: np.ndarray | None = None
    auto_save: bool = False
    save_filename: str = "hprqp_autosave.ckpt"
    verbose: bool = True
    use_gpu: bool = True
    # extensions
    precision: str = "fp64"
    polish_tol: float = -1.0
    lambda_max_A_override: float = -1.0
    lambda_max_Q_override: float = -1.0
    profile_passes: bool = False

    def to_struct(self) -> Params:
        p = _abi.default_params()
        for name in ("stoptol", "sigma", "time_limit", "eig_factor", "polish_tol",
                     "lambda_max_A_override", "lambda_max_Q_override"):
            setattr(p, name, float(getattr(self, name)))
        p.lambda_ = float(self.lambda_)
        p.max_iter = int(self.max_iter)
        p.check_iter = int(self.check_iter)
        p.print_frequency = int(self.print_frequency)
        p.device_number = int(self.device_number)
        for name in ("sigma_fixed", "warm_up", "use_Ruiz_scaling", "use_bc_scaling", "use_l2_scaling",
                     "use_Pock_Chambolle_scaling", "auto_save", "verbose", "use_gpu", "profile_passes"):
            setattr(p, name, int(bool(getattr(self, name))))
        p.spmv_mode_Q = _spmv_mode(self.spmv_mode_Q)
        p.spmv_mode_A = _spmv_mode(self.spmv_mode_A)
        if self.problem_type not in _abi.PROBLEM_TYPES:
            raise ValueError(f"problem_type must be one of {list(_abi.PROBLEM_TYPES)}")
        p.problem_type = _abi.PROBLEM_TYPES[self.problem_type]
        if self.precision not in _abi.PRECISIONS:
            raise ValueError(f"precision must be one of {list(_abi.PRECISIONS)}")
        p.precision = _abi.PRECISIONS[self.precision]
        return p


def _spmv_mode(v) -> int:
    """'auto' (autotuned), 'CUSPARSE'/'customized' (reference names, treated
    as auto), 'sell' (SELL-32), 'ell' (ELL), 'split' (long rows cut into
    equal pieces), 'staged' (column blocks of the input vector in shared
    memory), or an explicit CSR threads-per-row 1..32."""
    if isinstance(v, str):
        return {"sell": 7, "ell": 8, "split": 9, "staged": 10}.get(v.lower(), 0)
    t = int(v)
    if t not in (1, 2, 4, 8, 16, 32):
        raise ValueError("threads per row must be 1, 2, 4, 8, 16 or 32")
    return int(np.log2(t)) + 1


@dataclass
class HPRQP_results:
    """HPRQP_results (src/structs.jl:292-309) plus the library's extras."""
    iter: int = 0
    iter_4: int = 0
    iter_6: int = 0
    time: float = 0.0
    time_4: float = 0.0
    time_6: float = 0.0
    power_time: float = 0.0
    primal_obj: float = 0.0
    residuals: float = 0.0
    gap: float = 0.0
    status: str = ""
    x: np.ndarray = field(default_factory=lambda: np.zeros(0))
    y: np.ndarray = field(default_factory=lambda: np.zeros(0))
    z: np.ndarray = field(default_factory=lambda: np.zeros(0))
    w: np.ndarray = field(default_factory=lambda: np.zeros(0))
    # extras
    dual_obj: float = 0.0
    err_Rp: float = 0.0
    err_Rd: float = 0.0
    setup_time: float = 0.0
    sigma: float = 0.0
    lambda_max_A: float = 0.0
    lambda_max_Q: float = 0.0
    restarts: int = 0
    iter_fp32: int = 0
    gpu_launches: int = 0
    Q_is_diag: bool = False
    device_time: float = 0.0
    power_iter_A: int = 0
    power_iter_Q: int = 0
    power_bytes: float = 0.0
    h2d_bytes: int = 0
    d2h_bytes: int = 0


def _stats_dict(st):
    passes = []
    for k in range(st.npass):
        passes.append(dict(name=st.name[k].value.decode(), ms=st.ms_per_launch[k],
                           bytes=st.bytes_per_launch[k], threads_per_row=st.threads_per_row[k],
                           ms_back_to_back=st.ms_back_to_back[k]))
    return dict(path=st.path, iters=st.iters, ms_per_iter=st.ms_per_iter, bytes_per_iter=st.bytes_per_iter,
                passes=passes)


def _ptr(a):
    return None if a is None else a.ctypes.data


class Solver:
    """A libhprqp handle bound to one device and one loaded model.  Reusing
    it across solves keeps the scaled problem resident in HBM."""

    def __init__(self, device: int = 0):
        L = load()
        h = C.c_void_p()
        check(L.hprqp_create(C.byref(h), int(device)), None)
        self._L, self.h = L, h
        self.model = None
        self._view = None

    def load(self, model):
        self._view = ProblemView(model)  # keeps the arrays alive during the copy
        check(self._L.hprqp_load(self.h, C.addressof(self._view.struct)), self.h)
        self.model = model
        self._view = None
        self._qmap_cb = None
        if model.Q.kind == _abi.Q_CUSTOM:
            self._bind_qmap(model.Q)
        return self

    def _bind_qmap(self, op):
        """Bind a CustomQ's device_qmap as the library's hprqp_qmap_fn; the
        ctypes thunk is kept on the solver for as long as it may be called.
        An exception in the operator becomes a nonzero return, which stops
        the solve with HPRQP_E_CALLBACK (the exception is chained to it)."""
        def thunk(x, qx, precision, user, stream):
            try:
                rc = op.device_qmap(x or 0, qx or 0, int(precision), stream or 0)
                return int(rc or 0)
            except Exception as e:  # noqa: BLE001 - reported through the return code
                self._qmap_error = e
                return -1
        self._qmap_error = None
        self._qmap_cb = _abi.QMAP_FN(thunk)
        check(self._L.hprqp_set_qmap(self.h, self._qmap_cb, None), self.h)

    def prepare(self, params: HPRQP_parameters):
        check(self._L.hprqp_prepare(self.h, C.byref(params.to_struct())), self.h)

    def set_trace(self, iters: int):
        n, m = self.model.n, self.model.m
        self._trace = (np.zeros((iters, n)), np.zeros((iters, m)), np.zeros((iters, n))) if iters else None
        t = self._trace
        check(self._L.hprqp_set_trace(self.h, iters, *( [_ptr(a) for a in t] if t else [None] * 3)), self.h)
        self._strace = (np.zeros(iters), np.zeros(iters, dtype=np.int64)) if iters else None
        st = self._strace
        check(self._L.hprqp_set_trace_scalars(self.h, *([_ptr(a) for a in st] if st else [None] * 2)), self.h)
        return self._trace

    def scalar_trace(self):
        """(sigma, inner) of each iteration traced by the last solve after
        set_trace: the sigma the step used and its Halpern counter (0 right
        after a restart)."""
        return self._strace

    def solve(self, params: HPRQP_parameters) -> HPRQP_results:
        return self._run(params, None)

    def resume(self, params: HPRQP_parameters, path: str) -> HPRQP_results:
        """Continue a solve of the loaded model from a checkpoint that
        params.auto_save wrote (hprqp_solve_resume)."""
        return self._run(params, path)

    def _run(self, params, resume_path):
        model = self.model
        n, m = model.n, model.m
        x, y, z, w = np.zeros(n), np.zeros(m), np.zeros(n), np.zeros(n)
        x0 = None if params.initial_x is None else np.ascontiguousarray(params.initial_x, dtype=np.float64)
        y0 = None if params.initial_y is None else np.ascontiguousarray(params.initial_y, dtype=np.float64)
        if x0 is not None and len(x0) != n:
            raise ValueError("initial_x has the wrong length")
        if y0 is not None and len(y0) != m:
            raise ValueError("initial_y has the wrong length")
        if params.auto_save:
            check(self._L.hprqp_set_save_file(self.h, str(params.save_filename).encode()), self.h)
        r = Result()
        try:
            if resume_path is None:
                rc = self._L.hprqp_solve(self.h, C.byref(params.to_struct()), _ptr(x0), _ptr(y0), C.byref(r),
                                         _ptr(x), _ptr(y), _ptr(z), _ptr(w))
            else:
                rc = self._L.hprqp_solve_resume(self.h, C.byref(params.to_struct()), str(resume_path).encode(),
                                                C.byref(r), _ptr(x), _ptr(y), _ptr(z), _ptr(w))
            check(rc, self.h)
        except Exception as e:
            err = getattr(self, "_qmap_error", None)
            if err is not None:
                self._qmap_error = None
                raise e from err
            raise
        out = HPRQP_results()
        for f, _ in Result._fields_:
            if f == "status":
                out.status = STATUS_NAMES[r.status]
            elif hasattr(out, f):
                setattr(out, f, getattr(r, f))
        out.Q_is_diag = bool(r.Q_is_diag)
        out.x, out.y, out.z, out.w = x, (y if m > 0 else np.zeros(0)), z, w
        return out

    def pass_stats(self):
        """Per-pass CUDA-event timings of the last solve run with
        params.profile_passes (fp64 and fp32 engines)."""
        a, b = _abi.PassStats(), _abi.PassStats()
        check(self._L.hprqp_get_pass_stats(self.h, C.byref(a), C.byref(b)), self.h)
        return {"fp64": _stats_dict(a), "fp32": _stats_dict(b)}

    def profile_iterations(self, params: HPRQP_parameters, iters: int = 50, full: bool = False):
        """Run `iters` HPR iterations from the zero state and time each pass."""
        st = _abi.PassStats()
        check(self._L.hprqp_profile_iterations(self.h, C.byref(params.to_struct()), iters, int(full),
                                               C.byref(st)), self.h)
        return _stats_dict(st)

    def close(self):
        if self.h:
            self._L.hprqp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def optimize(model, params: HPRQP_parameters | None = None) -> HPRQP_results:
    """optimize(model, params) (src/algorithm.jl:1511-1554) on the GPU."""
    params = params or HPRQP_parameters()
    s = Solver(params.device_number).load(model)
    try:
        return s.solve(params)
    finally:
        s.close()
