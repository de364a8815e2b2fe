"""ctypes mirrors of the structs in include/hprqp.h.

Field order and types must match the C header exactly; tests/test_abi.py
checks the sizes against the compiled library's own sizeof() report.
"""
import ctypes as C

c_i32p = C.POINTER(C.c_int32)
c_f64p = C.POINTER(C.c_double)

HPRQP_OK = 0
HPRQP_E_ARG = -1
HPRQP_E_CUDA = -2
HPRQP_E_OOM = -3
HPRQP_E_STATE = -4
HPRQP_E_UNSUPPORTED = -5

STATUS_NAMES = {0: "OPTIMAL", 1: "MAX_ITER", 2: "TIME_LIMIT", 3: "NUMERICAL_ERROR"}

Q_SPARSE, Q_LASSO, Q_QAP, Q_CUSTOM = 0, 1, 2, 3
HPRQP_E_CALLBACK = -6

# int32_t qmap(const void* x, void* Qx, int32_t precision, void* user, void* stream)
QMAP_FN = C.CFUNCTYPE(C.c_int32, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p)
PROBLEM_TYPES = {"QP": 0, "LASSO": 1, "QAP": 2}
PRECISIONS = {"fp64": 0, "fp32_polish": 1}


class Problem(C.Structure):
    _fields_ = [
        ("n", C.c_int64), ("m", C.c_int64),
        ("index_base", C.c_int32), ("Q_kind", C.c_int32),
        ("A_colptr", c_i32p), ("A_rowval", c_i32p), ("A_nzval", c_f64p),
        ("c", c_f64p), ("AL", c_f64p), ("AU", c_f64p), ("l", c_f64p), ("u", c_f64p),
        ("obj_constant", C.c_double), ("lambda_", C.c_double),
        ("Q_colptr", c_i32p), ("Q_rowval", c_i32p), ("Q_nzval", c_f64p),
        ("lasso_m", C.c_int64),
        ("L_colptr", c_i32p), ("L_rowval", c_i32p), ("L_nzval", c_f64p),
        ("qap_n", C.c_int64),
        ("qap_A", c_f64p), ("qap_B", c_f64p), ("qap_S", c_f64p), ("qap_T", c_f64p),
    ]


class Params(C.Structure):
    _fields_ = [
        ("stoptol", C.c_double), ("sigma", C.c_double), ("max_iter", C.c_int64),
        ("sigma_fixed", C.c_int32), ("time_limit", C.c_double), ("eig_factor", C.c_double),
        ("check_iter", C.c_int32), ("warm_up", C.c_int32),
        ("spmv_mode_Q", C.c_int32), ("spmv_mode_A", C.c_int32),
        ("print_frequency", C.c_int32), ("device_number", C.c_int32),
        ("use_Ruiz_scaling", C.c_int32), ("use_bc_scaling", C.c_int32),
        ("use_l2_scaling", C.c_int32), ("use_Pock_Chambolle_scaling", C.c_int32),
        ("problem_type", C.c_int32), ("lambda_", C.c_double),
        ("auto_save", C.c_int32), ("verbose", C.c_int32), ("use_gpu", C.c_int32),
        ("precision", C.c_int32), ("polish_tol", C.c_double),
        ("lambda_max_A_override", C.c_double), ("lambda_max_Q_override", C.c_double),
        ("profile_passes", C.c_int32),
    ]


class Result(C.Structure):
    _fields_ = [
        ("iter", C.c_int64), ("iter_4", C.c_int64), ("iter_6", C.c_int64),
        ("time", C.c_double), ("time_4", C.c_double), ("time_6", C.c_double),
        ("power_time", C.c_double), ("setup_time", C.c_double),
        ("primal_obj", C.c_double), ("dual_obj", C.c_double),
        ("residuals", C.c_double), ("gap", C.c_double),
        ("err_Rp", C.c_double), ("err_Rd", C.c_double),
        ("status", C.c_int32), ("Q_is_diag", C.c_int32),
        ("sigma", C.c_double), ("lambda_max_A", C.c_double), ("lambda_max_Q", C.c_double),
        ("restarts", C.c_int64), ("iter_fp32", C.c_int64), ("gpu_launches", C.c_int64),
        ("device_time", C.c_double), ("h2d_bytes", C.c_int64), ("d2h_bytes", C.c_int64),
        ("power_iter_A", C.c_int64), ("power_iter_Q", C.c_int64), ("power_bytes", C.c_double),
    ]


MAX_PASSES = 8


class PassStats(C.Structure):
    _fields_ = [
        ("npass", C.c_int32), ("path", C.c_int32),
        ("name", (C.c_char * 32) * MAX_PASSES),
        ("ms_per_launch", C.c_double * MAX_PASSES),
        ("bytes_per_launch", C.c_double * MAX_PASSES),
        ("threads_per_row", C.c_int32 * MAX_PASSES),
        ("ms_per_iter", C.c_double), ("bytes_per_iter", C.c_double), ("iters", C.c_int64),
        ("ms_back_to_back", C.c_double * MAX_PASSES),
    ]


def default_params():
    """HPRQP_parameters() defaults (reference src/structs.jl:274)."""
    p = Params()
    p.stoptol = 1e-6
    p.sigma = -1.0
    p.max_iter = 2**31 - 1
    p.sigma_fixed = 0
    p.time_limit = 3600.0
    p.eig_factor = 1.05
    p.check_iter = 100
    p.warm_up = 0
    p.spmv_mode_Q = 0
    p.spmv_mode_A = 0
    p.print_frequency = -1
    p.device_number = 0
    p.use_Ruiz_scaling = 1
    p.use_bc_scaling = 0
    p.use_l2_scaling = 0
    p.use_Pock_Chambolle_scaling = 1
    p.problem_type = 0
    p.lambda_ = 0.0
    p.auto_save = 0
    p.verbose = 1
    p.use_gpu = 1
    p.precision = 0
    p.polish_tol = -1.0
    p.lambda_max_A_override = -1.0
    p.lambda_max_Q_override = -1.0
    p.profile_passes = 0
    return p


def _ptr(arr, ctype):
    return arr.ctypes.data_as(C.POINTER(ctype)) if arr is not None else None


class ProblemView:
    """Owns contiguous numpy copies of a problem and a Problem struct that
    points into them (the struct is only valid while this object lives)."""

    def __init__(self, model):
        import numpy as np
        f64 = lambda v: None if v is None else np.ascontiguousarray(v, dtype=np.float64)
        i32 = lambda v: None if v is None else np.ascontiguousarray(v, dtype=np.int32)
        s = Problem()
        self._keep = []

        def keep(a):
            self._keep.append(a)
            return a

        s.n, s.m = model.n, model.m
        s.index_base = 0
        A = model.A.tocsc()
        A.sort_indices()
        s.A_colptr = _ptr(keep(i32(A.indptr)), C.c_int32)
        s.A_rowval = _ptr(keep(i32(A.indices)), C.c_int32)
        s.A_nzval = _ptr(keep(f64(A.data)), C.c_double)
        for name in ("c", "AL", "AU", "l", "u"):
            setattr(s, name, _ptr(keep(f64(getattr(model, name))), C.c_double))
        s.obj_constant = float(model.obj_constant)
        s.lambda_ = float(model.lambda_)
        Q = model.Q
        kind = Q.kind
        s.Q_kind = kind
        if kind == Q_SPARSE:
            Qc = Q.Q.tocsc()
            Qc.sort_indices()
            s.Q_colptr = _ptr(keep(i32(Qc.indptr)), C.c_int32)
            s.Q_rowval = _ptr(keep(i32(Qc.indices)), C.c_int32)
            s.Q_nzval = _ptr(keep(f64(Qc.data)), C.c_double)
        elif kind == Q_LASSO:
            L = Q.A.tocsc()
            L.sort_indices()
            s.lasso_m = L.shape[0]
            s.L_colptr = _ptr(keep(i32(L.indptr)), C.c_int32)
            s.L_rowval = _ptr(keep(i32(L.indices)), C.c_int32)
            s.L_nzval = _ptr(keep(f64(L.data)), C.c_double)
        elif kind == Q_QAP:
            s.qap_n = Q.n
            for name in ("A", "B", "S", "T"):
                arr = keep(np.asfortranarray(getattr(Q, name), dtype=np.float64))
                setattr(s, "qap_" + name, _ptr(arr, C.c_double))
        self.struct = s
