/*
 * hprqp.h — C ABI of libhprqp.so, the B200 (sm_100a) iteration engine of the
 * HPR-QP solver (dual Halpern Peaceman–Rachford method for convex composite
 * quadratic programs).
 *
 *     minimize    0.5 x'Qx + c'x + obj_constant  [+ lambda*||x||_1 for LASSO]
 *     subject to  AL <= A x <= AU,   l <= x <= u
 *
 * The library replaces the `use_gpu = true` branch of the reference solver's
 * `solve(model, params)` (src/algorithm.jl:1904-2039): everything after
 * `prepare_model` (src/algorithm.jl:1326-1333) — scaling, eigenvalue
 * estimation, warm start, the HPR loop, residuals, restarts, sigma updates
 * and result collection — runs behind these entry points.  A Julia `ccall`
 * shim (julia/HPRQPGPU.jl) or Python `ctypes` (hprqp_b200/_lib.py) binds it.
 *
 * Conventions
 *  - Plain C types only; no exceptions cross the boundary.  Every function
 *    returns 0 on success and a negative HPRQP_E* code on failure; the text
 *    of the last failure is available from hprqp_last_error().
 *  - The caller owns every host array.  hprqp_load() copies what it needs;
 *    output arrays are caller-allocated.
 *  - There is NO CPU fallback: if CUDA is unusable or the device number is
 *    invalid, hprqp_create() fails with HPRQP_E_CUDA.  (The reference's
 *    validate_gpu_parameters!, src/utils.jl:14-31, silently falls back to the
 *    CPU instead.)
 *  - A handle is not thread-safe; use one handle per host thread.
 */
#ifndef HPRQP_H
#define HPRQP_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HPRQP_ABI_VERSION 1

/* ---- return codes -------------------------------------------------------- */
#define HPRQP_OK             0
#define HPRQP_E_ARG         -1   /* invalid argument (sizes, NaN data, l > u, ...) */
#define HPRQP_E_CUDA        -2   /* CUDA unusable / kernel launch or copy failed   */
#define HPRQP_E_OOM         -3   /* device allocation failed                        */
#define HPRQP_E_STATE       -4   /* call order (solve before load, ...)             */
#define HPRQP_E_UNSUPPORTED -5   /* option the library does not implement           */
#define HPRQP_E_CALLBACK    -6   /* the custom Q operator's callback returned nonzero */

/* ---- solver status (reference strings, src/algorithm.jl:558-576) --------- */
#define HPRQP_STATUS_OPTIMAL          0   /* "OPTIMAL"          */
#define HPRQP_STATUS_MAX_ITER         1   /* "MAX_ITER"         */
#define HPRQP_STATUS_TIME_LIMIT       2   /* "TIME_LIMIT"       */
#define HPRQP_STATUS_NUMERICAL_ERROR  3   /* NaN/Inf in a residual (new)    */

/* ---- kind of Q (the Q-operator plug-ins of src/Q_operators) ---------- */
#define HPRQP_Q_SPARSE 0   /* explicit sparse Q (may have 0 nonzeros: LP)      */
#define HPRQP_Q_LASSO  1   /* implicit Q = A_d' A_d  (LASSO_operator.jl)       */
#define HPRQP_Q_QAP    2   /* implicit Q(X) = 2(A X B - S X - X T) (QAP_operator.jl) */
#define HPRQP_Q_CUSTOM 3   /* user operator: Q x through a device callback (hprqp_set_qmap) */

/* ---- problem_type (reference params.problem_type string) ----------------- */
#define HPRQP_PROBLEM_QP    0
#define HPRQP_PROBLEM_LASSO 1
#define HPRQP_PROBLEM_QAP   2

/* ---- precision modes (new) ----------------------------------------------- */
#define HPRQP_PRECISION_FP64        0  /* plain FP64 HPR, the reference arithmetic */
#define HPRQP_PRECISION_FP32_POLISH 1  /* FP32 storage + FP64 anchors/reductions,
                                          then FP64 polish to the tolerance        */

/*
 * Problem data: the fields of the reference's QP_info_cpu
 * (src/structs.jl:98-149).  Sparse matrices are CSC with int32 indices, as a
 * Julia SparseMatrixCSC{Float64,Int32}; `index_base` is 1 for Julia arrays
 * passed as-is and 0 for scipy/C arrays.  Vectors are float64.  Infinite
 * bounds are +-INFINITY.
 */
typedef struct hprqp_problem {
    int64_t n;                 /* number of variables                          */
    int64_t m;                 /* number of rows of A (0 allowed)              */
    int32_t index_base;        /* 0 or 1, for every CSC array below            */
    int32_t Q_kind;            /* HPRQP_Q_*                                    */
    /* constraint matrix A (m x n), CSC */
    const int32_t* A_colptr;   /* n+1                                          */
    const int32_t* A_rowval;   /* nnz(A)                                       */
    const double*  A_nzval;    /* nnz(A)                                       */
    const double*  c;          /* n                                            */
    const double*  AL;         /* m                                            */
    const double*  AU;         /* m                                            */
    const double*  l;          /* n                                            */
    const double*  u;          /* n                                            */
    double obj_constant;
    double lambda;             /* LASSO regularisation (QP_info_cpu.lambda)    */
    /* HPRQP_Q_SPARSE: Q (n x n), CSC, symmetric (as left by qp_formulation)  */
    const int32_t* Q_colptr;
    const int32_t* Q_rowval;
    const double*  Q_nzval;
    /* HPRQP_Q_LASSO: data matrix A_d (lasso_m x n), CSC                       */
    int64_t lasso_m;
    const int32_t* L_colptr;
    const int32_t* L_rowval;
    const double*  L_nzval;
    /* HPRQP_Q_QAP: dense n_qap x n_qap column-major A, B, S, T; n = n_qap^2   */
    /* HPRQP_Q_CUSTOM: no Q data here; the operator comes from hprqp_set_qmap */
    int64_t qap_n;
    const double* qap_A;
    const double* qap_B;
    const double* qap_S;
    const double* qap_T;
} hprqp_problem;

/*
 * Solver parameters: every field of HPRQP_parameters (src/structs.jl:195-275),
 * strings mapped to ints, plus the library's own extensions at the end.
 * hprqp_default_params() gives the reference defaults (src/structs.jl:274).
 */
typedef struct hprqp_params {
    double  stoptol;                 /* 1e-6                                        */
    double  sigma;                   /* -1 = automatic (||b||/||c|| after scaling)  */
    int64_t max_iter;                /* typemax(Int32)                              */
    int32_t sigma_fixed;             /* 0                                           */
    double  time_limit;              /* 3600 s                                      */
    double  eig_factor;              /* 1.05                                        */
    int32_t check_iter;              /* 100                                         */
    int32_t warm_up;                 /* 0; accepted, no JIT to warm                 */
    int32_t spmv_mode_Q;             /* 0 = auto (autotuned row schedule); 1..6 =
                                        CSR with 1,2,4,...,32 threads per row;
                                        7 = SELL-32; 8 = ELL (short rows); 9 = row
                                        split (long rows cut into equal pieces,
                                        one warp each; CSR where no row is long);
                                        10 = staged column blocks (the input
                                        vector's blocks in shared memory, 16-bit
                                        columns; CSR where the matrix is small,
                                        its rows short or its input too long)      */
    int32_t spmv_mode_A;             /* same, for A and A'                          */
    int32_t print_frequency;         /* -1 = adaptive (print_step)                  */
    int32_t device_number;           /* 0                                           */
    int32_t use_Ruiz_scaling;        /* 1                                           */
    int32_t use_bc_scaling;          /* 0 (disabled in the reference, utils.jl:703) */
    int32_t use_l2_scaling;          /* 0 (never read by the reference algorithm)   */
    int32_t use_Pock_Chambolle_scaling; /* 1                                        */
    int32_t problem_type;            /* HPRQP_PROBLEM_*; L1 term in the objective
                                        only when LASSO (algorithm.jl:66)           */
    double  lambda;                  /* params.lambda: never read (reference quirk) */
    int32_t auto_save;               /* 1: write a checkpoint at every printed
                                        iteration and at the end (the reference's
                                        HDF5 datasets in the library's container,
                                        to the file of hprqp_set_save_file)        */
    int32_t verbose;                 /* 1: iteration log on stdout                  */
    int32_t use_gpu;                 /* must be 1 for this library                  */
    /* ---- extensions ---- */
    int32_t precision;               /* HPRQP_PRECISION_*                           */
    double  polish_tol;              /* FP32 phase stops when KKT < polish_tol
                                        (<= 0: automatic)                           */
    double  lambda_max_A_override;   /* > 0: use instead of power iteration         */
    double  lambda_max_Q_override;   /* > 0: use instead of power iteration         */
    int32_t profile_passes;          /* 1: time each fused pass of plain iterations
                                        with CUDA events during the solve (read
                                        them with hprqp_get_pass_stats)            */
} hprqp_params;

/* Results: HPRQP_results (src/structs.jl:292-309) minus the vectors, which go
 * to caller-allocated arrays in hprqp_solve(). */
typedef struct hprqp_result {
    int64_t iter, iter_4, iter_6;
    double  time, time_4, time_6;    /* seconds from t_start_alg (after setup)     */
    double  power_time, setup_time;
    double  primal_obj, dual_obj;
    double  residuals;               /* max(err_Rp, err_Rd, gap) (KKT)              */
    double  gap, err_Rp, err_Rd;
    int32_t status;                  /* HPRQP_STATUS_*                              */
    int32_t Q_is_diag;
    double  sigma;                   /* final sigma                                 */
    double  lambda_max_A, lambda_max_Q;
    int64_t restarts;
    int64_t iter_fp32;               /* iterations done in the FP32 phase           */
    int64_t gpu_launches;            /* kernels launched by this solve              */
    double  device_time;             /* CUDA-event time of the same span as `time`  */
    int64_t h2d_bytes, d2h_bytes;    /* host<->device bytes moved by this call      */
    int64_t power_iter_A, power_iter_Q; /* power-method steps of the two chains     */
    double  power_bytes;             /* algorithmic HBM bytes of those steps         */
} hprqp_result;

/* Per-pass timing of the hot loop (hprqp_profile_iterations). */
#define HPRQP_MAX_PASSES 8
typedef struct hprqp_pass_stats {
    int32_t npass;
    int32_t path;                        /* 0 QP, 1 QP-noC, 2 LP, 3 LASSO           */
    char    name[HPRQP_MAX_PASSES][32];
    double  ms_per_launch[HPRQP_MAX_PASSES];    /* CUDA events, averaged           */
    double  bytes_per_launch[HPRQP_MAX_PASSES]; /* algorithmic HBM bytes           */
    int32_t threads_per_row[HPRQP_MAX_PASSES];
    double  ms_per_iter;                 /* whole iteration, timed without per-pass events */
    double  bytes_per_iter;
    int64_t iters;
    double  ms_back_to_back[HPRQP_MAX_PASSES]; /* hprqp_profile_iterations only: the
                                        pass kernel launched alone, back to back
                                        (programmatic dependent launch as in the
                                        loop), per launch; 0 when not measured */
} hprqp_pass_stats;

typedef struct hprqp_ctx* hprqp_handle;

/* ---- entry points -------------------------------------------------------- */

/* ABI self-description: out[0] = HPRQP_ABI_VERSION, out[1..3] =
 * sizeof(hprqp_problem), sizeof(hprqp_params), sizeof(hprqp_result).  Lets
 * a binding check its struct layouts.  No reference counterpart. */
int hprqp_abi_info(int64_t* out);

/* Reference defaults, HPRQP_parameters() (src/structs.jl:274). */
void hprqp_default_params(hprqp_params* p);

/* Bind a handle to CUDA device `device`.  Replaces validate_gpu_parameters! +
 * CUDA.device! (src/utils.jl:14-31, src/algorithm.jl:1910-1912); an unusable
 * device is an error, not a CPU fallback. */
int hprqp_create(hprqp_handle* h, int32_t device);

/* Copy a problem (QP_info_cpu, src/structs.jl:98-149) into the handle.
 * Validates sizes, index ranges, NaN and l <= u, AL <= AU.  Replaces
 * transfer_to_gpu (src/algorithm.jl:1284-1322) and the Q plug-ins' to_gpu
 * (src/Q_operators). */
int hprqp_load(hprqp_handle h, const hprqp_problem* prob);

/* Setup only: scaling!, check_Q_diagonal, workspace allocation, upload and
 * SpMV schedule selection (src/algorithm.jl:1914-1935).  Optional: hprqp_solve
 * performs it when the handle is not prepared for these params.  Lets a
 * caller time the iteration engine with the data already resident. */
int hprqp_prepare(hprqp_handle h, const hprqp_params* params);

/* optimize(model, params) for the loaded problem (src/algorithm.jl:1511-1554
 * and 1904-2039).  initial_x (length n) / initial_y (length m) may be NULL
 * (params.initial_x / initial_y = nothing).  x, z, w (length n) and y
 * (length m) receive the unscaled solution (collect_results!,
 * src/algorithm.jl:611-643); any of them may be NULL. */
int hprqp_solve(hprqp_handle h, const hprqp_params* params,
                const double* initial_x, const double* initial_y,
                hprqp_result* result,
                double* x, double* y, double* z, double* w);

/* The file params.auto_save writes (the reference's save_filename,
 * src/structs.jl:195-275; default "hprqp_autosave.ckpt").  save_state_to_hdf5!
 * (src/algorithm.jl:183-301) writes HDF5; this library writes the same
 * datasets (current/..., best/..., parameters/...) into its own container
 * of named arrays (a u16-length name, a type byte, a u64 count and the
 * little-endian payload per record after the magic "HPRQPCK1";
 * hprqp_b200/checkpoint.py reads it), written to <path>.tmp and renamed,
 * plus a resume/... section for hprqp_solve_resume. */
int hprqp_set_save_file(hprqp_handle h, const char* path);

/* Continue a solve from a checkpoint written by params.auto_save for the
 * loaded problem (no reference counterpart: the reference writes its
 * checkpoints but cannot continue from them).  The scaled state, sigma,
 * lambda_max and the restart records come from the file, so the continued
 * solve takes exactly the steps the interrupted one would have taken after
 * the checkpoint's iteration.  `params` may change max_iter, time_limit,
 * stoptol and the like; the scaling parameters must be those of the
 * checkpoint.  A checkpoint of a solve that ended OPTIMAL (or in a
 * numerical error) is rejected; one of the FP32 phase needs precision
 * HPRQP_PRECISION_FP32_POLISH.  Results as hprqp_solve; iter counts the
 * iterations of both parts. */
int hprqp_solve_resume(hprqp_handle h, const hprqp_params* params, const char* path, hprqp_result* result,
                       double* x, double* y, double* z, double* w);

/* Parity hook: record the scaled working iterates x, y, w after each of the
 * first `iters` HPR iterations of the next hprqp_solve() into caller-owned
 * arrays of iters*n, iters*m, iters*n doubles (NULL entries are skipped).
 * iters = 0 disables tracing.  Tracing synchronises every iteration. */
int hprqp_set_trace(hprqp_handle h, int64_t iters,
                    double* x_trace, double* y_trace, double* w_trace);

/* Parity hook, beside hprqp_set_trace: for each traced iteration k
 * (k < iters of the last hprqp_set_trace) record the sigma the step used
 * (after update_sigma!, src/algorithm.jl:323-423) and the inner counter of
 * its Halpern weight 1/(inner + 2) (0 right after a restart, do_restart!,
 * src/algorithm.jl:522-555).  Arrays of `iters` entries; NULL disables. */
int hprqp_set_trace_scalars(hprqp_handle h, double* sigma_trace, int64_t* inner_trace);

/* Measurement hook: prepare, estimate lambda_max, then run `iters` plain
 * (partial, `full` = 0) or full HPR iterations of the loaded problem from
 * the zero state and report the CUDA-event time and the algorithmic bytes
 * of each fused pass.  Used by bench.py for the roofline; no reference
 * counterpart. */
int hprqp_profile_iterations(hprqp_handle h, const hprqp_params* params, int64_t iters,
                             int32_t full, hprqp_pass_stats* out);

/* Per-pass CUDA-event timings collected by the last hprqp_solve() run with
 * params.profile_passes = 1: one hprqp_pass_stats per engine precision
 * (fp64, fp32; npass = 0 when that engine did not run). */
int hprqp_get_pass_stats(hprqp_handle h, hprqp_pass_stats* fp64, hprqp_pass_stats* fp32);

/* A user's Q operator (an AbstractQOperator with its own Qmap!,
 * src/Q_operators/Q_operator_interface.jl:33-92): Qx = Q x for n-vectors in
 * device memory, FP64 (precision 0: x, Qx are double*) or FP32 (precision 1:
 * float*, the FP32 phase of HPRQP_PRECISION_FP32_POLISH), enqueued on
 * `stream` (a cudaStream_t); x must not be changed.  The library calls it
 * from the solving thread wherever the method applies Q: twice per HPR
 * iteration on the QP path, in the residuals, the M-norm and the sigma
 * update, and in every step of the power method on Q (give
 * lambda_max_Q_override to skip that).  Returns 0, or nonzero to stop the
 * solve with HPRQP_E_CALLBACK.  As for the reference's operators, Q must be
 * symmetric positive semidefinite, and an operator Q gets no scaling
 * (src/utils.jl:364-406). */
typedef int32_t (*hprqp_qmap_fn)(const void* x, void* Qx, int32_t precision, void* user, void* stream);

/* Bind the Q operator of a loaded HPRQP_Q_CUSTOM problem (replaces the
 * reference's to_gpu + Qmap! of a custom operator type); `user` is passed
 * back to every call.  Must follow hprqp_load and precede hprqp_prepare /
 * hprqp_solve of that problem; hprqp_load drops the binding. */
int hprqp_set_qmap(hprqp_handle h, hprqp_qmap_fn qmap, void* user);

/* lambda_max(A A') by the power method, for a CSR matrix A (m x n, int32,
 * 0-based) and its transpose A' (n x m) that the caller already holds in
 * device memory.  It allocates nothing; use it when device memory cannot be
 * allocated where the estimate is needed: in a program whose device memory
 * belongs to another framework's pool allocator, or in a loop that must not
 * allocate after start-up.  No counterpart in the reference.
 *  - Scratch: a fixed block inside the library (8 MiB of work vectors plus
 *    256 KiB of control), reserved on every GPU that loads the library until
 *    the process exits.  Requires 2m + n <= 1,048,576; larger problems get
 *    HPRQP_E_ARG with the reason in hprqp_last_error(NULL).
 *  - The first call in each CUDA context (a device's primary context, or
 *    one the caller made current) looks up the scratch address there; make
 *    that call before any stream capture.
 *  - All calls share the scratch: calls that overlap on the GPU (different
 *    streams, threads or processes on one device) race.  Each call clears
 *    what must start at zero.
 *  - Same start vector, products and stopping test (err < tol, at most
 *    max_iter steps) as the solver's power method (threads_per_row 1..32
 *    selects the CSR schedule), so lambda agrees with hprqp_solve's
 *    lambda_max_A / eig_factor for the same matrix to rounding (the solver
 *    sums its dot products in another order).  When max_iter ends the
 *    method, lambda is that step's estimate and *iters_out = max_iter.
 *  - stream: a cudaStream_t (NULL = legacy default stream); the call
 *    returns after the stream has finished the work.  */
int hprqp_power_lambda_noalloc(int64_t m, int64_t n,
                               const int32_t* A_rowptr, const int32_t* A_colind, const double* A_val,
                               const int32_t* AT_rowptr, const int32_t* AT_colind, const double* AT_val,
                               int32_t threads_per_row, double tol, int32_t max_iter,
                               void* stream, double* lambda_out, int32_t* iters_out);

/* C = alpha * A * B + beta * C for N x N column-major FP32 matrices in
 * device memory, as a 3xTF32 split-precision GEMM on the tensor cores
 * (tcgen05, FP32 accumulate): the product kernel of the QAP operator
 * (src/Q_operators/QAP_operator.jl:52-61) in the FP32 phase, where the
 * reference calls a cuBLAS GEMM.  Returns after the stream has finished;
 * HPRQP_E_CUDA if a bounded wait inside the kernel gave up. */
int hprqp_gemm_3xtf32(int32_t n, float alpha, const float* A, const float* B, float beta, float* C,
                      void* stream);

/* The same product with a caller-owned workspace `ws` of
 * hprqp_gemm_3xtf32_ws_floats(n) floats (device memory) that holds the
 * operands pre-split into TF32 hi/lo images; enqueued on `stream` without
 * synchronising (a timed-out internal wait is reported by the next
 * hprqp_gemm_3xtf32 call). */
int64_t hprqp_gemm_3xtf32_ws_floats(int32_t n);
int hprqp_gemm_3xtf32_ws(int32_t n, float alpha, const float* A, const float* B, float beta, float* C, float* ws,
                         void* stream);

/* Text of the last error on this handle ("" if none); valid until the next
 * call on the handle.  h may be NULL for errors from hprqp_create. */
const char* hprqp_last_error(hprqp_handle h);

/* Free every device and host resource of the handle. */
int hprqp_destroy(hprqp_handle h);

#ifdef __cplusplus
}
#endif
#endif /* HPRQP_H */
