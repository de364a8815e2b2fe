# HPRQPGPU.jl — Julia binding of libhprqp.so (include/hprqp.h) for HPR-QP.
#
# Drop-in for the `params.use_gpu == true` branch of HPRQP.solve
# (src/algorithm.jl:1904-2039): the model built by build_from_* (QP_info_cpu)
# crosses the C ABI unchanged — CSC arrays are passed as-is with
# index_base = 1 — and the library returns an HPRQP_results-shaped record.
# CUDA.jl, cuSPARSE and KernelAbstractions are not involved.
#
# Include it inside module HPRQP, after structs.jl:
#     include(joinpath(@__DIR__, "..", "..", "hprqp_b200_repo", "julia", "HPRQPGPU.jl"))
# (any path to this file), so that solve_gpu returns HPRQP.HPRQP_results.
#
# This file is not executed in the build container (no Julia there); the
# same ABI is exercised from Python (hprqp_b200/_lib.py) by the test-suite,
# and tests/test_julia_shim.py checks this file's struct mirrors and result
# fields against include/hprqp.h and the reference's HPRQP_results.

module HPRQPGPU

using SparseArrays

const libhprqp = get(ENV, "HPRQP_LIB", joinpath(@__DIR__, "..", "hprqp_b200", "libhprqp.so"))

const Q_SPARSE, Q_LASSO, Q_QAP, Q_CUSTOM = Int32(0), Int32(1), Int32(2), Int32(3)
const E_CALLBACK = -6
const STATUS = Dict(0 => "OPTIMAL", 1 => "MAX_ITER", 2 => "TIME_LIMIT", 3 => "NUMERICAL_ERROR")

# mirrors `hprqp_problem`
struct CProblem
    n::Int64
    m::Int64
    index_base::Int32
    Q_kind::Int32
    A_colptr::Ptr{Int32}
    A_rowval::Ptr{Int32}
    A_nzval::Ptr{Float64}
    c::Ptr{Float64}
    AL::Ptr{Float64}
    AU::Ptr{Float64}
    l::Ptr{Float64}
    u::Ptr{Float64}
    obj_constant::Float64
    lambda::Float64
    Q_colptr::Ptr{Int32}
    Q_rowval::Ptr{Int32}
    Q_nzval::Ptr{Float64}
    lasso_m::Int64
    L_colptr::Ptr{Int32}
    L_rowval::Ptr{Int32}
    L_nzval::Ptr{Float64}
    qap_n::Int64
    qap_A::Ptr{Float64}
    qap_B::Ptr{Float64}
    qap_S::Ptr{Float64}
    qap_T::Ptr{Float64}
end

# mirrors `hprqp_params`
mutable struct CParams
    stoptol::Float64
    sigma::Float64
    max_iter::Int64
    sigma_fixed::Int32
    time_limit::Float64
    eig_factor::Float64
    check_iter::Int32
    warm_up::Int32
    spmv_mode_Q::Int32
    spmv_mode_A::Int32
    print_frequency::Int32
    device_number::Int32
    use_Ruiz_scaling::Int32
    use_bc_scaling::Int32
    use_l2_scaling::Int32
    use_Pock_Chambolle_scaling::Int32
    problem_type::Int32
    lambda::Float64
    auto_save::Int32
    verbose::Int32
    use_gpu::Int32
    precision::Int32
    polish_tol::Float64
    lambda_max_A_override::Float64
    lambda_max_Q_override::Float64
    profile_passes::Int32
end

# mirrors `hprqp_result`
mutable struct CResult
    iter::Int64; iter_4::Int64; iter_6::Int64
    time::Float64; time_4::Float64; time_6::Float64
    power_time::Float64; setup_time::Float64
    primal_obj::Float64; dual_obj::Float64
    residuals::Float64; gap::Float64; err_Rp::Float64; err_Rd::Float64
    status::Int32; Q_is_diag::Int32
    sigma::Float64; lambda_max_A::Float64; lambda_max_Q::Float64
    restarts::Int64; iter_fp32::Int64; gpu_launches::Int64
    device_time::Float64; h2d_bytes::Int64; d2h_bytes::Int64
    power_iter_A::Int64; power_iter_Q::Int64; power_bytes::Float64
    CResult() = new()
end

i32(v) = convert(Vector{Int32}, v)
lasterr(h) = unsafe_string(ccall((:hprqp_last_error, libhprqp), Cstring, (Ptr{Cvoid},), h))
check(rc, h) = rc == 0 || error("libhprqp error $rc: $(lasterr(h))")

function cparams(p)
    c = CParams(zeros(26)...)  # filled by hprqp_default_params, then overwritten
    ccall((:hprqp_default_params, libhprqp), Cvoid, (Ref{CParams},), c)
    c.stoptol = p.stoptol; c.sigma = p.sigma; c.max_iter = p.max_iter
    c.sigma_fixed = p.sigma_fixed; c.time_limit = p.time_limit; c.eig_factor = p.eig_factor
    c.check_iter = p.check_iter; c.warm_up = p.warm_up; c.print_frequency = p.print_frequency
    c.device_number = p.device_number
    c.use_Ruiz_scaling = p.use_Ruiz_scaling; c.use_bc_scaling = p.use_bc_scaling
    c.use_l2_scaling = p.use_l2_scaling; c.use_Pock_Chambolle_scaling = p.use_Pock_Chambolle_scaling
    c.problem_type = p.problem_type == "LASSO" ? 1 : p.problem_type == "QAP" ? 2 : 0
    c.lambda = p.lambda; c.auto_save = p.auto_save; c.verbose = p.verbose; c.use_gpu = 1
    return c
end

# The reference's result type, HPRQP_results (src/structs.jl:292-309).  This
# file is include()d inside module HPRQP after structs.jl (see the seam in
# INTEGRATION.md), so the type is the parent module's own; a caller that
# includes it elsewhere passes the type explicitly.
function _results_type()
    parent = parentmodule(@__MODULE__)
    isdefined(parent, :HPRQP_results) || error("HPRQPGPU: include this file inside module HPRQP, " *
                                               "or pass results_type = HPRQP.HPRQP_results")
    return getfield(parent, :HPRQP_results)
end

# ---------------------------------------------------------------------------
# Custom Q operators (the reference's AbstractQOperatorCPU / AbstractQOperator
# with their own to_gpu and Qmap!, src/Q_operators/Q_operator_interface.jl:
# 33-92) cross the C ABI as a device callback (hprqp_set_qmap).  Their Qmap!
# works on CuVectors, so this path uses CUDA.jl, which the enclosing module
# HPRQP already loads; the built-in operators need no CUDA.jl.
# ---------------------------------------------------------------------------
_parent(name) = getfield(parentmodule(@__MODULE__), name)

mutable struct QmapCtx
    Qgpu::Any   # to_gpu(Q_cpu) of the user's operator
    n::Int
    err::Any    # an exception raised inside the callback, rethrown by solve_gpu
end

# hprqp_qmap_fn: Qx = Q x on n-vectors in device memory, precision 0 = Float64,
# 1 = Float32 (the FP32 phase), ordered after the library's stream.
function qmap_thunk(x::Ptr{Cvoid}, Qx::Ptr{Cvoid}, precision::Int32, user::Ptr{Cvoid}, stream::Ptr{Cvoid})::Int32
    ctx = unsafe_pointer_to_objref(user)::QmapCtx
    try
        CU = _parent(:CUDA)
        CU.cuStreamSynchronize(reinterpret(CU.CUstream, stream))  # the library's writes of x are done
        T = precision == 0 ? Float64 : Float32
        xv = unsafe_wrap(CU.CuArray, CU.CuPtr{T}(UInt(x)), ctx.n)
        yv = unsafe_wrap(CU.CuArray, CU.CuPtr{T}(UInt(Qx)), ctx.n)
        if T === Float64
            _parent(:Qmap!)(xv, yv, ctx.Qgpu)
        else  # the reference's operators compute in Float64
            y64 = CU.zeros(Float64, ctx.n)
            _parent(:Qmap!)(Float64.(xv), y64, ctx.Qgpu)
            yv .= Float32.(y64)
        end
        CU.synchronize()  # Qx is complete before the library's next kernel reads it
        return Int32(0)
    catch e
        ctx.err = e
        return Int32(-1)
    end
end

"""
    solve_gpu(model::QP_info_cpu, params::HPRQP_parameters) -> HPRQP_results

The GPU body of `solve` through libhprqp.  Returns the reference's own
`HPRQP_results` (src/structs.jl:292-309), every field filled, so that
`optimize` and `MOI.optimize!` (which stores it in a
`Union{Nothing,HPRQP_results}` field, src/MOI_wrapper.jl:63,494) work
unchanged.
"""
function solve_gpu(model, params; results_type = _results_type())
    m, n = size(model.A)
    A = model.A
    Acp, Arv = i32(A.colptr), i32(A.rowval)
    keep = Any[Acp, Arv, A.nzval, model.c, model.AL, model.AU, model.l, model.u]
    Qk = Q_SPARSE
    Qcp = Qrv = Ptr{Int32}(0); Qnz = Ptr{Float64}(0)
    lm = 0; Lcp = Lrv = Ptr{Int32}(0); Lnz = Ptr{Float64}(0)
    qn = 0; qA = qB = qS = qT = Ptr{Float64}(0)
    Q = model.Q
    qctx = nothing
    if Q isa SparseMatrixCSC
        a, b = i32(Q.colptr), i32(Q.rowval); push!(keep, a, b, Q.nzval)
        Qcp, Qrv, Qnz = pointer(a), pointer(b), pointer(Q.nzval)
    elseif nameof(typeof(Q)) == :LASSO_Q_operator_cpu
        Qk = Q_LASSO
        a, b = i32(Q.A.colptr), i32(Q.A.rowval); push!(keep, a, b, Q.A.nzval)
        lm = size(Q.A, 1); Lcp, Lrv, Lnz = pointer(a), pointer(b), pointer(Q.A.nzval)
    elseif nameof(typeof(Q)) == :QAP_Q_operator_cpu
        Qk = Q_QAP
        push!(keep, Q.A, Q.B, Q.S, Q.T)
        qn = Q.n; qA, qB, qS, qT = pointer(Q.A), pointer(Q.B), pointer(Q.S), pointer(Q.T)
    else  # a custom operator: its GPU form and the callback that applies it
        Qk = Q_CUSTOM
        qctx = QmapCtx(_parent(:to_gpu)(Q), n, nothing)
        push!(keep, qctx)
    end
    x = zeros(n); y = zeros(m); z = zeros(n); w = zeros(n)
    res = CResult()
    h = Ref{Ptr{Cvoid}}(C_NULL)
    GC.@preserve keep begin
        prob = CProblem(n, m, Int32(1), Qk, pointer(Acp), pointer(Arv), pointer(A.nzval),
                        pointer(model.c), pointer(model.AL), pointer(model.AU), pointer(model.l),
                        pointer(model.u), model.obj_constant, model.lambda,
                        Qcp, Qrv, Qnz, lm, Lcp, Lrv, Lnz, qn, qA, qB, qS, qT)
        check(ccall((:hprqp_create, libhprqp), Cint, (Ref{Ptr{Cvoid}}, Int32), h, params.device_number), C_NULL)
        try
            check(ccall((:hprqp_load, libhprqp), Cint, (Ptr{Cvoid}, Ref{CProblem}), h[], prob), h[])
            if params.auto_save  # the reference's save_filename; the library's container, same datasets
                check(ccall((:hprqp_set_save_file, libhprqp), Cint, (Ptr{Cvoid}, Cstring), h[],
                            params.save_filename), h[])
            end
            if Qk == Q_CUSTOM
                fn = @cfunction(qmap_thunk, Int32, (Ptr{Cvoid}, Ptr{Cvoid}, Int32, Ptr{Cvoid}, Ptr{Cvoid}))
                check(ccall((:hprqp_set_qmap, libhprqp), Cint, (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}),
                            h[], fn, pointer_from_objref(qctx)), h[])
            end
            x0 = params.initial_x === nothing ? C_NULL : pointer(params.initial_x)
            y0 = params.initial_y === nothing ? C_NULL : pointer(params.initial_y)
            GC.@preserve params begin
                rc = ccall((:hprqp_solve, libhprqp), Cint,
                           (Ptr{Cvoid}, Ref{CParams}, Ptr{Float64}, Ptr{Float64}, Ref{CResult},
                            Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}),
                           h[], cparams(params), x0, y0, res, x, y, z, w)
                if rc == E_CALLBACK && Qk == Q_CUSTOM && qctx.err !== nothing
                    throw(qctx.err)  # the user's Qmap! failed: its own exception
                end
                check(rc, h[])
            end
        finally
            ccall((:hprqp_destroy, libhprqp), Cint, (Ptr{Cvoid},), h[])
        end
    end
    # collect_results! / handle_termination (src/algorithm.jl:611-643,1039-1097)
    out = results_type()
    out.iter = res.iter
    out.iter_4 = res.iter_4
    out.iter_6 = res.iter_6
    out.time = res.time
    out.time_4 = res.time_4
    out.time_6 = res.time_6
    out.power_time = res.power_time
    out.primal_obj = res.primal_obj
    out.residuals = res.residuals
    out.gap = res.gap
    out.status = STATUS[res.status]
    out.x = x
    out.y = m > 0 ? y : Float64[]
    out.z = z
    out.w = w
    return out
end

end # module
