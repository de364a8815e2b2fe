# MOI_extras.jl — additions to HPR-QP's MathOptInterface wrapper
# (src/MOI_wrapper.jl) that the GPU drop-in makes worth having:
#
#  1. ConstraintPrimal of affine rows.  The reference returns
#     MOI.Utilities.get_fallback for them (src/MOI_wrapper.jl:622-631),
#     which needs ConstraintFunction support the Optimizer does not have.
#     Here the row activity a_i' x is computed from the constraint matrix
#     the Optimizer already keeps in its cache (MatrixOfConstraints,
#     src/MOI_wrapper.jl:27-40; its row i is the ConstraintIndex value i,
#     as ConstraintDual assumes at :652-668) and the returned x.
#  2. Raw attributes "use_gpu", "problem_type" and "lambda".  The reference's
#     MOI.set already has a "use_gpu" branch but SUPPORTED_PARAMETERS
#     (src/MOI_wrapper.jl:141-163) omits it, so MOI.supports rejects it;
#     "problem_type" and "lambda" are HPRQP_parameters fields
#     (src/structs.jl:195-275) with no branch at all.
#
# This file is a patch, not a stand-alone module: Julia refuses to overwrite
# a method while a package precompiles, so a maintainer replaces, in
# src/MOI_wrapper.jl, the SUPPORTED_PARAMETERS tuple and the affine
# ConstraintPrimal method with the definitions below, and ends the `else`
# branches of MOI.set / MOI.get(::Optimizer, ::MOI.RawOptimizerAttribute)
# with `_set_extra!(model, name, value) || throw(MOI.UnsupportedAttribute(param))`
# and `return _get_extra(model, name, param)` (INTEGRATION.md shows where).
# Julia is not installed where this was written; tests/test_julia_shim.py
# checks it as text.

const SUPPORTED_PARAMETERS = (
    "stoptol",
    "sigma",
    "max_iter",
    "sigma_fixed",
    "time_limit",
    "eig_factor",
    "check_iter",
    "warm_up",
    "spmv_mode_Q",
    "spmv_mode_A",
    "print_frequency",
    "device_number",
    "use_Ruiz_scaling",
    "use_bc_scaling",
    "use_l2_scaling",
    "use_Pock_Chambolle_scaling",
    "initial_x",
    "initial_y",
    "auto_save",
    "save_filename",
    "verbose",
    "use_gpu",
    "problem_type",
    "lambda",
)

# The three parameters the reference's MOI.set / MOI.get branches lack (or
# that SUPPORTED_PARAMETERS hid): true when `name` was one of them.
function _set_extra!(model::Optimizer, name::String, value)
    if name == "use_gpu"
        model.params.use_gpu = Bool(value)
    elseif name == "problem_type"
        v = String(value)
        v in ("QP", "LASSO", "QAP") || throw(ArgumentError("problem_type must be \"QP\", \"LASSO\" or \"QAP\""))
        model.params.problem_type = v
    elseif name == "lambda"
        model.params.lambda = Float64(value)
    else
        return false
    end
    return true
end

function _get_extra(model::Optimizer, name::String, param)
    name == "use_gpu" && return model.params.use_gpu
    name == "problem_type" && return model.params.problem_type
    name == "lambda" && return model.params.lambda
    throw(MOI.UnsupportedAttribute(param))
end

# a_i' x for every row i of the cached constraint matrix (CSC, one-based),
# from the returned primal solution; computed once per result object (the
# results are a mutable HPRQP_results, so the weak key is its identity)
const _ROW_ACTIVITY = WeakKeyDict{Any,Vector{Float64}}()

function _row_activity(model::Optimizer)
    return get!(() -> _compute_row_activity(model), _ROW_ACTIVITY, model.results)
end

function _compute_row_activity(model::Optimizer)
    A = model.cache.constraints.coefficients
    x = model.results.x
    ax = zeros(Float64, A.m)
    @inbounds for j in 1:A.n
        xj = x[j]
        for k in A.colptr[j]:(A.colptr[j+1]-1)
            ax[A.rowval[k]] += A.nzval[k] * xj
        end
    end
    return ax
end

function MOI.get(
    model::Optimizer,
    attr::MOI.ConstraintPrimal,
    c::MOI.ConstraintIndex{MOI.ScalarAffineFunction{Float64},<:SCALAR_SETS},
)
    MOI.check_result_index_bounds(model, attr)
    if model.results === nothing
        error("No results available.")
    end
    if model.cache === nothing
        error("No problem has been loaded.")
    end
    # MOI keeps scalar affine constraints with a zero constant (a nonzero one
    # is ScalarFunctionConstantNotZero), so the row activity is the value of
    # the constraint function
    return _row_activity(model)[c.value]
end
