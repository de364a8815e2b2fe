"""CPU checks of the Julia binding julia/HPRQPGPU.jl (Julia is not installed
here, so the file is checked as text):

 - its struct mirrors CProblem, CParams and CResult have the fields of
   hprqp_problem, hprqp_params and hprqp_result in include/hprqp.h, in the
   same order and with matching types (a mismatch would corrupt every
   ccall);
 - a custom operator (the reference's AbstractQOperator with its own Qmap!)
   is bound through hprqp_set_qmap with a callback of the header's type;
 - solve_gpu builds and returns the reference's own HPRQP_results and fills
   every one of its fields (src/structs.jl:292-309), so that MOI.optimize!,
   which stores the result in a Union{Nothing,HPRQP_results} field
   (src/MOI_wrapper.jl:63,494), keeps working.
"""
import os
import re

from tests.conftest import ROOT

JL = os.path.join(ROOT, "julia", "HPRQPGPU.jl")
HDR = os.path.join(ROOT, "include", "hprqp.h")

# HPRQP_results (src/structs.jl:292-309), in declaration order
HPRQP_RESULTS_FIELDS = ["iter", "iter_4", "iter_6", "time", "time_4", "time_6", "power_time", "primal_obj",
                        "residuals", "gap", "status", "x", "y", "z", "w"]

C2JL = {"int64_t": "Int64", "int32_t": "Int32", "double": "Float64"}


def c_struct(name):
    src = re.sub(r"/\*.*?\*/", "", open(HDR).read(), flags=re.S)
    body = re.search(r"typedef struct %s \{(.*?)\} %s;" % (name, name), src, flags=re.S).group(1)
    fields = []
    for decl in body.split(";"):
        decl = decl.strip()
        if not decl:
            continue
        m = re.match(r"(const\s+)?(\w+)\s*(\*?)\s*(.*)", decl)
        base, ptr, names = m.group(2), m.group(3), m.group(4)
        for nm in names.split(","):
            nm = nm.strip().lstrip("*")
            jl = C2JL[base]
            fields.append((nm, f"Ptr{{{jl}}}" if ptr else jl))
    return fields


def jl_struct(name):
    src = open(JL).read()
    body = re.search(r"struct %s\n(.*?)\nend" % name, src, flags=re.S).group(1)
    fields = []
    for part in re.split(r"[;\n]", body):
        part = part.strip()
        m = re.match(r"(\w+)::([\w{}]+)$", part)
        if m:
            fields.append((m.group(1), m.group(2)))
    return fields


def test_struct_mirrors_match_header():
    for c_name, jl_name in (("hprqp_problem", "CProblem"), ("hprqp_params", "CParams"),
                            ("hprqp_result", "CResult")):
        c = c_struct(c_name)
        j = jl_struct(jl_name)
        assert [f for f, _ in c] == [f for f, _ in j], (c_name, c, j)
        assert c == j, (c_name, [(a, b) for a, b in zip(c, j) if a != b])


def test_solve_gpu_returns_reference_results_type():
    src = open(JL).read()
    body = src[src.index("function solve_gpu("):]
    body = body[:body.index("\nend\n")]
    assert re.search(r"out = results_type\(\)", body)
    assert re.search(r"return out\s*$", body.strip())
    assert "NamedTuple" not in body and "return (" not in body
    assigned = re.findall(r"out\.(\w+) = ", body)
    assert assigned == HPRQP_RESULTS_FIELDS, assigned
    # the default type is the reference's HPRQP_results of the enclosing module
    assert "getfield(parent, :HPRQP_results)" in src
    # custom operators: the callback has the header's hprqp_qmap_fn signature
    assert "@cfunction(qmap_thunk, Int32, (Ptr{Cvoid}, Ptr{Cvoid}, Int32, Ptr{Cvoid}, Ptr{Cvoid}))" in src
    assert "hprqp_set_qmap" in src and 'error("custom Q operators' not in src
    hdr = open(HDR).read()
    assert ("typedef int32_t (*hprqp_qmap_fn)(const void* x, void* Qx, int32_t precision, void* user, "
            "void* stream);") in hdr
    # statuses are the reference strings (src/algorithm.jl:558-576)
    assert '0 => "OPTIMAL"' in src and '1 => "MAX_ITER"' in src and '2 => "TIME_LIMIT"' in src


MOI_EXTRAS = os.path.join(ROOT, "julia", "MOI_extras.jl")

# HPRQP_parameters fields a user sets through MOI (src/structs.jl:195-275),
# with the three the reference's wrapper leaves out (src/MOI_wrapper.jl:141-163)
MOI_PARAMETERS = ["stoptol", "sigma", "max_iter", "sigma_fixed", "time_limit", "eig_factor", "check_iter",
                  "warm_up", "spmv_mode_Q", "spmv_mode_A", "print_frequency", "device_number", "use_Ruiz_scaling",
                  "use_bc_scaling", "use_l2_scaling", "use_Pock_Chambolle_scaling", "initial_x", "initial_y",
                  "auto_save", "save_filename", "verbose", "use_gpu", "problem_type", "lambda"]


def test_moi_extras_expose_the_missing_raw_attributes():
    src = open(MOI_EXTRAS).read()
    tup = re.search(r"const SUPPORTED_PARAMETERS = \((.*?)\n\)", src, flags=re.S).group(1)
    names = re.findall(r'"(\w+)"', tup)
    assert names == MOI_PARAMETERS, names
    for name in ("use_gpu", "problem_type", "lambda"):
        assert f'name == "{name}"' in src[src.index("function _set_extra!"):src.index("function _get_extra")]
        assert f'name == "{name}" && return model.params.{name}' in src


def test_moi_extras_constraint_primal_of_affine_rows():
    src = open(MOI_EXTRAS).read()
    body = src[src.index("function MOI.get(\n    model::Optimizer,\n    attr::MOI.ConstraintPrimal"):]
    assert "MOI.ScalarAffineFunction{Float64},<:SCALAR_SETS" in body
    assert "get_fallback" not in body
    assert "_row_activity(model)[c.value]" in body
    # the activity is A x from the cached constraint matrix and the returned x
    act = src[src.index("function _compute_row_activity"):]
    assert "model.cache.constraints.coefficients" in act and "model.results.x" in act
    assert "ax[A.rowval[k]] += A.nzval[k] * xj" in act
