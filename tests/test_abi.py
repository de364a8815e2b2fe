"""CPU tests of the C-ABI boundary: the library loads, exports every entry
point declared in include/hprqp.h, its struct layouts match the ctypes
mirrors, and without a GPU it refuses to run (no CPU fallback)."""
import ctypes as C
import os
import re

import pytest

from hprqp_b200 import _abi, _lib
from tests.conftest import ROOT, gpu_available


def declared_entry_points(header="hprqp.h"):
    src = open(os.path.join(ROOT, "include", header)).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(hprqp_[a-z0-9_]+)\s*\(", src)))


HEADERS = sorted(f for f in os.listdir(os.path.join(ROOT, "include")) if f.endswith(".h"))


def test_header_declares_all_bound_exports():
    decl = declared_entry_points()
    assert set(_lib.EXPORTS) == set(decl), decl


@pytest.mark.parametrize("header", HEADERS)
def test_library_exports_every_declared_symbol(lib_built, header):
    L = C.CDLL(lib_built)
    names = declared_entry_points(header)
    assert names, header
    for name in names:
        assert hasattr(L, name), (header, name)


def test_struct_layouts_match(lib_built):
    L = _lib.load()
    out = (C.c_int64 * 4)()
    assert L.hprqp_abi_info(out) == 0
    assert out[0] == 1
    assert out[1] == C.sizeof(_abi.Problem)
    assert out[2] == C.sizeof(_abi.Params)
    assert out[3] == C.sizeof(_abi.Result)


def test_default_params_match_reference(lib_built):
    L = _lib.load()
    p = _abi.Params()
    L.hprqp_default_params(C.byref(p))
    q = _abi.default_params()
    for f, _ in _abi.Params._fields_:
        assert getattr(p, f) == getattr(q, f), f
    # src/structs.jl:274
    assert p.stoptol == 1e-6 and p.sigma == -1 and p.max_iter == 2**31 - 1 and p.time_limit == 3600.0
    assert p.eig_factor == 1.05 and p.check_iter == 100 and p.print_frequency == -1
    assert p.use_Ruiz_scaling == 1 and p.use_Pock_Chambolle_scaling == 1 and p.use_bc_scaling == 0


@pytest.mark.skipif(gpu_available(), reason="checks the no-GPU error path")
def test_no_gpu_is_an_error_not_a_fallback(lib_built):
    L = _lib.load()
    h = C.c_void_p()
    rc = L.hprqp_create(C.byref(h), 0)
    assert rc == _abi.HPRQP_E_CUDA
    assert b"CUDA" in L.hprqp_last_error(None)
    from hprqp_b200 import optimize
    from hprqp_b200 import workloads as W
    with pytest.raises(_lib.HPRQPError):
        optimize(W.toy_qp())


@pytest.mark.parametrize("m,n", [(1 << 20, 1 << 20), (1 << 62, 1), (1, 1 << 62), ((1 << 19) + 1, 0 + 1)])
def test_power_lambda_noalloc_rejects_oversize(lib_built, m, n):
    """The size check of the allocation-free entry point runs before any CUDA
    call or dereference, so it is exercised here without a GPU; sizes that
    would overflow 2m + n are rejected as well."""
    L = _lib.load()
    lam, its = C.c_double(), C.c_int32()
    dummy = C.c_void_p(8)  # never dereferenced: the size check comes first
    rc = L.hprqp_power_lambda_noalloc(m, n, dummy, dummy, dummy, dummy, dummy, dummy, 1, 1e-4, 10, None,
                                      C.byref(lam), C.byref(its))
    assert rc == _abi.HPRQP_E_ARG
    assert b"too large" in L.hprqp_last_error(None)
    with pytest.raises(_lib.HPRQPError):
        _lib.check(rc)
