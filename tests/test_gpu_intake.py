"""GPU tests of the CSC intake (hprqp_load): the caller's CSC arrays become
the library's CSR copies of A, A', Q and Q' (csc_to_csr, csc_as_transpose).
Large matrices (64Ki entries and more) are transposed by a per-thread
histogram counting sort, small ones by the row-range scatter; both must give
the CSR a serial pass gives.

 - the same problem passed 0-based and sorted, 1-based, and with the row
   indices of every column shuffled (A and Q) solves to bit-identical
   iterates, at a size on each transpose path;
 - NaN entries, row indices out of range and crossed bounds are refused
   with the reference's messages, naming the first offending index.
"""
import ctypes as C

import numpy as np
import pytest

from hprqp_b200 import HPRQP_parameters, Solver
from hprqp_b200 import workloads as W
from hprqp_b200._abi import ProblemView, _ptr
from hprqp_b200._lib import HPRQPError, check

pytestmark = pytest.mark.gpu

SIZES = {"histogram": dict(n=20000, m=15000, density_A=0.0004, b_rows=800, density_B=0.001),
         "row-range": dict(n=300, m=200, density_A=0.02, b_rows=30, density_B=0.02)}


def load_view(model, edit=None):
    """A solver with `model` loaded through a ProblemView that `edit` may
    change (arrays it makes are kept alive by the view)."""
    s = Solver()
    v = ProblemView(model)
    if edit:
        edit(v)
    try:
        check(s._L.hprqp_load(s.h, C.addressof(v.struct)), s.h)
    except Exception:
        s.close()
        raise
    s.model = model
    return s


def shuffled_csc(M, rng):
    """The CSC arrays of M with the entries of every column in random order."""
    M = M.tocsc()
    M.sort_indices()
    rows, vals = M.indices.astype(np.int32).copy(), M.data.copy()
    for j in range(M.shape[1]):
        a, b = M.indptr[j], M.indptr[j + 1]
        if b - a > 1:
            p = a + rng.permutation(b - a)
            rows[a:b], vals[a:b] = rows[p], vals[p]
    return M.indptr.astype(np.int32), rows, vals


def set_csc(v, prefix, ptr, rows, vals):
    v._keep += [ptr, rows, vals]
    setattr(v.struct, prefix + "_colptr", _ptr(ptr, C.c_int32))
    setattr(v.struct, prefix + "_rowval", _ptr(rows, C.c_int32))
    setattr(v.struct, prefix + "_nzval", _ptr(vals, C.c_double))


def one_based(model):
    def edit(v):
        v.struct.index_base = 1
        for prefix, M in (("A", model.A), ("Q", model.Q.Q)):
            M = M.tocsc()
            M.sort_indices()
            set_csc(v, prefix, (M.indptr + 1).astype(np.int32), (M.indices + 1).astype(np.int32), M.data.copy())
    return edit


def unsorted(model):
    def edit(v):
        rng = np.random.default_rng(3)
        set_csc(v, "A", *shuffled_csc(model.A, rng))
        set_csc(v, "Q", *shuffled_csc(model.Q.Q, rng))
    return edit


def solve(model, edit=None):
    s = load_view(model, edit)
    r = s.solve(HPRQP_parameters(verbose=False, max_iter=300, check_iter=50))
    s.close()
    return r


@pytest.mark.parametrize("path", list(SIZES))
def test_index_base_and_unsorted_columns_give_the_same_solve(path):
    model = W.random_qp(seed=41, **SIZES[path])
    assert (model.A.nnz >= 65536) == (path == "histogram")
    ref = solve(model)
    for edit in (one_based(model), unsorted(model)):
        r = solve(model, edit)
        assert r.iter == ref.iter
        assert np.array_equal(r.x, ref.x) and np.array_equal(r.y, ref.y)


@pytest.mark.parametrize("path", list(SIZES))
def test_bad_entries_are_refused_with_the_first_index(path):
    model = W.random_qp(seed=42, **SIZES[path])
    A = model.A.tocsc()
    A.sort_indices()

    def bad_value(v):
        vals = A.data.copy()
        vals[len(vals) // 2] = np.nan
        set_csc(v, "A", A.indptr.astype(np.int32), A.indices.astype(np.int32), vals)

    def bad_row(v):
        rows = A.indices.astype(np.int32).copy()
        rows[-1] = A.shape[0]
        set_csc(v, "A", A.indptr.astype(np.int32), rows, A.data.copy())

    def crossed(name_lo, name_hi, idx):
        def edit(v):
            lo = getattr(model, name_lo).astype(np.float64).copy()
            hi = getattr(model, name_hi).astype(np.float64).copy()
            for i in idx:
                lo[i], hi[i] = 1.0, 0.0
            v._keep += [lo, hi]
            setattr(v.struct, name_lo, _ptr(lo, C.c_double))
            setattr(v.struct, name_hi, _ptr(hi, C.c_double))
        return edit

    cases = [(bad_value, "A matrix contains NaN or Inf values."),
             (bad_row, "A matrix: row index out of range"),
             (crossed("l", "u", [123, 7, model.n - 1]), "l > u at index 7"),
             (crossed("AL", "AU", [model.m - 1, 5, 9]), "AL > AU at row 5")]
    for edit, msg in cases:
        with pytest.raises(HPRQPError) as e:
            load_view(model, edit)
        assert msg in str(e.value), (msg, str(e.value))
