"""GPU test of the batched LASSO family on the staged pass (k_bstage_pass:
each instance's column block of the input in shared memory, 16-bit local
columns in 8-entry chunks, tiles of whole rows of one instance).  A family
large enough for the staged copies (8 instances of 500 x 3,000 at 2%):

 - with the staged passes forced (HPRQP_BATCH_STAGED=1) and with them off
   (=0, the CSR row passes), every instance reaches OPTIMAL with the same
   objective to 1e-9 and, in FP64, iteration counts within 2%: the two
   differ only in the order of the row sums;
 - the staged batch matches each instance's own single solve (status,
   objective to 1e-6), in both precision modes;
 - one instance of the staged FP64 batch against the oracle: its status,
   objective (1e-6), and an iteration count within 10% (the batch's lockstep
   power method starts from its own vector, so lambda differs in the last
   digits of its 1e-4 stopping test).
"""
import os

import numpy as np
import pytest

from hprqp_b200 import HPRQP_parameters, Solver
from hprqp_b200 import workloads as W
from hprqp_b200.batch import solve_batch
from oracle import oracle as O
from tests.test_gpu_parity import oracle_params

pytestmark = pytest.mark.gpu

_fam = None


def family():
    global _fam
    if _fam is None:
        _fam = W.lasso_family(8, m=500, n=3000, density=0.02, start=900)
    return _fam


def run(mode, precision):
    os.environ["HPRQP_BATCH_STAGED"] = mode
    try:
        return solve_batch(family(), HPRQP_parameters(verbose=False, problem_type="LASSO", precision=precision))
    finally:
        os.environ.pop("HPRQP_BATCH_STAGED", None)


def test_family_is_large_enough_for_the_staged_copy():
    A = family()[0].Q.A
    assert A.nnz * len(family()) >= 65536 and A.nnz / A.shape[0] >= 8 and A.nnz / A.shape[1] >= 8


@pytest.mark.parametrize("precision", ["fp64", "fp32_polish"])
def test_staged_batch_matches_csr_batch_and_single_solves(precision):
    staged = run("1", precision)
    plain = run("0", precision)
    for m, rs, rp in zip(family(), staged, plain):
        assert rs.status == rp.status == "OPTIMAL"
        assert rs.residuals < 1e-6
        assert abs(rs.primal_obj - rp.primal_obj) <= 1e-9 * (1 + abs(rp.primal_obj)), (rs.primal_obj, rp.primal_obj)
        if precision == "fp64":
            assert abs(rs.iter - rp.iter) <= max(10, 0.02 * rp.iter), (rs.iter, rp.iter)
        s = Solver().load(m)
        r1 = s.solve(HPRQP_parameters(verbose=False, problem_type="LASSO"))
        s.close()
        assert r1.status == "OPTIMAL"
        tol = 1e-6 if precision == "fp64" else 1e-5
        assert abs(rs.primal_obj - r1.primal_obj) / (1 + abs(r1.primal_obj)) < tol
        assert np.max(np.abs(rs.x - r1.x)) / max(1.0, np.max(np.abs(r1.x))) < 1e-3


def test_staged_batch_instance_matches_oracle():
    m = family()[3]
    rb = run("1", "fp64")[3]
    ref = O.solve(m, oracle_params("LASSO", max_iter=50000))
    assert ref.status_name == rb.status == "OPTIMAL"
    assert abs(rb.primal_obj - ref.primal_obj) / (1 + abs(ref.primal_obj)) < 1e-6
    assert abs(rb.iter - ref.iter) <= max(20, 0.1 * ref.iter), (rb.iter, ref.iter)
