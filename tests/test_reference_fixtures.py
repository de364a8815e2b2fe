"""CPU tests: the oracle on the reference's own test problems (AUG2D,
AUG3DCQP under test/runtests.jl:254-280 and :704-788; esc64a as a QAP at
:467-506), stored in tests/golden/reference_fixtures.npz.  They pin the
oracle to the reference suite's assertions (status OPTIMAL, residuals
< 1e-6) and to its own recorded solves (same iteration count, sigma
sequence and restart iterations; objective to 1e-12), and check the stored
problems against a fresh read of the data files when the reference tree is
available (HPRQP_REFERENCE_DATA)."""
import os

import numpy as np
import pytest

from hprqp_b200._abi import default_params
from oracle import oracle as O
from tests import reference_fixtures as RF
from tests.kkt import kkt


def params(name):
    p = default_params()
    p.verbose = 0
    p.problem_type = {"QP": 0, "QAP": 2}[RF.PTYPE[name]]
    p.max_iter = RF.MAX_ITER[name]
    return p


@pytest.mark.parametrize("name", RF.NAMES)
def test_oracle_solves_reference_problem(name):
    m = RF.model(name)
    ref = RF.ref(name)
    r = O.solve(m, params(name), trace_iters=ref["iter"])
    # the reference test's own assertions
    assert r.status_name == "OPTIMAL" and r.residuals < 1e-6
    # the recorded solve, step for step
    assert r.iter == ref["iter"] and r.restarts == ref["restarts"]
    assert abs(r.primal_obj - ref["primal_obj"]) <= 1e-12 * (1 + abs(ref["primal_obj"]))
    assert np.array_equal(r.sigma_trace, ref["sigma"])
    assert np.array_equal(r.inner_trace, ref["inner"])
    # a restart decided at the final check has no traced step after it
    assert ref["restarts"] - 1 <= len(RF.restart_iterations(ref["inner"])) <= ref["restarts"]
    if RF.PTYPE[name] == "QP":
        k = kkt(m, r.x, r.y, r.z)
        assert k["err_Rp"] < 1e-5 and k["err_Rd"] < 1e-5


@pytest.mark.skipif(not os.environ.get("HPRQP_REFERENCE_DATA"), reason="reference data files not given")
@pytest.mark.parametrize("name", RF.NAMES)
def test_stored_problem_matches_data_file(name):
    data = os.environ["HPRQP_REFERENCE_DATA"]
    if name == "esc64a":
        import scipy.io as sio
        d = sio.loadmat(os.path.join(data, "esc64a.mat"))
        for k, v in zip("ABST", RF.raw(name)):
            assert np.array_equal(np.asarray(d[k], dtype=np.float64), v)
        return
    from tests.mps import read_mps
    fresh = read_mps(os.path.join(data, name + ".mps"))
    for a, b in zip(fresh, RF.raw(name)):
        if hasattr(a, "toarray"):
            assert (a != b).nnz == 0
        else:
            assert np.array_equal(np.asarray(a, dtype=np.float64), b)
