"""GPU tests of the learned warm start: the MLP's hand-written backward
kernels against an FP64 numpy backpropagation on the same BF16-rounded
values (the CPU oracle of the network), training reduces the loss, and a
trained network started on held-out instances of a LASSO family reaches the
same certified optimum in fewer HPR iterations than a cold start."""
import numpy as np
import pytest

from hprqp_b200 import learned
from hprqp_b200 import workloads as W

pytestmark = pytest.mark.gpu


def bf16(a):
    """Round float32 to bfloat16 (nearest even) and back."""
    u = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def numpy_grads(W1, b1, W2, b2, W3, b3, X, T):
    """FP64 forward/backward mirroring the kernels' BF16 rounding points."""
    f = lambda a: bf16(a).astype(np.float64)
    Xb = f(X)
    Z1 = Xb @ f(W1).T + b1
    H1 = f(np.maximum(Z1, 0))
    Z2 = H1 @ f(W2).T + b2
    H2 = f(np.maximum(Z2, 0))
    Y = H2 @ f(W3).T + b3
    R = X.shape[0]
    E = Y - T
    loss = 0.5 * np.sum(E * E) / R
    dY = f(E / R)
    gW3, gb3 = dY.T @ H2, dY.sum(0)
    dZ2 = f((dY @ f(W3)) * (Z2 > 0))
    gW2, gb2 = dZ2.T @ H1, dZ2.sum(0)
    dZ1 = f((dZ2 @ f(W2)) * (Z1 > 0))
    gW1, gb1 = dZ1.T @ Xb, dZ1.sum(0)
    return loss, [gW1, gb1, gW2, gb2, gW3, gb3]


def test_mlp_gradients_match_numpy_oracle():
    rng = np.random.default_rng(0)
    n_in, width, n_out, R = 37, 48, 21, 13
    net = learned.MLP(n_in, n_out, width=width, batch=64, seed=3)
    p = net.get_params()
    p[:] = bf16(p)  # make the master weights exactly representable
    net.set_params(p)
    X = rng.standard_normal((R, n_in)).astype(np.float32)
    T = rng.standard_normal((R, n_out)).astype(np.float32)
    loss, g = net.gradients(X, T)
    ref_loss, ref = numpy_grads(*[a.astype(np.float64) for a in net.unpack(p)], X.astype(np.float64),
                                T.astype(np.float64))
    assert abs(loss - ref_loss) <= 1e-3 * ref_loss
    for got, want in zip(net.unpack(g), ref):
        err = np.linalg.norm(got - want) / max(np.linalg.norm(want), 1e-12)
        assert err < 2e-2, err
    net.close()


def test_mlp_gradients_match_numpy_oracle_multi_tile():
    """Shapes that take several 64-wide K chunks and several 128 x 128
    output tiles (with partial ones) in every product of the network."""
    rng = np.random.default_rng(4)
    n_in, width, n_out, R = 300, 256, 130, 100
    net = learned.MLP(n_in, n_out, width=width, batch=128, seed=5)
    p = net.get_params()
    p[:] = bf16(p)
    net.set_params(p)
    X = bf16(rng.standard_normal((R, n_in))).astype(np.float32)
    T = rng.standard_normal((R, n_out)).astype(np.float32)
    loss, g = net.gradients(X, T)
    ref_loss, ref = numpy_grads(*[a.astype(np.float64) for a in net.unpack(p)], X.astype(np.float64),
                                T.astype(np.float64))
    assert abs(loss - ref_loss) <= 2e-3 * ref_loss
    for got, want in zip(net.unpack(g), ref):
        err = np.linalg.norm(got - want) / max(np.linalg.norm(want), 1e-12)
        assert err < 3e-2, err
    net.close()


def test_mlp_training_reduces_loss():
    rng = np.random.default_rng(1)
    X = rng.standard_normal((512, 64)).astype(np.float32)
    Wt = rng.standard_normal((64, 16)).astype(np.float32) / 8
    T = np.tanh(X @ Wt).astype(np.float32)
    net = learned.MLP(64, 16, width=128, batch=128, seed=2)
    first = net.train_batch(X[:128], T[:128], 1e-3)
    for ep in range(60):
        for i in range(0, 512, 128):
            last = net.train_batch(X[i:i + 128], T[i:i + 128], 1e-3)
    assert last < 0.2 * first
    Y = net.predict(X[:7])
    assert Y.shape == (7, 16) and np.all(np.isfinite(Y))
    net.close()


def test_learned_warm_start_pipeline():
    # a small LASSO family (fixed pattern, perturbed values, varying b and
    # lambda); labels come from batched solves to 1e-8.  The network's
    # proposals carry little information about these solutions, so the
    # iteration count moves by a few per cent either way from run to run
    # (the labels' last bits depend on the autotuned row schedules); what
    # must hold is that training fits, every warm solve is certified at the
    # cold optimum, and the warm start costs no more than 5% extra.
    train = W.lasso_family(1000, m=120, n=400, density=0.05, start=0)
    test = W.lasso_family(24, m=120, n=400, density=0.05, start=100000)
    pairs = learned.generate_pairs(train, tol=1e-8)
    assert len(pairs) >= 950
    ws = learned.WarmStart.fit(pairs, epochs=300, lr=1e-3, width=256, batch=256)
    assert ws.history[-1] < 0.5 * ws.history[0]
    rows = learned.evaluate(test, ws, tol=1e-6)  # x0 from the network, sigma by the solver
    cold = np.array([r["cold_iter"] for r in rows])
    warm = np.array([r["warm_iter"] for r in rows])
    assert all(r["cold_status"] == r["warm_status"] == "OPTIMAL" for r in rows)
    for r in rows:  # the certified optimum is the same
        assert abs(r["warm_obj"] - r["cold_obj"]) <= 1e-5 * (1 + abs(r["cold_obj"]))
    assert warm.mean() <= 1.05 * cold.mean(), (warm.mean(), cold.mean())
