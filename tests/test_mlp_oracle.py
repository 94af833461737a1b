"""CPU checks of the cost-model oracle (oracle/mlp_ref.py): its backward pass
against central finite differences, its BF16 rounding and input encoding."""
import numpy as np

import oracle
from oracle import mlp_ref


def rand_params(seed):
    rng = np.random.default_rng(seed)
    p = rng.uniform(-0.2, 0.2, mlp_ref.NPARAMS).astype(np.float32)
    p[mlp_ref.OFF_B1:mlp_ref.OFF_W2] += 0.1  # keep most units active
    p[mlp_ref.OFF_B2:mlp_ref.OFF_W3] += 0.1
    return p


def test_bf16_rounding():
    x = np.array([1.0, 1.00390625, 1.005859375, -3.14159, 1e-30, 65504.0], np.float32)
    r = mlp_ref.bf16_round(x)
    assert r[0] == 1.0
    assert r[1] == 1.0            # tie (1 + 2^-8) rounds to even
    assert r[2] == 1.0078125      # above the tie rounds up
    assert abs(r[3] + 3.140625) < 1e-7
    assert (r.view(np.uint32) & 0xFFFF).max() == 0


def test_features_encoding():
    c, l, r = oracle.expand(8, 3)
    X = mlp_ref.features(8, c[:5], l[:5], r[:5])
    for t in range(5):
        for j in range(32):
            assert X[t, j] == ((int(c[t]) >> j) & 1 if j < 8 else 0)
            assert X[t, 32 + j] == ((int(l[t]) >> j) & 1 if j < 8 else 0)
            assert X[t, 64 + j] == ((int(r[t]) >> j) & 1 if j < 8 else 0)


def test_backward_matches_finite_differences():
    c, l, r = oracle.expand(12, 4)
    X = mlp_ref.features(12, c[:40], l[:40], r[:40])
    y = np.random.default_rng(1).uniform(5, 15, 40)
    p = rand_params(3)
    # Differentiate w.r.t. the already-rounded weights: round once, then step
    # in float64 around that point (the oracle rounds its input again, so
    # evaluate the loss with a float64 path that skips the rounding).
    W = p.copy()
    for a, b in ((mlp_ref.OFF_W1, mlp_ref.OFF_B1), (mlp_ref.OFF_W2, mlp_ref.OFF_B2), (mlp_ref.OFF_W3, mlp_ref.OFF_B3)):
        W[a:b] = mlp_ref.bf16_round(W[a:b])
    loss, g = mlp_ref.loss_and_grad(W, X, y)

    def loss64(q):
        W1 = q[mlp_ref.OFF_W1:mlp_ref.OFF_B1].reshape(128, 96)
        b1 = q[mlp_ref.OFF_B1:mlp_ref.OFF_W2]
        W2 = q[mlp_ref.OFF_W2:mlp_ref.OFF_B2].reshape(128, 128)
        b2 = q[mlp_ref.OFF_B2:mlp_ref.OFF_W3]
        W3 = q[mlp_ref.OFF_W3:mlp_ref.OFF_B3]
        h1 = np.maximum(X @ W1.T + b1, 0)
        h2 = np.maximum(h1 @ W2.T + b2, 0)
        out = h2 @ W3 + q[mlp_ref.OFF_B3]
        return np.mean((out - y) ** 2)

    q0 = W.astype(np.float64)
    assert abs(loss64(q0) - loss) < 1e-9 * max(1.0, loss)
    rng = np.random.default_rng(7)
    idx = np.concatenate([rng.choice(np.arange(mlp_ref.OFF_W1, mlp_ref.OFF_B1), 40),
                          rng.choice(np.arange(mlp_ref.OFF_W2, mlp_ref.OFF_B2), 40),
                          np.arange(mlp_ref.OFF_W3, mlp_ref.OFF_W3 + 8), [mlp_ref.OFF_B3],
                          np.arange(mlp_ref.OFF_B1, mlp_ref.OFF_B1 + 8)])
    h = 1e-6
    for i in idx:
        qp = q0.copy(); qp[i] += h
        qm = q0.copy(); qm[i] -= h
        fd = (loss64(qp) - loss64(qm)) / (2 * h)
        assert abs(fd - g[i]) <= 1e-5 * max(1.0, abs(g[i])), (i, fd, g[i])
