"""CPU oracle of the learned cost model (test infrastructure only).

Float64 NumPy restatement of the 96-128-128-1 ReLU MLP that
``n_queens_b200/csrc/mlp.cu`` trains and runs: the same input encoding, the
same BF16 rounding of the weights (round to nearest even, biases kept FP32),
the mean-squared-error loss and its exact gradient.  The GPU gradients and
predictions are checked against it; the oracle's own backward pass is pinned
by central finite differences (tests/test_mlp_oracle.py).  The reference has
no model of any kind: this checks the project's own kernels.
"""
from __future__ import annotations

import numpy as np

IN, H1, H2 = 96, 128, 128
OFF_W1 = 0
OFF_B1 = OFF_W1 + H1 * IN
OFF_W2 = OFF_B1 + H1
OFF_B2 = OFF_W2 + H2 * H1
OFF_W3 = OFF_B2 + H2
OFF_B3 = OFF_W3 + H2
NPARAMS = OFF_B3 + 1


def bf16_round(x: np.ndarray) -> np.ndarray:
    """Round float32 values to the nearest bfloat16 (ties to even), as float32."""
    b = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32)


def features(N, cols, ld, rd) -> np.ndarray:
    """96 input bits per task: bit j of cols, ld, rd at j, 32+j, 64+j (columns >= N cleared)."""
    cols = np.asarray(cols, np.uint64)
    n = cols.size
    Ns = np.broadcast_to(np.asarray(N, np.int64), (n,))
    last = np.where(Ns >= 32, 0xFFFFFFFF, (np.uint64(1) << Ns.astype(np.uint64)) - np.uint64(1)).astype(np.uint64)
    X = np.zeros((n, IN), np.float64)
    for off, m in ((0, cols), (32, np.asarray(ld, np.uint64)), (64, np.asarray(rd, np.uint64))):
        mm = m & last
        for j in range(32):
            X[:, off + j] = (mm >> np.uint64(j)) & np.uint64(1)
    return X


def unpack(params: np.ndarray):
    p = np.asarray(params, np.float32)
    W1 = bf16_round(p[OFF_W1:OFF_B1]).reshape(H1, IN).astype(np.float64)
    b1 = p[OFF_B1:OFF_W2].astype(np.float64)
    W2 = bf16_round(p[OFF_W2:OFF_B2]).reshape(H2, H1).astype(np.float64)
    b2 = p[OFF_B2:OFF_W3].astype(np.float64)
    W3 = bf16_round(p[OFF_W3:OFF_B3]).astype(np.float64)
    b3 = float(p[OFF_B3])
    return W1, b1, W2, b2, W3, b3


def forward(params, X, h1_bf16: bool = False):
    """Forward pass; h1_bf16 rounds the layer-1 outputs to BF16 (the tensor-core path's operand)."""
    W1, b1, W2, b2, W3, b3 = unpack(params)
    a1 = X @ W1.T + b1
    h1 = np.maximum(a1, 0)
    if h1_bf16:
        h1 = bf16_round(h1.astype(np.float32)).astype(np.float64)
    a2 = h1 @ W2.T + b2
    h2 = np.maximum(a2, 0)
    out = h2 @ W3 + b3
    return out, (X, a1, h1, a2, h2)


def loss_and_grad(params, X, y):
    """Mean squared error and its gradient w.r.t. the (BF16-rounded) weights, flat layout."""
    W1, b1, W2, b2, W3, b3 = unpack(params)
    out, (X, a1, h1, a2, h2) = forward(params, X)
    n = X.shape[0]
    e = out - np.asarray(y, np.float64)
    loss = float(np.mean(e * e))
    d = 2.0 * e / n
    g = np.zeros(NPARAMS, np.float64)
    g[OFF_W3:OFF_B3] = h2.T @ d
    g[OFF_B3] = d.sum()
    dh2 = (d[:, None] * W3[None, :]) * (a2 > 0)
    g[OFF_W2:OFF_B2] = (dh2.T @ h1).ravel()
    g[OFF_B2:OFF_W3] = dh2.sum(0)
    dh1 = (dh2 @ W2) * (a1 > 0)
    g[OFF_W1:OFF_B1] = (dh1.T @ X).ravel()
    g[OFF_B1:OFF_W2] = dh1.sum(0)
    return loss, g
