"""CPU oracle of the surrogate MLP's forward and backward passes (test infrastructure).

The surrogate has no counterpart in clapeyre/cupyram; this file restates the
mathematics its GPU kernels implement (cupyram_b200/csrc/mlp.cu,
cupyram_b200/surrogate.py: MLP) so that tests can check the kernels' gradients
against it:

    H_{l+1} = relu(H_l W_l^T + b_l)        (hidden layers)
    out     = H_{L-1} W_{L-1}^T + b_{L-1}
    loss    = mean over valid entries of (out - y)^2
    g_out   = 2 (out - y) / count          (valid entries, else 0)
    dW_l    = g_{l+1}^T H_l,  db_l = column sums of g_{l+1}
    g_l     = (g_{l+1} W_l) * [H_l > 0]

Arithmetic is float64.  With bf16=True the values are rounded to bfloat16
where the kernels store them (inputs, weights, hidden activations, output
gradients, propagated gradients), so a comparison isolates the kernels'
accumulation error.  Pinned by tests/test_mlp_oracle.py against central
finite differences of the loss (bf16=False).
"""
import numpy as np


def to_bf16(x):
    """Round to bfloat16 (nearest, ties to even) and return as float64."""
    u = np.asarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def forward(X, W, b, bf16=True):
    """Activations [H_0 .. H_{L-1}] and the output of the network."""
    r = to_bf16 if bf16 else (lambda a: np.asarray(a, np.float64))
    H = [r(X)]
    L = len(W)
    for l in range(L - 1):
        H.append(r(np.maximum(H[l] @ r(W[l]).T + b[l], 0.0)))
    out = H[-1] @ r(W[-1]).T + b[-1]
    return H, out


def loss_and_grads(X, Y, W, b, valid=None, bf16=True):
    """Mean squared error and its gradients (dW, db) for every layer."""
    r = to_bf16 if bf16 else (lambda a: np.asarray(a, np.float64))
    H, out = forward(X, W, b, bf16)
    y = r(Y)
    m = np.ones_like(out, dtype=bool) if valid is None else valid.astype(bool)
    cnt = max(int(m.sum()), 1)
    d = np.where(m, out - y, 0.0)
    loss = float(np.sum(d * d) / cnt)
    g = r(2.0 * d / cnt)
    dW, db = [None] * len(W), [None] * len(W)
    for l in range(len(W) - 1, -1, -1):
        dW[l] = g.T @ H[l]
        db[l] = g.sum(axis=0)
        if l > 0:
            g = r((g @ r(W[l])) * (H[l] > 0))
    return loss, dW, db
