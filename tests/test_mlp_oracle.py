"""The MLP oracle itself (CPU): its backward pass against finite differences.
Also the surrogate's host check of the tensor-core GEMM's wait flag."""
import numpy as np
import pytest

from oracle import mlp_oracle as M


def _net(rng, dims):
    W = [rng.normal(0, 1 / np.sqrt(a), (b, a)) for a, b in zip(dims[:-1], dims[1:])]
    b = [rng.normal(0, 0.1, d) for d in dims[1:]]
    return W, b


def test_gradients_match_finite_differences():
    rng = np.random.default_rng(3)
    dims = [6, 9, 7, 5]
    W, b = _net(rng, dims)
    X = rng.normal(size=(11, dims[0]))
    Y = rng.normal(size=(11, dims[-1]))
    valid = rng.random((11, dims[-1])) > 0.2
    _, dW, db = M.loss_and_grads(X, Y, W, b, valid, bf16=False)
    h = 1e-6
    for l in range(len(W)):
        for (i, j) in [(0, 0), (1, 2), (dims[l + 1] - 1, dims[l] - 1)]:
            Wp = [w.copy() for w in W]
            Wm = [w.copy() for w in W]
            Wp[l][i, j] += h
            Wm[l][i, j] -= h
            fd = (M.loss_and_grads(X, Y, Wp, b, valid, False)[0] - M.loss_and_grads(X, Y, Wm, b, valid, False)[0]) / (2 * h)
            assert abs(fd - dW[l][i, j]) < 1e-6 * max(1.0, abs(fd)), (l, i, j, fd, dW[l][i, j])
        k = dims[l + 1] // 2
        bp = [v.copy() for v in b]
        bm = [v.copy() for v in b]
        bp[l][k] += h
        bm[l][k] -= h
        fd = (M.loss_and_grads(X, Y, W, bp, valid, False)[0] - M.loss_and_grads(X, Y, W, bm, valid, False)[0]) / (2 * h)
        assert abs(fd - db[l][k]) < 1e-6 * max(1.0, abs(fd))


def test_bf16_rounding():
    x = np.array([1.0, 1.00390625, 1.005859375, -3.14159, 0.0])
    r = M.to_bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0  # halfway rounds to even
    assert r[2] == 1.0078125
    assert abs(r[3] + 3.140625) < 1e-12 and r[4] == 0.0


def test_tensor_core_wait_flag_is_checked(monkeypatch):
    """A set flag (a bounded wait of the tcgen05 GEMM gave up) makes training and
    serving raise instead of returning the incomplete results."""
    import torch
    from cupyram_b200 import surrogate as S
    monkeypatch.setattr(S, "_err", torch.zeros(1, dtype=torch.int32))
    S.check_tc_flag()
    S._err.fill_(1)
    with pytest.raises(RuntimeError, match="bounded wait"):
        S.check_tc_flag()
    monkeypatch.setattr(S, "_err", None)
    S.check_tc_flag()  # no GEMM has run: nothing to check
