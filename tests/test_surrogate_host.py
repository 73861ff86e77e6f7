"""Host side of the learned surrogate (CPU): seeded requests and their bounds,
the network's input features, march inputs whose outputs fall on the 4 x 4
sub-grid of every coarse cell, and the host form of the cell reduction."""
import numpy as np
import pytest

from cupyram_b200 import batch as B
from cupyram_b200 import surrogate as S


def test_requests_are_seeded_and_within_bounds():
    q, q2 = S.requests(3000, seed=5), S.requests(3000, seed=5)
    for f in q.__dataclass_fields__:
        assert np.array_equal(getattr(q, f), getattr(q2, f)), f
    assert not np.array_equal(S.requests(3000, seed=6).freq, q.freq)
    assert np.all((q.d0 >= 100.0) & (q.d0 <= 4000.0)) and np.all(np.abs(q.slope) <= 3.0)
    assert np.all(q.d1 >= 20.0)
    assert np.all((q.cb >= 1500.0) & (q.cb <= 1900.0)) and np.all((q.rhob >= 1.2) & (q.rhob <= 2.0))
    assert np.all((q.attn >= 0.1) & (q.attn <= 1.0)) and np.all((q.freq >= 25.0) & (q.freq <= 400.0))
    lam = 1500.0 / q.freq
    assert np.all(q.zs >= 0.11 * lam - 1e-12)  # below the march's first depth cell
    assert np.all(q.zs <= np.maximum(0.9 * q.d0, 0.11 * lam) + 1e-12)
    assert np.all(q.ssp_z[:, 0] == 0.0) and np.allclose(q.ssp_z[:, -1], np.maximum(q.d0, q.d1))
    sub = q.take(np.arange(10, 20))
    assert len(sub) == 10 and np.array_equal(sub.ssp_c, q.ssp_c[10:20])


def test_features_layout():
    q = S.requests(500, seed=1)
    f = S.features(q)
    assert f.shape == (500, S.D_IN) and f.dtype == np.float32
    assert np.all(np.isfinite(f)) and np.all(f[:, S.N_FEAT:] == 0.0)
    assert np.abs(f[:, :S.N_FEAT]).max() < 10.0  # normalised to order one


def test_march_inputs_put_outputs_on_the_cell_subgrid():
    q = S.requests(300, seed=2)
    args, kw = S.march_inputs(q)
    envs, p, zs, zr, pr = B.prepare(*args, dict(kw))
    b = B.build_batch(envs, p, zs, zr, pr, True)
    r = b.rays
    lam = 1500.0 / q.freq
    assert np.allclose(r["dr"] * r["ndr"], S.DR_CELL / S.SUB, rtol=1e-12)
    assert np.allclose(r["dz"] * r["ndz"], q.d0 / S.NZ_OUT / S.SUB, rtol=1e-12)
    assert np.all(r["nvr"] >= S.NR_OUT * S.SUB) and np.all(r["nvz"] >= S.NZ_OUT * S.SUB)
    assert np.all(r["dr"] <= S.NP_PADE * lam + 1e-9) and np.all(r["dz"] <= 0.1 * lam + 1e-12)
    assert np.all(np.floor(r["zs"] / r["dz"]) >= 1)  # the partial-fraction march applies
    assert np.all(r["np"] == S.NP_PADE)
    # the work estimate is the same grid
    assert np.array_equal(S.march_work(q), r["nz"].astype(np.float64) * r["nr"])


def test_coarse_tl_host_averages_the_subgrid():
    """|cp| = 1 everywhere: every cell's TL is -10 log10 of the mean of 1 / r
    over its sub-ranges."""
    q = S.requests(3, seed=3)
    args, kw = S.march_inputs(q)
    envs, p, zs, zr, pr = B.prepare(*args, dict(kw))
    b = B.build_batch(envs, p, zs, zr, pr, True)
    cpg = np.ones(b.grid_len, np.complex128)
    tl = S.coarse_tl_host(b, cpg)
    assert tl.shape == (3, S.NZ_OUT, S.NR_OUT)
    for i, ray in enumerate(b.rays):
        r = (np.arange(S.NR_OUT * S.SUB) + 1.0) * int(ray["ndr"]) * float(ray["dr"])
        expect = -10.0 * np.log10((1.0 / r).reshape(S.NR_OUT, S.SUB).mean(axis=1))
        assert np.allclose(tl[i], expect[None, :], atol=1e-4)
