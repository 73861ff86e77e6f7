"""Property test of the host pipeline's whole-batch checks (CPU): on random
ragged, NaN-padded batches, with NaN gaps and bad values planted at random,
whenever check_batch accepts a batch the per-environment loop accepts it too
and yields identical records (check_inputs falls back to the loop, and its
errors, in every other case)."""
import numpy as np
from hypothesis import given, settings, strategies as st

from cupyram_b200 import batch as B


@st.composite
def batches(draw):
    n = draw(st.integers(1, 5))
    seed = draw(st.integers(0, 2**31 - 1))
    rng = np.random.default_rng(seed)
    env = []
    for _ in range(n):
        nzs = int(rng.integers(2, 6))
        nrs, nzb, nrb, nbt = (int(rng.integers(1, 5)) for _ in range(4))
        depth = float(rng.uniform(50.0, 300.0))
        # a valid environment unless a fault is planted below: the profile
        # spans 0 .. depth + 50 m, so it covers the source, receiver and bottom
        env.append(dict(
            z_ss=np.concatenate([[0.0], np.sort(rng.uniform(0.0, depth + 50.0, nzs - 2)), [depth + 50.0]]),
            rp_ss=np.sort(rng.uniform(0.0, 5000.0, nrs)),
            cw=rng.uniform(1450.0, 1550.0, (nzs, nrs)),
            z_sb=np.sort(rng.uniform(0.0, 100.0, nzb)), rp_sb=np.sort(rng.uniform(0.0, 5000.0, nrb)),
            cb=rng.uniform(1600.0, 1800.0, (nzb, nrb)), rhob=rng.uniform(1.2, 2.0, (nzb, nrb)),
            attn=rng.uniform(0.1, 1.0, (nzb, nrb)),
            rbzb=np.stack([np.sort(rng.uniform(0.0, 6000.0, nbt)), rng.uniform(10.0, depth, nbt)], axis=1)))
    zs = rng.uniform(0.0, 60.0, n)
    zr = rng.uniform(0.0, 60.0, n)
    # plant faults: NaN gaps, NaN leads, infinities, non-positive speeds, deep bathymetry, shapes
    for _ in range(draw(st.integers(0, 3))):
        e = env[int(rng.integers(n))]
        key = ["z_ss", "rp_ss", "cw", "z_sb", "rp_sb", "cb", "rhob", "attn", "rbzb"][int(rng.integers(9))]
        a = e[key].astype(np.float64).copy()
        kind = int(rng.integers(5))
        flat = a.reshape(-1)
        if kind == 0:
            flat[int(rng.integers(flat.size))] = np.nan
        elif kind == 1:
            flat[int(rng.integers(flat.size))] = np.inf
        elif kind == 2:
            flat[int(rng.integers(flat.size))] = -1.0
        elif kind == 3 and key == "rbzb":
            a[:, 1] = 1e5
        elif kind == 4 and a.ndim == 2 and a.shape[0] > 1:
            a = a[:-1]
        e[key] = a
    return zs, zr, env


def _norm(env, key):
    return B.normalize_to_batch([e[key] for e in env], len(env), key)


@settings(max_examples=300, deadline=None)
@given(batches())
def test_whole_batch_checks_agree_with_the_loop(case):
    zs, zr, env = case
    keys = ["z_ss", "rp_ss", "cw", "z_sb", "rp_sb", "cb", "rhob", "attn", "rbzb"]
    try:
        norm = [_norm(env, k) for k in keys]
    except ValueError:
        return  # entries of differing dimensionality: rejected before either check
    fast = B.check_batch(len(env), zs, zr, *norm)
    if fast is None:
        return
    slow = B.check_each(len(env), zs, zr, *norm)  # must not raise
    assert len(fast) == len(slow)
    for a, b in zip(fast, slow):
        for f in a.__dataclass_fields__:
            x, y = getattr(a, f), getattr(b, f)
            assert x.shape == y.shape and np.array_equal(x, y), f
