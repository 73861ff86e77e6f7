"""Host pipeline (normalisation, validation, parameters) - reference semantics."""
import numpy as np
import pytest

from cupyram_b200 import batch as B
from golden_cases import load_case


def pekeris(**over):
    d = dict(freq=50.0, zs=100.0, zr=50.0, z_ss=np.array([0.0, 200.0]), rp_ss=np.array([0.0]),
             cw=np.array([[1500.0], [1500.0]]), z_sb=np.array([0.0]), rp_sb=np.array([0.0]),
             cb=np.array([[1700.0]]), rhob=np.array([[1.5]]), attn=np.array([[0.5]]),
             rbzb=np.array([[0.0, 200.0], [10000.0, 200.0]]))
    d.update(over)
    return d


ORDER = ["freq", "zs", "zr", "z_ss", "rp_ss", "cw", "z_sb", "rp_sb", "cb", "rhob", "attn", "rbzb"]


def prep(d, **kw):
    return B.prepare(*[d[k] for k in ORDER], kw)


def test_normalize_list_padding():
    x = B.normalize_to_batch([np.array([0.0, 1.0]), np.array([0.0, 1.0, 2.0])], 2, "x")
    assert x.shape == (2, 3) and np.isnan(x[0, 2])
    y = B.normalize_to_batch(np.array([1.0, 2.0]), 3, "y")
    assert y.shape == (3, 2)
    z = B.normalize_to_batch(5.0, 4, "z")
    assert z.shape == (4,)
    with pytest.raises(ValueError):
        B.normalize_to_batch([np.zeros(2)], 2, "w")


def test_valid_slice():
    a = np.array([1.0, 2.0, np.nan])
    v, n = B.valid_slice(a)
    assert n == 2 and v.tolist() == [1.0, 2.0]
    m = np.array([[1.0, 2.0, np.nan], [3.0, 4.0, np.nan], [np.nan, np.nan, np.nan]])
    v, n = B.valid_slice(m)
    assert v.shape == (2, 2) and n == 2


def test_defaults_follow_max_frequency():
    envs, p, *_ = prep(pekeris(freq=[50.0, 100.0, 200.0]), rmax=1000.0)
    assert p.dr[0] == pytest.approx(60.0)
    assert p.dz[0] == pytest.approx(0.75)


@pytest.mark.parametrize("bad", [
    dict(zs=300.0), dict(zr=-1.0), dict(cw=np.array([[1500.0, 1500.0], [1500.0, 1500.0]])),
    dict(cb=np.array([[1700.0], [1700.0]])), dict(rbzb=np.array([[0.0, 250.0], [1e4, 250.0]])),
])
def test_invalid_inputs_raise(bad):
    with pytest.raises(ValueError):
        prep(pekeris(**bad))


def test_source_below_grid_raises():
    envs, p, zs, zr, pr = prep(pekeris(), dz=2.0)
    b = B.build_batch(envs, p, zs, zr, pr, False)
    assert b.rays["nz"][0] > 100


def test_ragged_rbzb_extension_and_offsets():
    args, kw, fx = load_case("ragged_batch")
    envs, p, zs, zr, pr = B.prepare(*args, dict(kw))
    b = B.build_batch(envs, p, zs, zr, pr, True)
    # every ray's bathymetry ends at >= rmax; lines are packed back to back
    for k, e in enumerate(b.envs):
        zb_end = b.pool[e["off"] + e["n_zss"] + e["n_rss"] + e["n_rss"] * e["n_zss"] + e["n_zsb"]
                        + e["n_rsb"] + 3 * e["n_rsb"] * e["n_zsb"] + e["n_bt"] - 1]
        assert zb_end >= 3000.0
    assert np.array_equal(b.rays["line_off"], np.arange(b.n_rays) * b.rays["nvr"][0])


def test_per_ray_grids():
    d = pekeris(freq=[50.0, 100.0], zs=[100.0, 80.0], zr=[50.0, 60.0],
                z_ss=[np.array([0.0, 200.0])] * 2, rp_ss=[np.array([0.0])] * 2,
                cw=[np.array([[1500.0], [1500.0]])] * 2, z_sb=[np.array([0.0])] * 2,
                rp_sb=[np.array([0.0])] * 2, cb=[np.array([[1700.0]])] * 2,
                rhob=[np.array([[1.5]])] * 2, attn=[np.array([[0.5]])] * 2,
                rbzb=[np.array([[0.0, 200.0], [5000.0, 200.0]])] * 2)
    envs, p, zs, zr, pr = B.prepare(*[d[k] for k in ORDER], dict(batch_size=2, per_ray=True))
    b = B.build_batch(envs, p, zs, zr, pr, False)
    assert b.rays["nz"][1] > b.rays["nz"][0]          # finer dz at higher frequency
    assert b.rays["lyrw_lambda"][0] == pytest.approx(20 * 1500.0 / 50.0)
    assert b.rays["lyrw_lambda"][1] == pytest.approx(20 * 1500.0 / 100.0)


def _uniform_batch(n, seed, bad=None):
    """n equal-shaped per-ray environments; about half of the bathymetry lines end
    short of rmax (so build_batch extends them) and the rest reach beyond it."""
    rng = np.random.default_rng(seed)
    depth = rng.uniform(150.0, 400.0, n)
    z_ss = np.linspace(0.0, 1.0, 6)[None, :] * (depth + 50.0)[:, None]
    cw = 1500.0 + rng.uniform(-5.0, 5.0, (n, 6, 2))
    r_end = np.where(rng.random(n) < 0.5, 3000.0, 5000.0)
    rbzb = np.zeros((n, 3, 2))
    rbzb[:, 1, 0], rbzb[:, 2, 0] = 1000.0, r_end
    rbzb[:, :, 1] = depth[:, None] * np.array([1.0, 0.9, 0.8])[None, :]
    zs = rng.uniform(10.0, 100.0, n)
    if bad is not None:
        zs[bad] = z_ss[bad, -1] + 1.0
    args = [rng.uniform(40.0, 80.0, n), zs, zs * 0.5, list(z_ss), [np.array([0.0, 2000.0])] * n, list(cw),
            [np.array([0.0, 100.0])] * n, [np.array([0.0])] * n,
            [np.array([[1700.0], [1800.0]])] * n, [np.array([[1.5], [1.6]])] * n, [np.array([[0.5], [0.5]])] * n,
            list(rbzb)]
    return args, dict(batch_size=n, per_ray=True, rmax=4000.0)


def test_whole_batch_checks_match_per_environment_loop():
    args, kw = _uniform_batch(40, 5)
    norm = [B.normalize_to_batch(x, 40, "x") for x in args[3:]]
    zs, zr = np.asarray(args[1]), np.asarray(args[2])
    fast = B.check_batch(40, zs, zr, *norm)
    slow = B.check_each(40, zs, zr, *norm)
    assert fast is not None and len(fast) == len(slow)
    for a, b in zip(fast, slow):
        for f in a.__dataclass_fields__:
            x, y = getattr(a, f), getattr(b, f)
            assert x.shape == y.shape and np.array_equal(x, y), f


def test_whole_batch_pool_matches_per_environment_packing():
    args, kw = _uniform_batch(40, 6)
    envs, p, zs, zr, pr = B.prepare(*args, dict(kw))
    b = B.build_batch(envs, p, zs, zr, pr, True)
    assert 0 < int(np.sum(b.envs["n_bt"] == 4)) < 40  # both extended and unextended lines
    zsb_abs = [e.z_sb + e.z_ss[-1] for e in envs]
    bt_ext = [np.vstack([e.rbzb, [4000.0, e.rbzb[-1, 1]]]) if e.rbzb[-1, 0] < 4000.0 else e.rbzb for e in envs]
    env_ref, pool_ref = B._pack_each(envs, zsb_abs, bt_ext, np.zeros(len(envs), dtype=b.envs.dtype))
    assert b.envs.tobytes() == env_ref.tobytes()
    assert b.pool.tobytes() == pool_ref.tobytes()


def test_ray_table_matches_per_ray_restatement():
    args, kw = _uniform_batch(24, 7)
    envs, p, zs, zr, pr = B.prepare(*args, dict(kw))
    b = B.build_batch(envs, p, zs, zr, pr, True)
    line = grid = 0
    for k, r in enumerate(b.rays):
        assert (r["freq"], r["c0"], r["zs"], r["zr"]) == (p.freqs[k], p.c0_env[k], zs[k], zr[k])
        assert (r["dz"], r["dr"], r["rs"], r["env"]) == (p.dz[k], p.dr[k], p.rs[k], k)
        assert (r["line_off"], r["grid_off"]) == (line, grid)
        line += int(r["nvr"])
        grid += int(r["nvr"]) * int(r["nvz"])
        assert np.array_equal(b.vr[k], np.arange(1, r["nvr"] + 1) * p.dr[k] * r["ndr"])
        assert np.array_equal(b.vz[k], np.arange(1, r["nvz"] + 1) * p.dz[k] * r["ndz"])
    assert (b.line_len, b.grid_len) == (line, grid)


def test_whole_batch_errors_name_the_first_bad_ray():
    args, kw = _uniform_batch(30, 8, bad=17)
    with pytest.raises(ValueError, match="Ray 17: Source depth"):
        B.prepare(*args, dict(kw))
    args, kw = _uniform_batch(30, 8)
    args[5][4] = args[5][4].copy()
    args[5][4][2, 1] = -1.0
    with pytest.raises(ValueError, match="Ray 4: sound speeds"):
        B.prepare(*args, dict(kw))


def _ragged_batch(n, seed):
    """n per-ray environments whose profiles, tables and bathymetry lines all differ in length."""
    rng = np.random.default_rng(seed)
    nzs, nrs, nzb, nrb, nbt = (rng.integers(lo, hi, n) for lo, hi in ((3, 9), (1, 4), (1, 4), (1, 3), (1, 5)))
    depth = rng.uniform(150.0, 400.0, n)
    bt = []
    for i in range(n):
        r = np.sort(rng.uniform(0.0, 6000.0, nbt[i]))
        r[0] = 0.0
        bt.append(np.stack([r, depth[i] * rng.uniform(0.7, 1.0, nbt[i])], axis=1))
    zs = rng.uniform(10.0, 100.0, n)
    args = [rng.uniform(40.0, 80.0, n), zs, zs * 0.5,
            [np.linspace(0.0, depth[i] + 50.0, nzs[i]) for i in range(n)],
            [np.linspace(0.0, 3000.0, nrs[i]) for i in range(n)],
            [1500.0 + rng.uniform(-5.0, 5.0, (nzs[i], nrs[i])) for i in range(n)],
            [np.linspace(0.0, 100.0, nzb[i]) for i in range(n)],
            [np.linspace(0.0, 2000.0, nrb[i]) for i in range(n)],
            [rng.uniform(1600.0, 1800.0, (nzb[i], nrb[i])) for i in range(n)],
            [rng.uniform(1.3, 2.0, (nzb[i], nrb[i])) for i in range(n)],
            [rng.uniform(0.1, 1.0, (nzb[i], nrb[i])) for i in range(n)], bt]
    return args, dict(batch_size=n, per_ray=True, rmax=4000.0)


def test_padded_batch_checks_match_per_environment_loop():
    args, kw = _ragged_batch(60, 9)
    norm = [B.normalize_to_batch(x, 60, "x") for x in args[3:]]
    assert all(np.isnan(a).any() for a in norm)  # every input is NaN-padded
    zs, zr = np.asarray(args[1]), np.asarray(args[2])
    fast = B.check_batch(60, zs, zr, *norm)
    slow = B.check_each(60, zs, zr, *norm)
    assert fast is not None
    for a, b in zip(fast, slow):
        for f in a.__dataclass_fields__:
            x, y = getattr(a, f), getattr(b, f)
            assert x.shape == y.shape and np.array_equal(x, y), f
    envs, p, zs, zr, pr = B.prepare(*args, dict(kw))
    b = B.build_batch(envs, p, zs, zr, pr, True)
    assert b.envs["n_zss"].tolist() == [len(z) for z in args[3]]


def test_padded_batch_errors_name_the_first_bad_ray():
    # a NaN inside a profile's valid part leaves a gap that the loop reports
    args, kw = _ragged_batch(20, 10)
    args[5][11] = args[5][11].copy()
    args[5][11][0, 0] = np.nan
    norm = [B.normalize_to_batch(x, 20, "x") for x in args[3:]]
    assert B.check_batch(20, np.asarray(args[1]), np.asarray(args[2]), *norm) is None
    with pytest.raises(ValueError, match="Ray 11: cw contains non-finite"):
        B.prepare(*args, dict(kw))


@pytest.mark.parametrize("kw,match", [
    (dict(np=0), "np must be"), (dict(np=11), "np must be"), (dict(dr=-1.0), "dr and dz"), (dict(dz=0.0), "dr and dz"),
    (dict(ns=3), "ns must be"), (dict(ndr=0), "ndr and ndz"), (dict(ndz=0), "ndr and ndz"),
    (dict(batch_size=0), "batch_size"), (dict(rmax=1.0, dr=50.0), "rmax must cover"),
])
def test_invalid_parameters_raise(kw, match):
    with pytest.raises(ValueError, match=match):
        envs, p, zs, zr, pr = prep(pekeris(), **kw)
        B.build_batch(envs, p, zs, zr, pr, False)


@pytest.mark.parametrize("freq", [0.0, -50.0, float("nan"), []])
def test_invalid_frequency_raises(freq):
    with pytest.raises(ValueError, match="freq"):
        prep(pekeris(freq=freq))


def test_per_ray_values_must_match_the_batch():
    d = pekeris(z_ss=[np.array([0.0, 200.0])] * 2, rp_ss=[np.array([0.0])] * 2,
                cw=[np.array([[1500.0], [1500.0]])] * 2, z_sb=[np.array([0.0])] * 2, rp_sb=[np.array([0.0])] * 2,
                cb=[np.array([[1700.0]])] * 2, rhob=[np.array([[1.5]])] * 2, attn=[np.array([[0.5]])] * 2,
                rbzb=[np.array([[0.0, 200.0], [5000.0, 200.0]])] * 2)
    with pytest.raises(ValueError, match="zs"):
        B.prepare(*[dict(d, zs=[100.0, 90.0, 80.0])[k] for k in ORDER], dict(batch_size=2, per_ray=True))
    with pytest.raises(ValueError, match="scalars unless per_ray"):
        B.prepare(*[dict(d, zs=[100.0, 90.0])[k] for k in ORDER], dict(batch_size=2))
    with pytest.raises(ValueError, match="list length"):
        B.prepare(*[d[k] for k in ORDER], dict(batch_size=3))
    # per-ray np, dr and output decimation are taken ray by ray
    envs, p, zs, zr, pr = B.prepare(*[dict(d, freq=[50.0, 100.0])[k] for k in ORDER],
                                    dict(batch_size=2, per_ray=True, np=np.array([4, 8]), ndr=np.array([1, 2]),
                                         ndz=np.array([2, 3])))
    b = B.build_batch(envs, p, zs, zr, pr, True)
    assert b.rays["np"].tolist() == [4, 8] and b.rays["ndr"].tolist() == [1, 2] and b.rays["ndz"].tolist() == [2, 3]
    assert b.rays["dr"].tolist() == [4 * 1500.0 / 50.0, 8 * 1500.0 / 100.0]  # dr = np c / f per ray


def test_c0_override_and_default():
    envs, p, *_ = prep(pekeris(cw=np.array([[1490.0], [1510.0]])), rmax=1000.0)
    assert p.c0_env[0] == pytest.approx(1500.0)  # mean of the first water profile
    envs, p, *_ = prep(pekeris(), rmax=1000.0, c0=1480.0)
    assert p.c0_env[0] == 1480.0 and p.c0_report == 1480.0
