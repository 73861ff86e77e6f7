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
