"""run()'s result layout on the host: reshape to [E, F, ...] and the reference's
squeeze rules (cupyram.py:335-380), applied to synthetic engine outputs in
which every entry encodes its ray and position."""
import numpy as np
import pytest

from golden_cases import load_case
from cupyram_b200 import CuPyRAM


def _fake_outputs(b):
    """Line entry = ray * 1e6 + range index; grid entry = ray * 1e6 + depth * 1e3 + range."""
    tll = np.zeros(b.line_len)
    tlg = np.zeros(max(b.grid_len, 1))
    for k, r in enumerate(b.rays):
        lo, nvr, nvz = int(r["line_off"]), int(r["nvr"]), int(r["nvz"])
        tll[lo:lo + nvr] = k * 1e6 + np.arange(nvr)
        if b.compute_grids:
            go = int(r["grid_off"])
            tlg[go:go + nvz * nvr] = (k * 1e6 + np.arange(nvz)[:, None] * 1e3 + np.arange(nvr)[None, :]).ravel()
    return {"tll": tll, "cpl": tll.astype(np.complex128), "tlg": tlg, "cpg": tlg.astype(np.complex128)}


def _results(args, kw):
    c = CuPyRAM(*args, **kw)
    b = c.setup()
    return c._results(b, _fake_outputs(b)), b


@pytest.mark.parametrize("n_env,freqs,shape", [
    (1, [50.0], ()), (3, [50.0], (3,)), (1, [40.0, 50.0], (2,)), (3, [40.0, 50.0], (3, 2)),
])
def test_squeeze_and_ray_order(n_env, freqs, shape):
    args, kw, _ = load_case("pekeris_small")
    args = [freqs if len(freqs) > 1 else freqs[0]] + list(args[1:])
    res, b = _results(args, dict(kw, batch_size=n_env))
    nvr, nvz = int(b.rays["nvr"][0]), int(b.rays["nvz"][0])
    tl = np.asarray(res["TL Line"])
    assert tl.shape == shape + (nvr,)
    assert np.asarray(res["TL Grid"]).shape == shape + (nvz, nvr)
    assert np.asarray(res["CP Line"]).shape == tl.shape and np.asarray(res["CP Grid"]).shape == shape + (nvz, nvr)
    # calculation order: environment-major, then frequency (ray = e * n_freq + f)
    full = tl.reshape(n_env, len(freqs), nvr)
    for e in range(n_env):
        for f in range(len(freqs)):
            assert full[e, f, 3] == (e * len(freqs) + f) * 1e6 + 3
    grid = np.asarray(res["TL Grid"]).reshape(n_env, len(freqs), nvz, nvr)
    assert grid[n_env - 1, len(freqs) - 1, 2, 5] == (n_env * len(freqs) - 1) * 1e6 + 2e3 + 5
    assert np.array_equal(res["Ranges"], (np.arange(nvr) + 1) * float(b.rays["dr"][0]) * int(b.rays["ndr"][0]))


def test_without_grids_the_grid_entries_are_none():
    args, kw, _ = load_case("pekeris_small")
    res, _ = _results(args, dict(kw, compute_grids=False))
    assert res["TL Grid"] is None and res["CP Grid"] is None
    assert np.asarray(res["TL Line"]).ndim == 1


def test_per_ray_grids_of_different_sizes_come_back_as_lists():
    args, kw, _ = load_case("pekeris_small")
    n = 3
    per = [[30.0, 50.0, 70.0], np.array([100.0, 90.0, 80.0]), np.array([50.0, 60.0, 70.0])] + list(args[3:])
    res, b = _results(per, dict(kw, batch_size=n, per_ray=True, rmax=np.array([1000.0, 1500.0, 2000.0])))
    assert isinstance(res["TL Line"], list) and len(res["TL Line"]) == n
    for k in range(n):
        nvr, nvz = int(b.rays["nvr"][k]), int(b.rays["nvz"][k])
        assert res["TL Line"][k].shape == (nvr,) and res["TL Line"][k][0] == k * 1e6
        assert res["TL Grid"][k].shape == (nvz, nvr)
        assert res["Ranges"][k].shape == (nvr,)
    assert len({x.size for x in res["TL Line"]}) == n
