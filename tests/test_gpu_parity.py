"""Parity of the sm_100a engine (through the C ABI) with the oracle and the reference.

Tolerances (dB of transmission loss):
* engine vs the oracle's plain complex128 form on the same inputs: 1e-3 dB on
  the TL line (the engine eliminates every other Pade term upwards, so the two
  differ only by rounding);
* engine vs the reference's own outputs (tests/golden): 0.01 dB max on the TL
  line - the reference's own parity bar against PyRAM (tests/test_utils.py:30-37);
* RAM v1.5 Fortran line: mean 0.01 dB (tests/test_reference.py:28,192).
"""
import numpy as np
import pytest

from golden_cases import CASES, GOLDEN, load_case
from cupyram_b200 import CuPyRAM
from cupyram_b200 import batch as B
from cupyram_b200.engine import Engine
from oracle import oracle

pytestmark = pytest.mark.gpu

TOL_ORACLE = 1e-3
TOL_REF = 0.01


def _batch(name, grids=True):
    args, kw, fx = load_case(name)
    envs, p, zs, zr, pr = B.prepare(*args, dict(kw))
    return B.build_batch(envs, p, zs, zr, pr, grids), fx


@pytest.mark.parametrize("march", ["batched", "column"])
@pytest.mark.parametrize("name", CASES)
def test_engine_vs_oracle(cuda_device, monkeypatch, name, march):
    """Both march kernels: batched tiles (CUPYRAM_B200_COL=0) and one cluster per ray (=1)."""
    monkeypatch.setenv("CUPYRAM_B200_COL", "0" if march == "batched" else "1")
    b, _ = _batch(name)
    with Engine(b) as eng:
        out = eng.run()
        st = eng.stats()
        assert st["rays_failed"] == 0
        if march == "column":
            assert st["column_rays"] == b.n_rays and st["column_launches"] >= 1
        else:
            assert st["column_rays"] == 0
    ref = oracle.run(b, "plain")
    n = b.line_len
    d = np.abs(out["tll"][:n] - ref["tll"][:n])
    assert d.max() < TOL_ORACLE, d.max()
    cp = np.abs(out["cpl"][:n] - ref["cpl"][:n]).max() / np.abs(ref["cpl"][:n]).max()
    assert cp < 1e-6, cp
    g = np.abs(out["tlg"][:b.grid_len] - ref["tlg"][:b.grid_len])
    assert np.percentile(g, 99.9) < TOL_ORACLE
    gc = np.abs(out["cpg"][:b.grid_len] - ref["cpg"][:b.grid_len]).max() / np.abs(ref["cpg"][:b.grid_len]).max()
    assert gc < 1e-6, gc


@pytest.mark.parametrize("name", CASES)
def test_cupyram_vs_reference(cuda_device, name):
    args, kw, fx = load_case(name)
    res = CuPyRAM(*args, **kw).run()
    tl = np.asarray(res["TL Line"])
    assert tl.shape == fx["tl_line"].shape
    assert np.array_equal(res["Ranges"], fx["ranges"])
    assert np.allclose(res["Depths"], fx["depths"])
    d = np.abs(tl - fx["tl_line"])
    assert d.max() <= TOL_REF, d.max()
    grid = np.asarray(res["TL Grid"])
    assert grid.shape == fx["tl_grid"].shape
    dg = np.abs(grid - fx["tl_grid"])
    assert np.percentile(dg, 99) <= TOL_REF and dg.max() <= 0.05


def test_pekeris_full_size_column_march(cuda_device):
    """The single-ray Pekeris configuration (nz 2399, 4999 steps, np 8, TL grid): the
    default policy marches it on one cluster; TL line and grid against the oracle."""
    from cupyram_b200 import workloads
    b = workloads.build(*workloads.pekeris(), compute_grids=True)
    with Engine(b) as eng:
        out = eng.run()
        st = eng.stats()
    assert st["column_rays"] == 1 and st["rays_failed"] == 0
    ref = oracle.run(b, "plain")
    n = b.line_len
    assert np.abs(out["tll"][:n] - ref["tll"][:n]).max() < TOL_ORACLE
    g = np.abs(out["tlg"][:b.grid_len] - ref["tlg"][:b.grid_len])
    assert np.percentile(g, 99.9) < TOL_ORACLE


@pytest.mark.parametrize("rays", [3, 5])
def test_column_march_deep_columns_vs_oracle(cuda_device, monkeypatch, rays):
    """Deep Munk columns (nz 5350-5800) on the column kernel: clusters of up to
    16 CTAs whose slices differ in length, against the oracle and against the
    batched kernel on the same rays."""
    from cupyram_b200 import workloads
    b = workloads.build(*workloads.munk_batch(rays, seed=5, rmax=1500.0), compute_grids=False)
    monkeypatch.setenv("CUPYRAM_B200_COL", "1")
    with Engine(b) as eng:
        out = eng.run()
        assert eng.stats()["column_rays"] == rays
    monkeypatch.setenv("CUPYRAM_B200_COL", "0")
    with Engine(b) as eng:
        bat = eng.run()
    ref = oracle.run(b, "plain")
    n = b.line_len
    assert np.abs(out["tll"][:n] - ref["tll"][:n]).max() < TOL_ORACLE
    assert np.abs(out["tll"][:n] - bat["tll"][:n]).max() < TOL_ORACLE


def test_homogeneous_batch_stays_on_the_batched_kernel(cuda_device):
    """The 4096-ray Munk batch: every ray's lockstep march is close to the
    batch's balanced time, so the default policy keeps all of them on the
    batched kernel (engine creation only, no march)."""
    from cupyram_b200 import workloads
    b = workloads.build(*workloads.munk_batch(4096, seed=2024), compute_grids=False)
    with Engine(b) as eng:
        assert eng.stats()["column_rays"] == 0


def test_ram_v15_vs_fortran(cuda_device):
    args, kw, _ = load_case("ram_v15")
    res = CuPyRAM(*args, **kw).run()
    f = np.load(GOLDEN / "ram_v15_fortran.npz")
    assert np.array_equal(res["Ranges"], f["ranges"])
    assert np.mean(np.abs(res["TL Line"] - f["tl"])) <= 0.01


def test_no_grid_still_computes_line(cuda_device):
    args, kw, fx = load_case("pekeris_small")
    res = CuPyRAM(*args, compute_grids=False, **kw).run()
    assert res["TL Grid"] is None and res["CP Grid"] is None
    assert np.abs(res["TL Line"] - fx["tl_line"]).max() <= TOL_REF


@pytest.mark.parametrize("name", ["ram_v15", "ragged_batch", "wedge_switch"])
def test_product_form_kernel_vs_oracle(cuda_device, monkeypatch, name):
    """The product-form march (used when a source sits in the first depth cell)."""
    monkeypatch.setenv("CUPYRAM_B200_SUM", "0")
    b, _ = _batch(name)
    with Engine(b) as eng:
        out = eng.run()
    ref = oracle.run(b, "plain")
    n = b.line_len
    assert np.abs(out["tll"][:n] - ref["tll"][:n]).max() < TOL_ORACLE


def test_surface_source_falls_back_to_product_form(cuda_device):
    """zs < dz puts the source in the surface row; the engine must still match."""
    args, kw, _ = load_case("pekeris_small")
    args = list(args)
    args[1] = 2.0  # zs = 2 m < dz = 3 m
    envs, p, zs, zr, pr = B.prepare(*args, dict(kw))
    b = B.build_batch(envs, p, zs, zr, pr, False)
    with Engine(b) as eng:
        out = eng.run()
    ref = oracle.run(b, "plain")
    assert np.abs(out["tll"][:b.line_len] - ref["tll"][:b.line_len]).max() < TOL_ORACLE


def _mixed_batch(n_short=3500, idx=None):
    """3500 short rays (nz 99, 59 steps) and two long ones (nz 299, 2999 steps),
    per-ray grids: a ray's lockstep march alone (0.3 us per row and step)
    exceeds 1.25x the batch's balanced time (work / 1.3e10 per s) only for the
    long rays.  idx selects a subset of the same rays."""
    long_ids = {0, n_short // 2 + 1}
    is_long = [i in long_ids for i in range(n_short + 2)]
    if idx is not None:
        is_long = [is_long[i] for i in idx]
    n = len(is_long)
    rmax = np.array([30000.0 if L else 600.0 for L in is_long])
    dep = [200.0 if L else 40.0 for L in is_long]
    args = [np.full(n, 100.0), np.full(n, 10.0), np.full(n, 10.0),
            [np.array([0.0, 250.0 if L else 60.0]) for L in is_long], [np.array([0.0])] * n,
            [np.array([[1500.0], [1500.0]])] * n, [np.array([0.0, 20.0 if L else 10.0]) for L in is_long],
            [np.array([0.0])] * n, [np.array([[1700.0], [1700.0]])] * n, [np.array([[1.5], [1.5]])] * n,
            [np.array([[0.5], [0.5]])] * n, [np.array([[0.0, d], [r, d]]) for d, r in zip(dep, rmax)]]
    kw = dict(batch_size=n, per_ray=True, dz=1.0, dr=10.0, rmax=rmax, np=4, lyrw=2)
    envs, p, zs, zr, pr = B.prepare(*args, kw)
    return B.build_batch(envs, p, zs, zr, pr, False), sorted(long_ids)


def test_mixed_batch_column_and_batched_vs_oracle(cuda_device):
    """The default policy splits this batch: the two long rays go to the column
    kernel, the short ones stay on the batched kernel, and both launches run
    concurrently.  The long rays and every 70th short ray are checked against
    the oracle (rays are independent, so a sub-batch of the same rays serves)."""
    b, longs = _mixed_batch()
    with Engine(b) as eng:
        out = eng.run()
        st = eng.stats()
    assert st["rays_failed"] == 0
    assert st["column_rays"] == 2
    idx = sorted(set(longs) | set(range(1, b.n_rays, 70)))
    sub, _ = _mixed_batch(idx=idx)
    ref = oracle.run(sub, "plain")
    for j, i in enumerate(idx):
        r, s = b.rays[i], sub.rays[j]
        assert (int(r["nvr"]), int(r["nz"])) == (int(s["nvr"]), int(s["nz"]))
        lo, so, n = int(r["line_off"]), int(s["line_off"]), int(r["nvr"])
        d = np.abs(out["tll"][lo:lo + n] - ref["tll"][so:so + n]).max()
        assert d < TOL_ORACLE, (i, d)
        c = np.abs(out["cpl"][lo:lo + n] - ref["cpl"][so:so + n]).max() / np.abs(ref["cpl"][so:so + n]).max()
        assert c < 1e-6, (i, c)
