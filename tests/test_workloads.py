"""The benchmark workloads as specified (CPU): grid sizes, seeded value ranges
and the exact grid-point update counts that the benchmark lines report."""
import numpy as np

from cupyram_b200 import workloads as W


def test_pekeris_grid():
    """50 Hz, 100 m water over 200 m of sediment, 10-wavelength layer: zmax
    600 m, so nz 2399 at dz 0.25; rmax 10 km at dr 2 m: 4999 steps, 5000
    outputs; TL grid every 4th row to zmplt 100 m: 100 depths."""
    b = W.build(*W.pekeris(), compute_grids=True)
    r = b.rays[0]
    assert (int(r["nz"]), int(r["nr"]), int(r["nvr"]), int(r["nvz"]), int(r["np"])) == (2399, 4999, 5000, 100, 8)
    assert b.point_updates == 2399 * 4999


def test_munk_batch():
    args, kw = W.munk_batch()
    b = W.build(args, kw)
    r = b.rays
    assert b.n_rays == 4096 and np.all(r["np"] == 6) and np.all(r["nr"] == 1999)
    assert np.all((r["freq"] >= 50.0) & (r["freq"] <= 200.0)) and np.all((r["zs"] >= 50.0) & (r["zs"] <= 1000.0))
    assert np.all(r["dr"] == 25.0) and np.all(r["dz"] == 1.0) and np.all(r["zr"] == 500.0)
    assert len(args[3][0]) == 501 and np.array_equal(args[4][0], np.arange(0.0, 50000.0, 5000.0))
    assert args[5][0].shape == (501, 10)
    assert b.point_updates == 44858653453.0
    c = np.asarray(args[5])
    pert = c - W.munk_speed(args[3][0])[None, :, None]
    assert 1.8 < pert.std() < 2.2  # sigma 2 m/s


def test_wedge_batch():
    args, kw = W.wedge_batch(10000, seed=2024)  # the benchmark's seed
    b = W.build(args, kw)
    r = b.rays
    lam = 1500.0 / r["freq"]
    assert b.n_rays == 10000
    assert np.all((r["freq"] >= 25.0) & (r["freq"] <= 500.0)) and set(np.unique(r["np"])) == {4, 5, 6, 7, 8}
    assert np.allclose(r["dr"], lam / 4.0) and np.allclose(r["dz"], lam / 8.0)
    rmax = np.asarray(kw["rmax"])
    assert np.all((rmax >= 5000.0) & (rmax <= 40000.0))
    assert b.point_updates == 64345723879.0
