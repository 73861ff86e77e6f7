"""The CPU oracle, pinned against the reference's own outputs.

* tests/golden/<case>.npz - the unmodified reference (clapeyre/cupyram) run on
  CPU under Numba's CUDA simulator by tests/golden/make_golden.py;
* tests/golden/ram_v15_fortran.npz - RAM v1.5's Fortran TL line (the
  reference's tests/tl_ref.line), pinned by the reference at mean |dTL| <= 0.01 dB
  (tests/test_reference.py:28,192);
* tests/golden/pade_ref.npz - the reference's pade.py, pinned at abs 1e-8
  (tests/test_pade_coefficients.py:23).
"""
import numpy as np
import pytest

from golden_cases import CASES, GOLDEN, load_case
from cupyram_b200 import batch as B
from oracle import oracle

# dB tolerances on the TL line (plain engine vs the reference: 0.01 dB)
TOL_LINE = 0.01
# simulator-promotion mode reproduces the fixtures at rounding level
TOL_SIM = 1e-3


def _prep(name, compute_grids=True):
    args, kw, fx = load_case(name)
    envs, p, zs, zr, per_ray = B.prepare(*args, dict(kw))
    b = B.build_batch(envs, p, zs, zr, per_ray, compute_grids)
    return b, fx


@pytest.mark.parametrize("name", CASES)
def test_grid_matches_reference(name):
    b, fx = _prep(name)
    assert int(b.nz[0]) == int(fx["nz"])
    assert b.zmax[0] == pytest.approx(float(fx["zmax"]), rel=1e-12)
    assert np.array_equal(b.vr[0], fx["ranges"])
    assert np.allclose(b.vz[0], fx["depths"])


@pytest.mark.parametrize("mode", ["sim", "ref", "plain", "f64"])
@pytest.mark.parametrize("name", CASES)
def test_oracle_tl_line_vs_reference(name, mode):
    b, fx = _prep(name)
    out = oracle.run(b, mode)
    n, nvr = b.n_rays, int(b.nvr[0])
    tl = out["tll"][: n * nvr].reshape(fx["tl_line"].shape)
    d = np.abs(tl - fx["tl_line"])
    assert np.all(np.isfinite(tl))
    assert d.max() <= (TOL_SIM if mode == "sim" else TOL_LINE), d.max()


@pytest.mark.parametrize("name", CASES)
def test_oracle_cp_line_vs_reference(name):
    b, fx = _prep(name)
    out = oracle.run(b, "sim")
    n, nvr = b.n_rays, int(b.nvr[0])
    cp = out["cpl"][: n * nvr].reshape(fx["cp_line"].shape)
    rel = np.max(np.abs(cp - fx["cp_line"])) / np.max(np.abs(fx["cp_line"]))
    assert rel < 1e-5, rel


@pytest.mark.parametrize("name", CASES)
def test_oracle_tl_grid_vs_reference(name):
    b, fx = _prep(name)
    out = oracle.run(b, "plain")
    n, nvr, nvz = b.n_rays, int(b.nvr[0]), int(b.nvz[0])
    tg = out["tlg"][: n * nvz * nvr].reshape(fx["tl_grid"].shape)
    d = np.abs(tg - fx["tl_grid"])
    # grid cells include interference nulls, where dTL amplifies rounding:
    # the bulk is held to 0.01 dB, every cell to 0.05 dB
    assert np.percentile(d, 99) <= TOL_LINE
    assert d.max() <= 0.05


@pytest.mark.parametrize("mode", ["ref", "plain", "f64"])
def test_oracle_vs_ram_fortran(mode):
    """RAM v1.5 test case against the Fortran output (mean |dTL| <= 0.01 dB)."""
    b, _ = _prep("ram_v15")
    f = np.load(GOLDEN / "ram_v15_fortran.npz")
    assert np.array_equal(b.vr[0], f["ranges"])
    out = oracle.run(b, mode)
    tl = out["tll"][: int(b.nvr[0])]
    d = np.abs(tl - f["tl"])
    assert d.mean() <= 0.01, d.mean()


def test_oracle_pade_vs_reference():
    d = np.load(GOLDEN / "pade_ref.npz")
    worst = 0.0
    for row, p1, p2 in zip(d["params"], d["pd1"], d["pd2"]):
        np_, ns, ip, freq, dr, c0 = row
        a, c = oracle.pade(freq, c0, int(np_), int(ns), dr, int(ip))
        n = int(np_)
        worst = max(worst, np.max(np.abs(a - p1[:n])), np.max(np.abs(c - p2[:n])))
    assert worst < 1e-8, worst


def test_oracle_batch_rays_independent():
    """A ray's result does not depend on the other rays of its batch."""
    b, _ = _prep("ragged_batch")
    full = oracle.run(b, "plain")
    for k in range(b.n_rays):
        one = oracle.run(b, "plain", rays=[k])
        lo, n = int(b.rays["line_off"][k]), int(b.rays["nvr"][k])
        # the single-ray run starts its line at the ray's own offset
        assert np.array_equal(one["tll"][lo:lo + n], full["tll"][lo:lo + n])


@pytest.mark.parametrize("name", ["mini_munk", "wedge_switch", "pekeris_small"])
def test_chosen_form_models(name):
    """The oracle's chosen-form models (complex64 sweeps; FP64 or FP32 term
    combination; FP64 or FP32 coupling) round, and on these short cases stay
    within 0.01 dB RMS of the FP64 sum form over cells with TL < 100 dB
    (the next test runs them at the Munk workload's full range)."""
    b, _ = _prep(name, False)
    ref = oracle.run(b, "sum")["tll"][: b.line_len]
    lit = ref < 100.0
    for mode in ("chosen", "chosen_c32", "chosen_f32"):
        d = (oracle.run(b, mode)["tll"][: b.line_len] - ref)[lit]
        assert 1e-7 < np.abs(d).max() and np.sqrt(np.mean(d * d)) < 0.01, (mode, np.abs(d).max())


def test_chosen_form_models_at_full_range():
    """Two full-range rays of the 4096-ray Munk batch (1999 steps, nz ~ 5600):
    the chosen-form model stays within 0.01 dB RMS of the FP64 sum form, and
    the all-FP32 inner loop within the chosen form's 0.1 dB RMS bar (cells with
    TL < 100 dB)."""
    from cupyram_b200 import workloads
    b = workloads.build(*workloads.munk_batch(4096, seed=2024), compute_grids=False)
    rays = [0, 2048]
    r = b.rays[rays]

    def lines(mode):
        out = oracle.run(b, mode, rays=rays)["tll"]
        return [out[int(x["line_off"]): int(x["line_off"]) + int(x["nvr"])] for x in r]

    ref = lines("sum")
    for mode, bar in (("chosen", 0.01), ("chosen_f32", 0.1)):
        for a, c in zip(ref, lines(mode)):
            d = (c - a)[a < 100.0]
            assert np.sqrt(np.mean(d * d)) < bar, (mode, np.sqrt(np.mean(d * d)))


@pytest.mark.parametrize("name", ["mini_munk", "wedge_switch", "pekeris_small"])
def test_refinement_model_recovers_fp64(name):
    """The refined form's model: one FP64-residual correction per complex64 solve
    brings the march back to the FP64 sum form (here to ~1e-10 dB), at least a
    thousand times closer than the unrefined chosen model."""
    b, _ = _prep(name, False)
    ref = oracle.run(b, "sum")["tll"][: b.line_len]
    lit = ref < 100.0
    rms = {}
    for mode in ("chosen", "refined"):
        d = (oracle.run(b, mode)["tll"][: b.line_len] - ref)[lit]
        rms[mode] = np.sqrt(np.mean(d * d))
    assert rms["refined"] < 1e-3 * rms["chosen"] and rms["refined"] < 1e-8, rms
