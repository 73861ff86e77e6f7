"""The reduced-precision forms against plain complex128: "chosen" (complex64
factors / workspace, FP32 sweeps, terms combined in FP64) and "fast" (the same
with an FP32 inner loop: couplings, M u and the term combination in FP32).

Accuracy bar: RMS TL error <= 0.1 dB against the FP64 (plain) march over the
cells with TL < 100 dB; every such cell within 1 dB.
"""
import numpy as np
import pytest

from golden_cases import CASES, load_case
from cupyram_b200 import batch as B, workloads
from cupyram_b200.engine import Engine

pytestmark = pytest.mark.gpu

RMS_DB = 0.1
MAX_DB = 1.0


def _errs(ref, tl):
    m = ref < 100.0
    d = np.abs(tl[m] - ref[m])
    return d.max(), np.sqrt(np.mean(d * d))


@pytest.mark.parametrize("form", ["chosen", "fast", "refined"])
@pytest.mark.parametrize("march", ["batched", "column"])
@pytest.mark.parametrize("name", CASES)
def test_chosen_vs_plain_golden(cuda_device, monkeypatch, name, march, form):
    monkeypatch.setenv("CUPYRAM_B200_COL", "0" if march == "batched" else "1")
    args, kw, _ = load_case(name)
    envs, p, zs, zr, pr = B.prepare(*args, dict(kw))
    b = B.build_batch(envs, p, zs, zr, pr, True)
    with Engine(b, precision="plain") as e1:
        ref = e1.run()
    with Engine(b, precision=form) as e2:
        out = e2.run()
    n = b.line_len
    mx, rms = _errs(ref["tll"][:n], out["tll"][:n])
    assert rms <= RMS_DB and mx <= MAX_DB, (mx, rms)
    g = b.grid_len
    mx, rms = _errs(ref["tlg"][:g], out["tlg"][:g])
    assert rms <= RMS_DB, (mx, rms)


@pytest.mark.parametrize("form", ["chosen", "fast", "refined"])
def test_chosen_vs_plain_munk_batch(cuda_device, form):
    b = workloads.build(*workloads.munk_batch(160, seed=11, rmax=20000.0), compute_grids=False)
    with Engine(b, precision="plain") as e1:
        ref = e1.run()
    with Engine(b, precision=form) as e2:
        out = e2.run()
    mx, rms = _errs(ref["tll"][:b.line_len], out["tll"][:b.line_len])
    assert rms <= RMS_DB and mx <= MAX_DB, (mx, rms)


@pytest.mark.parametrize("form", ["chosen", "fast", "refined"])
def test_reduced_forms_run_surface_sources(cuda_device, form):
    """zs < dz puts the source in the surface row, where only the product-form march
    applies; the reduced forms then run it in complex128 (reported in
    cr_stats.precision_used) and match the oracle like the plain form."""
    from oracle import oracle
    from cupyram_b200 import _lib
    args, kw, _ = load_case("pekeris_small")
    args = list(args)
    args[1] = 2.0  # zs = 2 m < dz = 3 m
    envs, p, zs, zr, pr = B.prepare(*args, dict(kw))
    b = B.build_batch(envs, p, zs, zr, pr, False)
    with Engine(b, precision=form) as eng:
        out = eng.run()
        assert eng.stats()["precision_used"] == _lib.CR_PLAIN_C128
    ref = oracle.run(b, "plain")
    assert np.abs(out["tll"][:b.line_len] - ref["tll"][:b.line_len]).max() < 1e-3


def test_refinement_step_recovers_complex128(cuda_device, monkeypatch):
    """The refined form's FP64-residual correction removes the complex64 solves'
    error: on Munk rays its TL line meets the plain form's parity bar against the
    oracle's complex128 march (1e-3 dB), far closer than the unrefined chosen
    form (the oracle's model of the refinement recovers FP64 to ~1e-10 dB)."""
    from oracle import oracle
    monkeypatch.setenv("CUPYRAM_B200_COL", "0")
    b = workloads.build(*workloads.munk_batch(64, seed=13, rmax=20000.0), compute_grids=False)
    outs = {}
    for form in ("chosen", "refined"):
        with Engine(b, precision=form) as eng:
            outs[form] = eng.run()["tll"][:b.line_len]
    sample = [0, 21, 42, 63]
    ref = oracle.run(b, "plain", rays=sample)["tll"]
    for i in sample:
        o, n = int(b.rays["line_off"][i]), int(b.rays["nvr"][i])
        d_r = np.abs(outs["refined"][o:o + n] - ref[o:o + n])
        d_c = np.abs(outs["chosen"][o:o + n] - ref[o:o + n])
        assert d_r.max() < 1e-3 and d_r.max() < 0.1 * d_c.max(), (i, d_r.max(), d_c.max())
