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


@pytest.mark.parametrize("form", ["chosen", "fast"])
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


@pytest.mark.parametrize("form", ["chosen", "fast"])
def test_chosen_vs_plain_munk_batch(cuda_device, form):
    b = workloads.build(*workloads.munk_batch(160, seed=11, rmax=20000.0), compute_grids=False)
    with Engine(b, precision="plain") as e1:
        ref = e1.run()
    with Engine(b, precision=form) as e2:
        out = e2.run()
    mx, rms = _errs(ref["tll"][:b.line_len], out["tll"][:b.line_len])
    assert rms <= RMS_DB and mx <= MAX_DB, (mx, rms)


def test_chosen_rejected_for_surface_source(cuda_device):
    args, kw, _ = load_case("pekeris_small")
    args = list(args)
    args[1] = 2.0  # zs < dz: product-form fallback, which has no chosen form
    envs, p, zs, zr, pr = B.prepare(*args, dict(kw))
    b = B.build_batch(envs, p, zs, zr, pr, False)
    with pytest.raises(ValueError, match="chosen"):
        Engine(b, precision="chosen")
