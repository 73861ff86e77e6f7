"""Parity on rays of the benchmark's own uneven wedge batch, not only the golden cases.

Twelve rays are drawn from the 10,000-ray wedge generator (the benchmark's
uneven-batch configuration: per-ray slope, bottom, frequency log-U[25,500] Hz,
np U{4..8}, dr = lambda/4, dz = lambda/8): for every Pade order the lowest-
and the highest-frequency ray, plus two more.  The march range is cut to
5 km (the generator's shortest) so that the oracle finishes in seconds; the depth grids (nz up to ~1500),
the sloping bottoms (the bathymetry index moves during the march), the
operators and the Pade sets are those of the full batch.

Every ray is marched on both kernels (batched warp tiles and one cluster per
ray) and by the default schedule, in the plain and the chosen form, against
the oracle's plain complex128 march of the same rays.  Bars as for the golden
cases: plain 1e-3 dB on the TL line; chosen RMS <= 0.1 dB and max <= 1 dB
over cells with TL < 100 dB.  This matches the reference's own wedge bar
(tests/test_wedge.py:340-351, 0.5 dB against PyRAM) with a wide margin.
"""
import numpy as np
import pytest

from cupyram_b200 import workloads
from cupyram_b200.engine import Engine
from oracle import oracle

pytestmark = pytest.mark.gpu

TOL_PLAIN = 1e-3
RMS_CHOSEN, MAX_CHOSEN = 0.1, 1.0
RMAX = 5000.0


def _pick(args, kw):
    """Indices of the sample: per np, the lowest- and highest-frequency rays, and two more."""
    f = np.asarray(args[0])
    npp = np.asarray(kw["np"])
    idx = []
    for p in range(4, 9):
        sel = np.flatnonzero(npp == p)
        idx += [int(sel[np.argmin(f[sel])]), int(sel[np.argmax(f[sel])])]
    idx += [17, 4242]
    return sorted(set(idx))


def _subset(args, kw, idx):
    sub_args = [np.asarray(a)[idx] if isinstance(a, np.ndarray) else [a[i] for i in idx] for a in args]
    sub_kw = {k: (np.asarray(v)[idx] if isinstance(v, np.ndarray) else v) for k, v in kw.items()}
    sub_kw["batch_size"] = len(idx)
    sub_kw["rmax"] = np.full(len(idx), RMAX)
    return sub_args, sub_kw


@pytest.fixture(scope="module")
def wedge_sample():
    args, kw = workloads.wedge_batch(10000, seed=7)
    idx = _pick(args, kw)
    b = workloads.build(*_subset(args, kw, idx), compute_grids=False)
    assert b.n_rays == len(idx) >= 8
    ref = oracle.run(b, "plain")
    return b, ref


def _lines(b, out, ref):
    for i in range(b.n_rays):
        o, n = int(b.rays["line_off"][i]), int(b.rays["nvr"][i])
        yield i, out["tll"][o:o + n], ref["tll"][o:o + n]


@pytest.mark.parametrize("schedule", ["batched", "column", "default"])
def test_wedge_rays_plain_vs_oracle(cuda_device, monkeypatch, wedge_sample, schedule):
    b, ref = wedge_sample
    if schedule == "default":
        monkeypatch.delenv("CUPYRAM_B200_COL", raising=False)
    else:
        monkeypatch.setenv("CUPYRAM_B200_COL", "0" if schedule == "batched" else "1")
    with Engine(b) as eng:
        out = eng.run()
        st = eng.stats()
    assert st["rays_failed"] == 0
    if schedule != "default":
        assert st["column_rays"] == (b.n_rays if schedule == "column" else 0)
    for i, tl, tr in _lines(b, out, ref):
        d = np.abs(tl - tr).max()
        assert d < TOL_PLAIN, (i, float(b.rays["freq"][i]), int(b.rays["np"][i]), d)


@pytest.mark.parametrize("schedule", ["batched", "column"])
def test_wedge_rays_chosen_vs_oracle(cuda_device, monkeypatch, wedge_sample, schedule):
    b, ref = wedge_sample
    monkeypatch.setenv("CUPYRAM_B200_COL", "0" if schedule == "batched" else "1")
    with Engine(b, precision="chosen") as eng:
        out = eng.run()
    d = np.concatenate([np.abs(tl - tr)[tr < 100.0] for _, tl, tr in _lines(b, out, ref)])
    assert np.sqrt(np.mean(d * d)) <= RMS_CHOSEN and d.max() <= MAX_CHOSEN, (np.sqrt(np.mean(d * d)), d.max())


def test_work_queue_matches_per_order_launches(cuda_device, monkeypatch, wedge_sample):
    """The persistent launch that takes tiles from the device work queue (any mix
    of lanes per ray; np 4..8 gives 2..4 lanes) gives bit-identical lines to one
    launch per lanes-per-ray value: the same tile code, only the order in which
    CTAs take the tiles differs."""
    b, ref = wedge_sample
    monkeypatch.setenv("CUPYRAM_B200_COL", "0")
    outs = {}
    for q in ("1", "0"):
        monkeypatch.setenv("CUPYRAM_B200_QUEUE", q)
        with Engine(b) as eng:
            outs[q] = eng.run()
            st = eng.stats()
        assert (st["queue_ctas"] > 0) == (q == "1")
        # the queue: one launch; otherwise one per run of tiles of equal lanes per ray
        assert st["kernel_launches"] == 1 if q == "1" else 1 <= st["kernel_launches"] <= 3
    assert np.array_equal(outs["1"]["tll"][:b.line_len], outs["0"]["tll"][:b.line_len])
    assert np.array_equal(outs["1"]["cpl"][:b.line_len], outs["0"]["cpl"][:b.line_len])


def test_tuner_costs_are_measured(cuda_device, monkeypatch, wedge_sample):
    """The default policy reports the batched costs the engine's tuner measured on
    this device (cr_stats.tuner_*), and they are of a plausible size."""
    b, _ = wedge_sample
    monkeypatch.delenv("CUPYRAM_B200_COL", raising=False)
    monkeypatch.delenv("CUPYRAM_B200_COSTS", raising=False)
    with Engine(b) as eng:
        st = eng.stats()
    assert 1e-8 < st["tuner_row_step_s"] < 1e-4
    assert 1e8 < st["tuner_updates_per_s"] < 1e12
