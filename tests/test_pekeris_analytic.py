"""The Pekeris waveguide against its normal-mode solution (oracle/pekeris_modes.py).

The configuration is the single-ray Pekeris case: 50 Hz, zs = zr = 50 m,
100 m of 1500 m/s water over a 1700 m/s, 1.5 g/cm3, 0.5 dB/lambda bottom,
dr 2 m, dz 0.25 m, np 8.  Over ranges of 2-10 km (20-100 water depths, where
the trapped modes carry the field) the march's TL line agrees with the
three-mode solution to a mean of 0.011 dB, 0.38 dB RMS and 0.77 dB at most.
The residual is the small wavenumber error of the discretised, Pade-
approximated march, seen as a slowly growing phase offset of the mode
interference.  Bars: |mean| <= 0.05 dB, RMS <= 0.5 dB, max <= 1 dB.
"""
import numpy as np
import pytest

from cupyram_b200 import workloads
from oracle import pekeris_modes as PM

MEAN_DB, RMS_DB, MAX_DB = 0.05, 0.5, 1.0


def _analytic(b):
    r = b.rays[0]
    nvr = int(r["nvr"])
    ranges = (np.arange(nvr) + 1) * float(r["dr"]) * int(r["ndr"])
    return ranges, PM.tl(50.0, 100.0, 1500.0, 1700.0, 1.0, 1.5, 0.5, zs=50.0, z=50.0, r=ranges)


def _check(ranges, tl, tl_nm):
    m = ranges >= 2000.0
    d = tl[m] - tl_nm[m]
    assert abs(d.mean()) <= MEAN_DB, d.mean()
    assert np.sqrt(np.mean(d * d)) <= RMS_DB, np.sqrt(np.mean(d * d))
    assert np.abs(d).max() <= MAX_DB, np.abs(d).max()


def test_modes_of_the_pekeris_guide():
    krs, k1, k2 = PM.modes(50.0, 100.0, 1500.0, 1700.0, 1.0, 1.5, 0.5)
    assert len(krs) == 3
    assert np.all((krs.real > k2.real) & (krs.real < k1))
    assert np.all(krs.imag > 0)  # attenuated by the lossy bottom


def test_restatement_matches_normal_modes():
    from oracle import oracle
    b = workloads.build(*workloads.pekeris(), compute_grids=False)
    out = oracle.run(b, "plain")
    ranges, tl_nm = _analytic(b)
    _check(ranges, out["tll"][: ranges.size], tl_nm)


@pytest.mark.gpu
def test_engine_matches_normal_modes(cuda_device):
    from cupyram_b200.engine import Engine
    b = workloads.build(*workloads.pekeris(), compute_grids=False)
    with Engine(b) as eng:
        out = eng.run()
    ranges, tl_nm = _analytic(b)
    _check(ranges, out["tll"][: ranges.size], tl_nm)
