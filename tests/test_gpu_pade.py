"""Device Pade (cr_pade_batch, the path cr_create takes) against the reference's own coefficients.

tests/golden/pade_ref.npz holds 2,760 coefficient sets computed by the
reference's cupyram/pade.py:180-273 (np 1..8, ns 0..2, ip 1 and 2, several
frequencies, range steps and reference sound speeds).  All of them are solved
in one device launch and compared at the reference's own bar
(tests/test_pade_coefficients.py:23: 1e-8 absolute on real and imaginary
parts).  The engine's Pade sets are checked through the same entry point; a
set whose Laguerre search fails reports its job.
"""
import numpy as np
import pytest

from cupyram_b200 import compute_pade_coefficients
from cupyram_b200.pade import pade_batch
from golden_cases import GOLDEN

pytestmark = pytest.mark.gpu


def test_device_pade_vs_reference_fixtures(cuda_device):
    d = np.load(GOLDEN / "pade_ref.npz")
    npp, ns, ip, freq, dr, c0 = (d["params"][:, k] for k in range(6))
    pd1, pd2, status = pade_batch(freq, c0, npp.astype(int), ns.astype(int), dr, ip.astype(int))
    assert not np.any(status)
    worst = 0.0
    for k in range(len(npp)):
        n = int(npp[k])
        worst = max(worst, np.abs(pd1[k, :n] - d["pd1"][k, :n]).max(), np.abs(pd2[k, :n] - d["pd2"][k, :n]).max())
        assert not np.any(pd1[k, n:]) and not np.any(pd2[k, n:])
    assert worst < 1e-8, worst


def test_device_pade_matches_host_pade(cuda_device):
    """Device and host (cr_pade) solve the same FP64 construction."""
    rng = np.random.default_rng(5)
    n = 64
    f = rng.uniform(20.0, 500.0, n)
    dr = rng.uniform(5.0, 100.0, n)
    npp = rng.integers(2, 11, n)
    pd1, pd2, status = pade_batch(f, 1500.0, npp, 1, dr, 1)
    assert not np.any(status)
    for k in range(n):
        q1, q2 = compute_pade_coefficients(f[k], 1500.0, int(npp[k]), ns=1, dr=dr[k], ip=1)
        assert np.abs(pd1[k, :npp[k]] - q1).max() < 1e-9 and np.abs(pd2[k, :npp[k]] - q2).max() < 1e-9


def test_device_pade_reports_a_failing_job(cuda_device):
    """np 10, ip 2, ns 1 at sigma = k0 dr = 0.19: the Laguerre search does not converge
    (as on the host); the other jobs of the launch are unaffected."""
    f = np.array([50.0, 50.0, 50.0])
    dr = np.array([10.0, 0.9076932507005218, 25.0])
    pd1, pd2, status = pade_batch(f, 1500.0, 10, 1, dr, 2)
    assert list(status) == [0, 3, 0]
    assert not np.any(pd1[1]) and np.any(pd1[0]) and np.any(pd1[2])
