"""Device Pade (cr_pade_batch, the path cr_create takes) against the reference's own coefficients.

tests/golden/pade_ref.npz holds 2,760 coefficient sets computed by the
reference's cupyram/pade.py:180-273 (np 1..8, ns 0..2, ip 1 and 2, several
frequencies, range steps and reference sound speeds).  All of them are solved
in one device launch and compared at the reference's own bar
(tests/test_pade_coefficients.py:23: 1e-8 absolute on real and imaginary
parts).  The engine's Pade sets are checked through the same entry point; a
set whose Laguerre search fails reports its job.

The coefficients are compared as sets: the order in which Laguerre's method
with deflation finds the roots is the order of the returned terms, and a
different last bit can change it; the step operator, a product (or a sum of
partial fractions) over the terms, does not depend on it.
"""
import numpy as np
import pytest

from cupyram_b200 import compute_pade_coefficients
from cupyram_b200.pade import pade_batch
from golden_cases import GOLDEN

pytestmark = pytest.mark.gpu


def _set_dist(a, b):
    """Largest |a_i - b_match(i)| (real and imaginary parts) under the nearest
    one-to-one matching of two coefficient sets of equal size."""
    rest = list(b)
    worst = 0.0
    for x in a:
        j = int(np.argmin([abs(x - y) for y in rest]))
        y = rest.pop(j)
        worst = max(worst, abs(x.real - y.real), abs(x.imag - y.imag))
    return worst


def test_device_pade_vs_reference_fixtures(cuda_device):
    d = np.load(GOLDEN / "pade_ref.npz")
    npp, ns, ip, freq, dr, c0 = (d["params"][:, k] for k in range(6))
    pd1, pd2, status = pade_batch(freq, c0, npp.astype(int), ns.astype(int), dr, ip.astype(int))
    assert not np.any(status)
    worst = 0.0
    for k in range(len(npp)):
        n = int(npp[k])
        worst = max(worst, _set_dist(pd1[k, :n], d["pd1"][k, :n]), _set_dist(pd2[k, :n], d["pd2"][k, :n]))
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
        assert _set_dist(pd1[k, :npp[k]], q1) < 1e-9 and _set_dist(pd2[k, :npp[k]], q2) < 1e-9


def test_device_pade_reports_a_failing_job(cuda_device):
    """Settings whose Laguerre search does not converge on the device are reported
    per job (status 3) with zero coefficients, and the other jobs of the launch
    are unaffected: a seeded sweep of small range steps at np 8..10 finds some."""
    rng = np.random.default_rng(11)
    n = 4096
    dr = np.exp(rng.uniform(np.log(5e-4), np.log(5.0), n))
    npp = rng.integers(8, 11, n)
    ns = rng.integers(0, 3, n)
    ip = rng.integers(1, 3, n)
    pd1, pd2, status = pade_batch(50.0, 1500.0, npp, ns, dr, ip)
    assert set(np.unique(status)) <= {0, 3}
    bad = status == 3
    assert bad.any() and (~bad).sum() > n // 2
    assert not np.any(pd1[bad]) and not np.any(pd2[bad])
    assert np.all(np.any(pd1[~bad] != 0, axis=1))
