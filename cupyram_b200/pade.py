"""Pade coefficients (host FP64, native).

``compute_pade_coefficients`` keeps the signature and return values of the
reference's ``cupyram/pade.py:180-273``: two complex128 arrays of length
``np_pade`` (product-form numerator and denominator coefficients).  A failed
Laguerre iteration raises ``ValueError('Laguerre method not converging')``
as the reference does (``pade.py:146-147``).
"""
import numpy as np

from . import _lib


def compute_pade_coefficients(freq, c0, np_pade, ns=1, dr=50.0, ip=1):
    lib = _lib.load()
    n = int(np_pade)
    if n < 1 or n > _lib.MAX_NP:
        raise ValueError(f"np_pade must be in 1..{_lib.MAX_NP}")
    pd1 = np.zeros(n, np.complex128)
    pd2 = np.zeros(n, np.complex128)
    rc = lib.cr_pade(float(freq), float(c0), n, int(ns), float(dr), int(ip), pd1.ctypes.data,
                     pd2.ctypes.data)
    _lib.check(rc)
    return pd1, pd2


def compute_pade_coefficients_batch(freq, c0_array, np_pade, ns, dr, ip, max_workers=8):
    """[np_pade, batch] coefficients for a batch of reference sound speeds."""
    c0 = np.asarray(c0_array, dtype=np.float64).reshape(-1)
    pd1 = np.zeros((int(np_pade), c0.size), np.complex128)
    pd2 = np.zeros_like(pd1)
    for b, c in enumerate(c0):
        pd1[:, b], pd2[:, b] = compute_pade_coefficients(freq, c, np_pade, ns, dr, ip)
    return pd1, pd2
