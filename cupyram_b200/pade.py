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


def pade_batch(freq, c0, np_pade, ns, dr, ip):
    """Pade coefficients of many jobs at once, solved on the current CUDA device
    (cr_pade_batch, one thread per job, the same FP64 construction as
    :func:`compute_pade_coefficients`).  Every argument is a scalar or an array
    broadcast to the batch.  Returns ``(pd1, pd2, status)``: complex128
    ``[n, CR_MAX_NP]`` arrays (zeros past each job's np) and the per-job
    status (0 ok, 3 Laguerre not converging).  Raises ``ValueError`` when any
    job fails, with the first failing job's index."""
    lib = _lib.load()
    f, c, npp, s, d, i = np.broadcast_arrays(np.asarray(freq, np.float64), np.asarray(c0, np.float64),
                                             np.asarray(np_pade, np.int32), np.asarray(ns, np.int32),
                                             np.asarray(dr, np.float64), np.asarray(ip, np.int32))
    f, c, d = (np.ascontiguousarray(x, np.float64).reshape(-1) for x in (f, c, d))
    npp, s, i = (np.ascontiguousarray(x, np.int32).reshape(-1) for x in (npp, s, i))
    n = f.size
    pd1 = np.zeros((n, _lib.MAX_NP), np.complex128)
    pd2 = np.zeros((n, _lib.MAX_NP), np.complex128)
    status = np.zeros(n, np.int32)
    rc = lib.cr_pade_batch(n, f.ctypes.data, c.ctypes.data, npp.ctypes.data, s.ctypes.data, d.ctypes.data,
                           i.ctypes.data, pd1.ctypes.data, pd2.ctypes.data, status.ctypes.data)
    if rc not in (_lib.CR_OK, _lib.CR_EPADE):
        _lib.check(rc)
    return pd1, pd2, status


def compute_pade_coefficients_batch(freq, c0_array, np_pade, ns, dr, ip, max_workers=8):
    """[np_pade, batch] coefficients for a batch of reference sound speeds
    (cupyram/pade.py:276-317), on the host like the reference's; the engine
    itself solves its Pade sets on the device (:func:`pade_batch`)."""
    c0 = np.asarray(c0_array, dtype=np.float64).reshape(-1)
    pd1 = np.zeros((int(np_pade), c0.size), np.complex128)
    pd2 = np.zeros_like(pd1)
    for b, c in enumerate(c0):
        pd1[:, b], pd2[:, b] = compute_pade_coefficients(freq, c, np_pade, ns, dr, ip)
    return pd1, pd2
