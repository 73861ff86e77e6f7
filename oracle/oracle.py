"""ctypes harness of the CPU oracle (TEST INFRASTRUCTURE - never imported by the product).

``run(batch, mode)`` marches every ray of a packed ``cupyram_b200.batch.Batch``
with the C restatement in ``ram_oracle.c`` and returns the same output
buffers the engine fills (tll, cpl and, with grids, tlg, cpg).

Modes: ``"ref"`` (the reference's float32 / complex64 storage and workspace
roundings), ``"plain"`` (the engine's plain complex128 form), ``"f64"``
(everything FP64), ``"sum"`` (plain in partial-fraction form) and the
chosen-form models ``"chosen"``, ``"chosen_c32"``, ``"chosen_f32"`` and the
refined form's model ``"refined"`` (see ram_oracle.c).  Parity of the oracle itself is pinned by
tests/test_oracle.py against tests/golden/ (the reference run on CPU under
Numba's CUDA simulator) and RAM v1.5's published TL line.
"""
import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "libram_oracle.so"
MODES = {"ref": 0, "plain": 1, "f64": 2, "sim": 3, "sum": 4, "chosen": 5, "chosen_c32": 6, "chosen_f32": 7,
         "refined": 8}
_lib = None


def build(force=False):
    src = HERE / "ram_oracle.c"
    hdr = HERE.parent / "include" / "cupyram_b200.h"
    if force or not LIB.exists() or LIB.stat().st_mtime < max(src.stat().st_mtime, hdr.stat().st_mtime):
        subprocess.run(["make", "-s", "-B" if force else "-C", str(HERE)] if force else
                       ["make", "-s", "-C", str(HERE)], check=True)
    return LIB


def load():
    global _lib
    if _lib is None:
        build()
        lib = ctypes.CDLL(str(LIB))
        lib.ram_oracle_run.restype = ctypes.c_int
        lib.ram_oracle_run.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                       ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
        lib.ram_oracle_pade.restype = ctypes.c_int
        lib.ram_oracle_pade.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                        ctypes.c_double, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
        _lib = lib
    return _lib


class _Batch(ctypes.Structure):
    _fields_ = [("n_rays", ctypes.c_int32), ("n_envs", ctypes.c_int32),
                ("rays", ctypes.c_void_p), ("envs", ctypes.c_void_p), ("pool", ctypes.c_void_p),
                ("pool_len", ctypes.c_int64), ("precision", ctypes.c_int32),
                ("compute_grids", ctypes.c_int32), ("line_len", ctypes.c_int64),
                ("grid_len", ctypes.c_int64)]


def run(batch, mode="plain", threads=None, rays=None):
    """March the batch (or the subset of ray indices ``rays``) on the host."""
    lib = load()
    r = np.ascontiguousarray(batch.rays if rays is None else batch.rays[np.asarray(rays)])
    e = np.ascontiguousarray(batch.envs)
    pool = np.ascontiguousarray(batch.pool, dtype=np.float64)
    line_len = int(np.max(r["line_off"] + r["nvr"])) if len(r) else 0
    grid_len = int(np.max(r["grid_off"] + r["nvz"] * r["nvr"])) if (len(r) and batch.compute_grids) else 0
    tll = np.zeros(max(line_len, 1))
    cpl = np.zeros(max(line_len, 1), np.complex128)
    tlg = np.zeros(max(grid_len, 1)) if batch.compute_grids else None
    cpg = np.zeros(max(grid_len, 1), np.complex128) if batch.compute_grids else None
    d = _Batch(len(r), len(e), r.ctypes.data, e.ctypes.data, pool.ctypes.data, pool.size, 0,
               1 if batch.compute_grids else 0, line_len, grid_len)
    nthr = threads or os.cpu_count() or 1
    rc = lib.ram_oracle_run(ctypes.byref(d), MODES[mode], tll.ctypes.data, cpl.ctypes.data,
                            tlg.ctypes.data if tlg is not None else None,
                            cpg.ctypes.data if cpg is not None else None, int(nthr))
    if rc != 0:
        raise ValueError(f"oracle failed with status {rc} (Pade not converging?)")
    out = {"tll": tll, "cpl": cpl}
    if batch.compute_grids:
        out["tlg"] = tlg
        out["cpg"] = cpg
    return out


def pade(freq, c0, np_pade, ns=1, dr=50.0, ip=1):
    lib = load()
    a = np.zeros(np_pade, np.complex128)
    b = np.zeros(np_pade, np.complex128)
    rc = lib.ram_oracle_pade(float(freq), float(c0), int(np_pade), int(ns), float(dr), int(ip),
                             a.ctypes.data, b.ctypes.data)
    if rc:
        raise ValueError("Laguerre method not converging")
    return a, b
