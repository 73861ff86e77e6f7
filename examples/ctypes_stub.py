"""The module a maintainer of clapeyre/cupyram would add to bind the B200 engine.

Saved in the reference's package as ``cupyram/_b200.py``, it lets
``cupyram.CuPyRAM.run()`` keep its own set-up and hand the whole range march
(cupyram/cupyram.py:296-317 and the launchers it calls) to the C ABI of
``include/cupyram_b200.h``.  It mirrors the package's own binding,
``cupyram_b200/_lib.py``, with only what ``run()`` needs: the record layouts
of ``struct cr_ray`` / ``struct cr_env``, the ``cr_batch`` / ``cr_outputs``
structs, and one ``march()`` call that creates an engine, runs it and frees it.
Errors come back as the library's own messages: ``ValueError`` for a bad
batch or a Pade set that does not converge (as the reference raises at
cupyram/cupyram.py:413-434 and cupyram/pade.py:146-147), ``RuntimeError``
for device failures.
"""
import ctypes
import os

import numpy as np

RAY = np.dtype([("freq", "f8"), ("c0", "f8"), ("zs", "f8"), ("zr", "f8"), ("dz", "f8"), ("dr", "f8"),
                ("zmax", "f8"), ("lyrw_lambda", "f8"), ("attnf", "f8"), ("rs", "f8"),
                ("nz", "i4"), ("nr", "i4"), ("np", "i4"), ("ns", "i4"), ("ndr", "i4"), ("ndz", "i4"),
                ("nvr", "i4"), ("nvz", "i4"), ("env", "i4"), ("reserved", "i4"),
                ("line_off", "i8"), ("grid_off", "i8")], align=True)    # struct cr_ray
ENV = np.dtype([("n_zss", "i4"), ("n_rss", "i4"), ("n_zsb", "i4"), ("n_rsb", "i4"), ("n_bt", "i4"),
                ("reserved", "i4"), ("off", "i8")], align=True)       # struct cr_env


class Batch(ctypes.Structure):                                      # struct cr_batch
    _fields_ = [("n_rays", ctypes.c_int32), ("n_envs", ctypes.c_int32),
                ("rays", ctypes.c_void_p), ("envs", ctypes.c_void_p), ("pool", ctypes.c_void_p),
                ("pool_len", ctypes.c_int64), ("precision", ctypes.c_int32),
                ("compute_grids", ctypes.c_int32), ("line_len", ctypes.c_int64),
                ("grid_len", ctypes.c_int64)]


class Outputs(ctypes.Structure):                                    # struct cr_outputs
    _fields_ = [("tll", ctypes.c_void_p), ("cpl", ctypes.c_void_p),
                ("tlg", ctypes.c_void_p), ("cpg", ctypes.c_void_p)]


lib = None


def load(path=None):
    """Open the shared library (default: $CUPYRAM_B200_LIB, else the loader's search path)."""
    global lib
    lib = ctypes.CDLL(path or os.environ.get("CUPYRAM_B200_LIB", "libcupyram_b200.so"))
    lib.cr_create.argtypes = [ctypes.POINTER(Batch), ctypes.POINTER(ctypes.c_void_p)]
    lib.cr_run.argtypes = [ctypes.c_void_p, ctypes.POINTER(Outputs)]
    lib.cr_last_error.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_size_t]
    lib.cr_global_error.argtypes = [ctypes.c_char_p, ctypes.c_size_t]
    lib.cr_destroy.argtypes = [ctypes.c_void_p]
    return lib


def march(rays, envs, pool, line_len, grid_len, compute_grids=True):
    """rays: RAY records (one per (env, freq) calculation); envs/pool: profiles."""
    if lib is None:
        load()
    b = Batch(len(rays), len(envs), rays.ctypes.data, envs.ctypes.data, pool.ctypes.data,
              pool.size, 0, int(compute_grids), line_len, grid_len)
    h = ctypes.c_void_p()
    if lib.cr_create(ctypes.byref(b), ctypes.byref(h)):
        msg = ctypes.create_string_buffer(512)
        lib.cr_global_error(msg, 512)
        raise ValueError(msg.value.decode())
    out = dict(tll=np.empty(line_len), cpl=np.empty(line_len, complex),
               tlg=np.empty(grid_len) if compute_grids else None,
               cpg=np.empty(grid_len, complex) if compute_grids else None)
    o = Outputs(*(a.ctypes.data if a is not None else None for a in out.values()))
    try:
        rc = lib.cr_run(h, ctypes.byref(o))
        if rc:
            msg = ctypes.create_string_buffer(512)
            lib.cr_last_error(h, msg, 512)
            raise (ValueError if rc in (1, 3) else RuntimeError)(msg.value.decode())
    finally:
        lib.cr_destroy(h)
    return out
