"""ctypes binding of ``libcupyram_b200.so`` (the C ABI in include/cupyram_b200.h).

The library is built in-tree by ``python -m cupyram_b200.build``.  There is no
fallback: if the shared object is missing or was built for another ABI the
import of anything that needs it raises ``RuntimeError``.
"""
import ctypes
import os
from pathlib import Path

import numpy as np

LIB_NAME = "libcupyram_b200.so"
LIB_PATH = Path(__file__).resolve().parent / LIB_NAME

ABI_VERSION = 3
MAX_NP = 10

# status codes (enum cr_status)
CR_OK, CR_EINVAL, CR_ECUDA, CR_EPADE, CR_ETIMEOUT, CR_ENAN, CR_ENOMEM, CR_ESTATE = range(8)
# precision forms (enum cr_precision)
CR_PLAIN_C128, CR_CHOSEN_C64R, CR_CHOSEN_C64, CR_C64_REFINED = 0, 1, 2, 3

RAY_DTYPE = np.dtype(
    [("freq", "f8"), ("c0", "f8"), ("zs", "f8"), ("zr", "f8"), ("dz", "f8"), ("dr", "f8"),
     ("zmax", "f8"), ("lyrw_lambda", "f8"), ("attnf", "f8"), ("rs", "f8"),
     ("nz", "i4"), ("nr", "i4"), ("np", "i4"), ("ns", "i4"), ("ndr", "i4"), ("ndz", "i4"),
     ("nvr", "i4"), ("nvz", "i4"), ("env", "i4"), ("reserved", "i4"),
     ("line_off", "i8"), ("grid_off", "i8")], align=True)
ENV_DTYPE = np.dtype(
    [("n_zss", "i4"), ("n_rss", "i4"), ("n_zsb", "i4"), ("n_rsb", "i4"), ("n_bt", "i4"),
     ("reserved", "i4"), ("off", "i8")], align=True)
assert RAY_DTYPE.itemsize == 136 and ENV_DTYPE.itemsize == 32


class CrBatch(ctypes.Structure):
    _fields_ = [("n_rays", ctypes.c_int32), ("n_envs", ctypes.c_int32),
                ("rays", ctypes.c_void_p), ("envs", ctypes.c_void_p), ("pool", ctypes.c_void_p),
                ("pool_len", ctypes.c_int64), ("precision", ctypes.c_int32),
                ("compute_grids", ctypes.c_int32), ("line_len", ctypes.c_int64),
                ("grid_len", ctypes.c_int64)]


class CrOutputs(ctypes.Structure):
    _fields_ = [("tll", ctypes.c_void_p), ("cpl", ctypes.c_void_p),
                ("tlg", ctypes.c_void_p), ("cpg", ctypes.c_void_p)]


class CrStats(ctypes.Structure):
    _fields_ = [("march_ms", ctypes.c_double), ("assemble_ms", ctypes.c_double),
                ("h2d_ms", ctypes.c_double), ("d2h_ms", ctypes.c_double),
                ("point_updates", ctypes.c_double), ("h2d_bytes", ctypes.c_int64),
                ("d2h_bytes", ctypes.c_int64), ("kernel_launches", ctypes.c_int32),
                ("rays_failed", ctypes.c_int32), ("tile_rays", ctypes.c_int32),
                ("n_tiles", ctypes.c_int32), ("device_bytes", ctypes.c_int64),
                ("column_rays", ctypes.c_int32), ("column_launches", ctypes.c_int32),
                ("queue_ctas", ctypes.c_int32), ("precision_used", ctypes.c_int32),
                ("create_ms", ctypes.c_double), ("pade_ms", ctypes.c_double),
                ("tuner_row_step_s", ctypes.c_double), ("tuner_updates_per_s", ctypes.c_double),
                ("tuner_slots", ctypes.c_double)]


# every symbol the header declares, with its signature
_SIGS = {
    "cr_abi_version": (ctypes.c_int, []),
    "cr_pade": (ctypes.c_int, [ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_int,
                               ctypes.c_double, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]),
    "cr_pade_batch": (ctypes.c_int, [ctypes.c_int] + [ctypes.c_void_p] * 9),
    "cr_create": (ctypes.c_int, [ctypes.POINTER(CrBatch), ctypes.POINTER(ctypes.c_void_p)]),
    "cr_upload": (ctypes.c_int, [ctypes.c_void_p]),
    "cr_march": (ctypes.c_int, [ctypes.c_void_p]),
    "cr_download": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(CrOutputs)]),
    "cr_run": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(CrOutputs)]),
    "cr_set_pade": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                   ctypes.c_void_p, ctypes.c_void_p]),
    "cr_ray_flags": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]),
    "cr_get_stats": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(CrStats)]),
    "cr_last_error": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_size_t]),
    "cr_global_error": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_size_t]),
    "cr_peak_fma": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                                   ctypes.POINTER(ctypes.c_double)]),
    "cr_destroy": (None, [ctypes.c_void_p]),
    "cr_release_cache": (ctypes.c_int, []),
    "cr_plan_columns": (ctypes.c_int, [ctypes.POINTER(CrBatch), ctypes.c_double, ctypes.c_double,
                                       ctypes.c_double, ctypes.c_void_p]),
    "cr_march_static": (ctypes.c_int, [ctypes.POINTER(CrBatch), ctypes.POINTER(CrOutputs), ctypes.c_void_p]),
    "cr_cell_tl": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                  ctypes.c_void_p]),
}

STATIC_SCRATCH_BYTES = 32 * 1024 * 1024  # CR_STATIC_SCRATCH_BYTES

_lib = None


def load():
    """Load the native library (once).  Raises RuntimeError when it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    path = os.environ.get("CUPYRAM_B200_LIB", str(LIB_PATH))
    if not Path(path).exists():
        raise RuntimeError(
            f"cupyram_b200 native library not found at {path}; build it with "
            "`python -m cupyram_b200.build` (needs nvcc)")
    lib = ctypes.CDLL(path)
    for name, (res, args) in _SIGS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if lib.cr_abi_version() != ABI_VERSION:
        raise RuntimeError(f"{path} has ABI {lib.cr_abi_version()}, expected {ABI_VERSION}")
    _lib = lib
    return lib


def global_error():
    buf = ctypes.create_string_buffer(1024)
    load().cr_global_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def engine_error(handle):
    buf = ctypes.create_string_buffer(1024)
    load().cr_last_error(handle, buf, len(buf))
    return buf.value.decode(errors="replace")


class EngineError(RuntimeError):
    """A native call returned a non-zero status."""

    def __init__(self, code, msg):
        super().__init__(f"[status {code}] {msg}")
        self.code = code


def check(code, handle=None):
    if code == CR_OK:
        return
    msg = engine_error(handle) if handle else global_error()
    if code in (CR_EINVAL, CR_EPADE):
        raise ValueError(msg)
    raise EngineError(code, msg)
