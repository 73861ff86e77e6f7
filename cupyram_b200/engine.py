"""Python handle on one native engine (cr_engine) and its host buffers."""
import ctypes

import numpy as np

from . import _lib
from .batch import Batch


# precision forms of the march (enum cr_precision): "plain" complex128;
# "chosen" complex64 sweeps with the terms combined in FP64; "fast" complex64
# sweeps with an FP32 inner loop (couplings, M u and the combination in FP32);
# "refined" the chosen form plus one FP64-residual refinement step per term
# and range step
PRECISIONS = {"plain": _lib.CR_PLAIN_C128, "chosen": _lib.CR_CHOSEN_C64R, "fast": _lib.CR_CHOSEN_C64,
              "refined": _lib.CR_C64_REFINED}


class Engine:
    """Owns a cr_engine built from a packed :class:`Batch`.

    ``run()`` is the full device march with host outputs.  ``upload`` /
    ``march`` / ``download`` expose the three phases separately (the bench
    times ``march`` alone with inputs resident, and ``run`` end to end).
    Output buffers may be supplied by the caller (e.g. pinned memory); they
    must be C-contiguous float64 (tll, tlg) and complex128 (cpl, cpg).
    """

    def __init__(self, batch: Batch, precision="plain"):
        self.lib = _lib.load()
        self.batch = batch
        prec = PRECISIONS.get(precision)
        if prec is None:
            raise ValueError(f"precision must be one of {sorted(PRECISIONS)}, got {precision!r}")
        self._keep = (np.ascontiguousarray(batch.rays), np.ascontiguousarray(batch.envs),
                      np.ascontiguousarray(batch.pool, dtype=np.float64))
        rays, envs, pool = self._keep
        desc = _lib.CrBatch()
        desc.n_rays = len(rays)
        desc.n_envs = len(envs)
        desc.rays = rays.ctypes.data
        desc.envs = envs.ctypes.data
        desc.pool = pool.ctypes.data
        desc.pool_len = pool.size
        desc.precision = prec
        desc.compute_grids = 1 if batch.compute_grids else 0
        desc.line_len = batch.line_len
        desc.grid_len = batch.grid_len
        handle = ctypes.c_void_p()
        _lib.check(self.lib.cr_create(ctypes.byref(desc), ctypes.byref(handle)))
        self.handle = handle

    # -- phases -------------------------------------------------------------
    def upload(self):
        _lib.check(self.lib.cr_upload(self.handle), self.handle)

    def march(self):
        _lib.check(self.lib.cr_march(self.handle), self.handle)

    def alloc_outputs(self):
        b = self.batch
        out = {"tll": np.empty(max(b.line_len, 1), np.float64),
               "cpl": np.empty(max(b.line_len, 1), np.complex128)}
        if b.compute_grids:
            out["tlg"] = np.empty(max(b.grid_len, 1), np.float64)
            out["cpg"] = np.empty(max(b.grid_len, 1), np.complex128)
        return out

    def _outputs_struct(self, out):
        o = _lib.CrOutputs()
        for name, dt in (("tll", np.float64), ("cpl", np.complex128), ("tlg", np.float64),
                         ("cpg", np.complex128)):
            a = out.get(name)
            if a is None:
                setattr(o, name, None)
                continue
            if isinstance(a, np.ndarray):
                if a.dtype != dt or not a.flags.c_contiguous:
                    raise ValueError(f"{name} must be C-contiguous {np.dtype(dt).name}")
                setattr(o, name, a.ctypes.data)
            else:  # an object exposing a raw pointer (e.g. a pinned torch tensor)
                setattr(o, name, int(a.data_ptr()))
        return o

    def download(self, out):
        o = self._outputs_struct(out)
        _lib.check(self.lib.cr_download(self.handle, ctypes.byref(o)), self.handle)
        return out

    def run(self, out=None):
        out = out if out is not None else self.alloc_outputs()
        o = self._outputs_struct(out)
        _lib.check(self.lib.cr_run(self.handle, ctypes.byref(o)), self.handle)
        return out

    def cell_tl(self, sz, sr, ncz, ncr):
        """[n_rays, ncz, ncr] float32 cell-averaged TL of the last march (cr_cell_tl)."""
        out = np.empty((self.batch.n_rays, ncz, ncr), np.float32)
        _lib.check(self.lib.cr_cell_tl(self.handle, sz, sr, ncz, ncr, out.ctypes.data), self.handle)
        return out

    def set_pade(self, ray, which, pd1, pd2):
        p1 = np.ascontiguousarray(pd1, dtype=np.complex128)
        p2 = np.ascontiguousarray(pd2, dtype=np.complex128)
        _lib.check(self.lib.cr_set_pade(self.handle, ray, which, p1.size, p1.ctypes.data,
                                        p2.ctypes.data), self.handle)

    def ray_flags(self):
        f = np.zeros(self.batch.n_rays, np.int32)
        _lib.check(self.lib.cr_ray_flags(self.handle, f.ctypes.data, f.size), self.handle)
        return f

    def stats(self):
        st = _lib.CrStats()
        _lib.check(self.lib.cr_get_stats(self.handle, ctypes.byref(st)), self.handle)
        return {k: getattr(st, k) for k, _ in st._fields_}

    def close(self):
        if getattr(self, "handle", None):
            self.lib.cr_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def plan_columns(batch: Batch, row_step_s, updates_per_s, slots=0):
    """The column policy's cost rule for given costs (cr_plan_columns, host only):
    a bool array, True for the rays whose lockstep march in a batched tile
    would outlast the whole batch's balanced time by the policy's margin."""
    lib = _lib.load()
    rays = np.ascontiguousarray(batch.rays)
    envs = np.ascontiguousarray(batch.envs)
    pool = np.ascontiguousarray(batch.pool, dtype=np.float64)
    desc = _lib.CrBatch()
    desc.n_rays, desc.n_envs = len(rays), len(envs)
    desc.rays, desc.envs, desc.pool = rays.ctypes.data, envs.ctypes.data, pool.ctypes.data
    desc.pool_len = pool.size
    desc.precision = _lib.CR_PLAIN_C128
    desc.compute_grids = 1 if batch.compute_grids else 0
    desc.line_len, desc.grid_len = batch.line_len, batch.grid_len
    out = np.zeros(len(rays), np.int32)
    _lib.check(lib.cr_plan_columns(ctypes.byref(desc), float(row_step_s), float(updates_per_s), float(slots),
                                   out.ctypes.data))
    return out.astype(bool)


def march_static(batch: Batch, dev_out, stream=0):
    """Run ``cr_march_static``: a whole march that allocates nothing.

    For callers that must not allocate device memory when they march (see the
    cr_march_static comment in include/cupyram_b200.h).  ``dev_out`` maps
    "tll", "cpl" (and "tlg", "cpg" when the batch computes grids) to device
    buffers the caller owns - objects with ``data_ptr()`` (e.g. CUDA torch
    tensors) or raw integer device addresses - laid out like
    :meth:`Engine.download`'s outputs.  ``stream`` is a raw cudaStream_t
    handle (0: the default stream).  The scratch holds
    ``CR_STATIC_SCRATCH_BYTES``; larger batches raise ``ValueError``.
    """
    lib = _lib.load()
    rays = np.ascontiguousarray(batch.rays)
    envs = np.ascontiguousarray(batch.envs)
    pool = np.ascontiguousarray(batch.pool, dtype=np.float64)
    desc = _lib.CrBatch()
    desc.n_rays, desc.n_envs = len(rays), len(envs)
    desc.rays, desc.envs, desc.pool = rays.ctypes.data, envs.ctypes.data, pool.ctypes.data
    desc.pool_len = pool.size
    desc.precision = _lib.CR_PLAIN_C128
    desc.compute_grids = 1 if batch.compute_grids else 0
    desc.line_len, desc.grid_len = batch.line_len, batch.grid_len

    need = {"tll": batch.line_len, "cpl": batch.line_len}
    if batch.compute_grids:
        need.update(tlg=batch.grid_len, cpg=batch.grid_len)
    kinds = {"tll": "float64", "tlg": "float64", "cpl": "complex128", "cpg": "complex128"}

    def ptr(name):
        a = dev_out.get(name)
        if a is None:
            if name in need:
                raise ValueError(f"march_static: dev_out[{name!r}] is required")
            return None
        if isinstance(a, int):
            return a  # a raw device address: the caller vouches for its size and type
        # a tensor-like buffer: the kernel writes need[name] elements of the given type into it
        dt = str(getattr(a, "dtype", "")).replace("torch.", "")
        if dt != kinds[name]:
            raise ValueError(f"march_static: dev_out[{name!r}] must be {kinds[name]}, got {dt or type(a).__name__}")
        if not getattr(a, "is_cuda", False):
            raise ValueError(f"march_static: dev_out[{name!r}] must be in device memory")
        if hasattr(a, "is_contiguous") and not a.is_contiguous():
            raise ValueError(f"march_static: dev_out[{name!r}] must be contiguous")
        n = int(a.numel()) if hasattr(a, "numel") else int(a.size)
        if name in need and n < need[name]:
            raise ValueError(f"march_static: dev_out[{name!r}] holds {n} elements, the batch writes {need[name]}")
        return int(a.data_ptr())

    o = _lib.CrOutputs(ptr("tll"), ptr("cpl"), ptr("tlg"), ptr("cpg"))
    _lib.check(lib.cr_march_static(ctypes.byref(desc), ctypes.byref(o), ctypes.c_void_p(stream or None)))
