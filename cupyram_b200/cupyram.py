"""``CuPyRAM``: drop-in replacement for clapeyre/cupyram's ``CuPyRAM`` class.

Same constructor (``freq, zs, zr, z_ss, rp_ss, cw, z_sb, rp_sb, cb, rhob, attn,
rbzb, **kwargs``), same keyword arguments, same ``run()`` result dictionary and
the same squeeze rules (``cupyram/cupyram.py:176-380`` of the reference).  The
range march itself runs in the native sm_100a engine (``libcupyram_b200.so``);
this class only normalises, validates and reshapes on the host.

Extra keyword arguments (not in the reference):

``precision``  ``"plain"`` (complex128, default), ``"chosen"`` (complex64
               sweeps in FP32 arithmetic; the Pade terms are combined in FP64
               and the field is kept in complex128) or ``"fast"`` (complex64
               sweeps with an FP32 inner loop: couplings, M u and the term
               combination in FP32 too).
``per_ray``    ``True`` pairs environment i with frequency i (no
               environment x frequency cross product) and gives every ray its
               own grid; ``zs``, ``zr``, ``dr``, ``dz``, ``np``, ``rmax`` may
               then be per-ray arrays.  Ragged outputs come back as lists.

Deliberate differences from the reference, all fixes of its defects:

* the TL line is computed even when ``compute_grids=False`` (the reference
  leaves it at zero, ``cupyram.py:306-307``);
* ``CP Grid`` is filled (the reference allocates it but never writes it,
  ``outpt.py:49-53``) and squeezed like ``TL Grid``
  (the reference mis-squeezes it, ``cupyram.py:361,368``);
* range-dependence is decided per ray, not from ray 0 (``cupyram.py:437-442``);
* ``Proc Time`` is wall-clock seconds of ``run()``; ``Propagation Time`` is the
  device time of the march alone.
"""
import time

import numpy as np

from . import batch as _batch
from .engine import PRECISIONS, Engine


class CuPyRAM:

    _np_default = 8
    _dzf = 0.1
    _ndr_default = 1
    _ndz_default = 1
    _ns_default = 1
    _lyrw_default = 20
    _id_default = 0

    def __init__(self, freq, zs, zr, z_ss, rp_ss, cw, z_sb, rp_sb, cb, rhob, attn, rbzb, **kwargs):
        self._batch_size = int(kwargs.get("batch_size", 1))
        self._compute_grids = bool(kwargs.get("compute_grids", True))
        self._max_workers = kwargs.get("max_workers", 8)
        self._precision = kwargs.get("precision", "plain")
        if self._precision not in PRECISIONS:
            raise ValueError(f"precision must be one of {sorted(PRECISIONS)}, got {self._precision!r}")
        self._benchmark_propagation = bool(kwargs.get("benchmark_propagation", False))
        envs, p, zs_env, zr_env, per_ray = _batch.prepare(
            freq, zs, zr, z_ss, rp_ss, cw, z_sb, rp_sb, cb, rhob, attn, rbzb, kwargs)
        self._envs, self._p, self._zs_env, self._zr_env = envs, p, zs_env, zr_env
        self._per_ray = per_ray
        self._freqs = p.freqs
        self._n_env = self._batch_size
        self._n_freq = 1 if per_ray else len(p.freqs)
        self._total_batch = self._n_env * self._n_freq
        self._zs, self._zr = zs, zr
        # reference-visible scalars (shared grid) or per-ray arrays
        self._np = int(p.np_pade[0]) if not per_ray else p.np_pade
        self._c0 = p.c0_report
        self._c0_array = p.c0_env
        self._lambda = p.lam[0] if not per_ray else p.lam
        self._dr = float(p.dr[0]) if not per_ray else p.dr
        self._dz = float(p.dz[0]) if not per_ray else p.dz
        self._ndr, self._ndz = p.ndr, p.ndz
        self._zmplt = float(p.zmplt[0]) if not per_ray else p.zmplt
        self._rmax = float(p.rmax[0]) if not per_ray else p.rmax
        self._ns = p.ns
        self._rs = float(p.rs[0]) if not per_ray else p.rs
        self._lyrw = p.lyrw
        self._id = p.ident
        self.proc_time = None
        self.propagation_time = 0.0 if self._benchmark_propagation else None
        self.engine_stats = None

    # ------------------------------------------------------------------
    def setup(self):
        """Grid and packed batch (nz, nzplt, vr, vz, zmax) - cupyram.py:528-726."""
        b = _batch.build_batch(self._envs, self._p, self._zs_env, self._zr_env, self._per_ray,
                               self._compute_grids)
        self._batch_desc = b
        if self._per_ray:
            self.nz = b.nz
            self._zmax = b.zmax
            self.vr, self.vz = b.vr, b.vz
            self._rmax = b.nvr * self._p.dr * self._p.ndr
        else:
            self.nz = int(b.nz[0])
            self._zmax = float(b.zmax[0])
            self.vr, self.vz = b.vr[0], b.vz[0]
            self._rmax = float(b.nvr[0] * self._p.dr[0] * self._p.ndr)
            self.nzplt = int(np.floor(self._zmplt / self._dz))
        return b

    def run(self):
        t0 = time.perf_counter()
        b = self.setup()
        with Engine(b, precision=self._precision) as eng:
            out = eng.run()
            self.engine_stats = eng.stats()
        self.proc_time = time.perf_counter() - t0
        if self._benchmark_propagation:
            self.propagation_time += self.engine_stats["march_ms"] * 1e-3
        return self._results(b, out)

    # ------------------------------------------------------------------
    def _results(self, b, out):
        n_calc = b.n_rays
        tll = out["tll"]
        cpl = out["cpl"]
        tlg = out.get("tlg")
        cpg = out.get("cpg")
        rays = b.rays
        uniform = len(set(zip(rays["nvr"].tolist(), rays["nvz"].tolist()))) == 1
        if uniform:
            nvr = int(rays["nvr"][0])
            nvz = int(rays["nvz"][0])
            self.tll = tll[:n_calc * nvr].reshape(n_calc, nvr)
            self.cpl = cpl[:n_calc * nvr].reshape(n_calc, nvr)
            if b.compute_grids:
                self.tlg = tlg[:n_calc * nvz * nvr].reshape(n_calc, nvz, nvr)
                self.cpg = cpg[:n_calc * nvz * nvr].reshape(n_calc, nvz, nvr)
            else:
                self.tlg = self.cpg = None
            self.tll = self.tll.reshape(self._n_env, self._n_freq, nvr)
            self.cpl = self.cpl.reshape(self._n_env, self._n_freq, nvr)
            if b.compute_grids:
                self.tlg = self.tlg.reshape(self._n_env, self._n_freq, nvz, nvr)
                self.cpg = self.cpg.reshape(self._n_env, self._n_freq, nvz, nvr)
            # PyRAM-compatible squeezing (cupyram.py:348-368)
            if self._n_freq == 1 and self._n_env == 1:
                sl = (0, 0)
            elif self._n_freq == 1:
                sl = (slice(None), 0)
            elif self._n_env == 1:
                sl = (0, slice(None))
            else:
                sl = (slice(None), slice(None))
            self.tll, self.cpl = self.tll[sl], self.cpl[sl]
            if b.compute_grids:
                self.tlg, self.cpg = self.tlg[sl], self.cpg[sl]
        else:
            # per-ray grids of different sizes: lists of per-ray arrays
            self.tll, self.cpl, self.tlg, self.cpg = [], [], [], []
            for r in rays:
                lo, n = int(r["line_off"]), int(r["nvr"])
                self.tll.append(tll[lo:lo + n])
                self.cpl.append(cpl[lo:lo + n])
                if b.compute_grids:
                    go, nz_ = int(r["grid_off"]), int(r["nvz"])
                    self.tlg.append(tlg[go:go + nz_ * n].reshape(nz_, n))
                    self.cpg.append(cpg[go:go + nz_ * n].reshape(nz_, n))
            if not b.compute_grids:
                self.tlg = self.cpg = None
        res = {"ID": self._id, "Proc Time": self.proc_time, "Ranges": self.vr, "Depths": self.vz,
               "TL Grid": self.tlg, "TL Line": self.tll, "CP Grid": self.cpg, "CP Line": self.cpl,
               "c0": self._c0}
        st = self.engine_stats or {}
        res["Propagation Time"] = st.get("march_ms", 0.0) * 1e-3
        res["Point Updates"] = b.point_updates
        return res
