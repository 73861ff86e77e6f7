#!/usr/bin/env python3
"""Generate golden fixtures by running the UNMODIFIED reference CuPyRAM on CPU.

The reference (clapeyre/cupyram) is pure Python: Numba ``@cuda.jit`` kernels
plus CuPy array glue.  This script runs it with Numba's CUDA simulator
(``NUMBA_ENABLE_CUDASIM=1``) and a NumPy-backed stand-in for ``cupy`` and
``nvtx`` (written here, into a temporary directory), then stores the outputs
as small ``.npz`` fixtures next to this file.  The fixtures travel with the
repository; the reference itself does not.

Usage (in a container that has the reference checked out)::

    python tests/golden/make_golden.py --ref /path/to/cupyram [case ...]

Cases are listed in ``CASES``; each is run in its own process so they can be
generated in parallel.  Padé coefficient fixtures (``pade_ref.npz``) come from
the reference's ``cupyram/pade.py`` imported directly (Numba CPU JIT).
"""
import argparse
import os
import subprocess
import sys
import tempfile
import textwrap
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent

# ---------------------------------------------------------------------------
# stand-in modules: NumPy behind the ``cupy`` name, a no-op ``nvtx``
# ---------------------------------------------------------------------------
_CUPY_SHIM = textwrap.dedent('''
    from numpy import *            # noqa: F401,F403  (zeros, asarray, sqrt, ...)
    import numpy as _np
    ndarray = _np.ndarray
    def asnumpy(x):
        return _np.asarray(x)
    class _Pool:
        def free_all_blocks(self):
            pass
        def used_bytes(self):
            return 0
        def total_bytes(self):
            return 0
    def get_default_memory_pool():
        return _Pool()
''')

_NVTX_SHIM = textwrap.dedent('''
    import contextlib, functools
    class annotate(contextlib.ContextDecorator):
        def __init__(self, *a, **k):
            pass
        def __enter__(self):
            return self
        def __exit__(self, *exc):
            return False
''')


def _install_shims():
    d = Path(tempfile.mkdtemp(prefix="refshim_"))
    (d / "cupy").mkdir()
    (d / "cupy" / "__init__.py").write_text(_CUPY_SHIM)
    (d / "nvtx").mkdir()
    (d / "nvtx" / "__init__.py").write_text(_NVTX_SHIM)
    return d


# ---------------------------------------------------------------------------
# cases: small enough for the simulator (it advances ~600 point-steps/s)
# ---------------------------------------------------------------------------
def _case_ram_v15():
    """The RAM v1.5 test case (range-dependent SSP, 200->400 m slope)."""
    return dict(
        freq=50.0, zs=50.0, zr=50.0,
        z_ss=np.array([0.0, 100.0, 400.0]),
        rp_ss=np.array([0.0, 25000.0]),
        cw=np.array([[1480.0, 1530.0], [1520.0, 1530.0], [1530.0, 1530.0]]),
        z_sb=np.array([0.0]), rp_sb=np.array([0.0]),
        cb=np.array([[1700.0]]), rhob=np.array([[1.5]]), attn=np.array([[0.5]]),
        rbzb=np.array([[0.0, 200.0], [40000.0, 400.0]]),
        kw=dict(rmax=50000.0, dr=500.0, dz=2.0, zmplt=500.0, c0=1600.0),
    )


def _case_pekeris_small():
    """Pekeris guide with a 4-point z_sb interface, np=4 (shortened range)."""
    return dict(
        freq=50.0, zs=100.0, zr=50.0,
        z_ss=np.array([0.0, 200.0]), rp_ss=np.array([0.0]),
        cw=np.array([[1500.0], [1500.0]]),
        z_sb=np.array([0.0, 200.0, 200.0, 300.0]), rp_sb=np.array([0.0]),
        cb=np.array([[1500.0], [1500.0], [1700.0], [1700.0]]),
        rhob=np.array([[1.0], [1.0], [1.5], [1.5]]),
        attn=np.array([[0.0], [0.0], [0.5], [0.5]]),
        rbzb=np.array([[0.0, 200.0], [2000.0, 200.0]]),
        kw=dict(rmax=2000.0, dr=50.0, dz=3.0, np=4, ns=1),
    )


def _case_ragged_batch():
    """3 rays with ragged rp_ss / rp_sb / rbzb lengths (NaN padding path)."""
    z_ss = [np.array([0.0, 100.0, 200.0])] * 3
    rp_ss = [np.array([0.0, 1000.0, 2000.0]),
             np.array([0.0, 500.0, 1200.0, 1800.0, 2500.0]),
             np.array([0.0, 700.0, 1600.0, 2400.0])]
    cw = [np.array([[1500.0, 1490.0, 1510.0], [1500.0, 1495.0, 1505.0], [1510.0, 1500.0, 1500.0]]),
          np.linspace(1480.0, 1520.0, 15).reshape(3, 5),
          np.linspace(1495.0, 1515.0, 12).reshape(3, 4)]
    z_sb = [np.array([0.0, 50.0])] * 3
    rp_sb = [np.array([0.0, 1000.0, 2000.0]),
             np.array([0.0, 500.0, 1200.0, 1800.0, 2500.0]),
             np.array([0.0, 700.0, 1600.0, 2400.0])]
    cb = [np.full((2, 3), 1600.0), np.linspace(1580.0, 1700.0, 10).reshape(2, 5),
          np.full((2, 4), 1650.0)]
    rhob = [np.full((2, 3), 1.5), np.full((2, 5), 1.7), np.linspace(1.3, 1.9, 8).reshape(2, 4)]
    attn = [np.full((2, 3), 0.5), np.full((2, 5), 0.3), np.full((2, 4), 0.8)]
    rbzb = [np.array([[0.0, 200.0], [3000.0, 200.0]]),
            np.array([[0.0, 180.0], [1500.0, 150.0], [3000.0, 190.0]]),
            np.array([[0.0, 160.0], [3000.0, 120.0]])]
    return dict(freq=50.0, zs=60.0, zr=40.0, z_ss=z_ss, rp_ss=rp_ss, cw=cw, z_sb=z_sb,
                rp_sb=rp_sb, cb=cb, rhob=rhob, attn=attn, rbzb=rbzb,
                kw=dict(rmax=3000.0, dr=50.0, dz=2.0, batch_size=3))


def _case_multifreq():
    """2 environments x 2 frequencies (N_calc = 4) sharing f1..f3."""
    z_ss = np.array([0.0, 100.0])
    env = dict(z_ss=[z_ss, z_ss], rp_ss=[np.array([0.0])] * 2,
               cw=[np.array([[1500.0], [1500.0]]), np.array([[1490.0], [1510.0]])],
               z_sb=[np.array([0.0, 10.0])] * 2, rp_sb=[np.array([0.0])] * 2,
               cb=[np.array([[1600.0], [1600.0]]), np.array([[1650.0], [1700.0]])],
               rhob=[np.array([[1.5], [1.5]]), np.array([[1.6], [1.8]])],
               attn=[np.array([[0.5], [0.5]]), np.array([[0.3], [0.6]])],
               rbzb=[np.array([[0.0, 100.0], [400.0, 100.0]]), np.array([[0.0, 90.0], [400.0, 95.0]])])
    return dict(freq=[80.0, 120.0], zs=10.0, zr=50.0, **env,
                kw=dict(rmax=400.0, dr=10.0, dz=1.0, batch_size=2))


def _case_wedge_switch():
    """Upslope wedge, np=6, ns=2, stability switch at rs, ndr=2, ndz=3."""
    r = np.linspace(0.0, 1000.0, 11)
    z = 60.0 - 30.0 * r / 1000.0
    return dict(
        freq=100.0, zs=10.0, zr=20.0,
        z_ss=np.array([0.0, 30.0, 60.0]), rp_ss=np.array([0.0]),
        cw=np.array([[1500.0], [1495.0], [1490.0]]),
        z_sb=np.array([0.0, 20.0]), rp_sb=np.array([0.0]),
        cb=np.array([[1650.0], [1750.0]]), rhob=np.array([[1.6], [1.9]]),
        attn=np.array([[0.4], [0.7]]),
        rbzb=np.column_stack([r, z]),
        kw=dict(rmax=1000.0, dr=20.0, dz=1.0, np=6, ns=2, rs=500.0, ndr=2, ndz=3, c0=1500.0),
    )


def _case_mini_munk():
    """Deep Munk column, 25 Hz, np=8, short range."""
    zz = np.linspace(0.0, 5000.0, 51)
    eta = 2.0 * (zz - 1300.0) / 1300.0
    c = 1500.0 * (1.0 + 0.00737 * (eta - 1.0 + np.exp(-eta)))
    return dict(
        freq=25.0, zs=1000.0, zr=1000.0,
        z_ss=zz, rp_ss=np.array([0.0]), cw=c.reshape(-1, 1),
        z_sb=np.array([0.0, 100.0]), rp_sb=np.array([0.0]),
        cb=np.array([[1600.0], [1600.0]]), rhob=np.array([[1.5], [1.5]]),
        attn=np.array([[0.5], [0.5]]),
        rbzb=np.array([[0.0, 5000.0], [2000.0, 5000.0]]),
        kw=dict(rmax=2000.0, dr=50.0, dz=6.0, np=8),
    )


CASES = {
    "ram_v15": _case_ram_v15,
    "pekeris_small": _case_pekeris_small,
    "ragged_batch": _case_ragged_batch,
    "multifreq": _case_multifreq,
    "wedge_switch": _case_wedge_switch,
    "mini_munk": _case_mini_munk,
}


def _pack_inputs(case):
    """Flatten a case into npz-storable arrays (lists become object-free stacks)."""
    out = {}
    for k, v in case.items():
        if k == "kw":
            for kk, vv in v.items():
                out["kw_" + kk] = np.asarray(vv)
        elif isinstance(v, list) and not np.isscalar(v[0]):
            out["in_" + k + "_n"] = np.asarray(len(v))
            for i, a in enumerate(v):
                out[f"in_{k}_{i}"] = np.asarray(a, dtype=np.float64)
        else:
            out["in_" + k] = np.asarray(v, dtype=np.float64)
    return out


def run_case(name, ref):
    shim = _install_shims()
    os.environ["NUMBA_ENABLE_CUDASIM"] = "1"
    sys.path.insert(0, str(shim))
    sys.path.insert(0, str(ref))
    from numba import cuda
    cuda.as_cuda_array = lambda x: x
    import cupyram.cupyram as cr_mod  # noqa: E402
    case = CASES[name]()
    kw = dict(case["kw"])
    def _copy(v):
        if isinstance(v, np.ndarray):
            return v.copy()
        if isinstance(v, list):
            return [np.array(a, copy=True) if isinstance(a, np.ndarray) else a for a in v]
        return v
    args = {k: _copy(v) for k, v in case.items() if k != "kw"}
    t0 = time.time()
    model = cr_mod.CuPyRAM(args.pop("freq"), args.pop("zs"), args.pop("zr"), args.pop("z_ss"),
                           args.pop("rp_ss"), args.pop("cw"), args.pop("z_sb"), args.pop("rp_sb"),
                           args.pop("cb"), args.pop("rhob"), args.pop("attn"), args.pop("rbzb"), **kw)
    res = model.run()
    wall = time.time() - t0
    out = _pack_inputs(case)
    out.update(
        tl_line=np.asarray(res["TL Line"]), tl_grid=np.asarray(res["TL Grid"]),
        cp_line=np.asarray(res["CP Line"]), ranges=np.asarray(res["Ranges"]),
        depths=np.asarray(res["Depths"]), nz=np.asarray(model.nz), dz=np.asarray(model._dz),
        dr=np.asarray(model._dr), zmax=np.asarray(model._zmax), c0=np.asarray(res["c0"]),
        sim_wall_s=np.asarray(wall),
    )
    np.savez_compressed(HERE / f"{name}.npz", **out)
    print(f"{name}: nz={model.nz} nvr={len(res['Ranges'])} wall={wall:.1f}s", flush=True)


def run_pade(ref):
    """Padé coefficients from the reference's pade.py for a grid of cases."""
    sys.path.insert(0, str(ref))
    import importlib.util
    spec = importlib.util.spec_from_file_location("ref_pade", str(Path(ref) / "cupyram" / "pade.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    rows, pd1s, pd2s = [], [], []
    for np_pade in (1, 2, 3, 4, 5, 6, 7, 8):
        for ns in (0, 1, 2):
            for ip in (1, 2):
                for freq in (25.0, 50.0, 100.0, 200.0, 500.0):
                    for dr in (2.0, 10.0, 25.0, 50.0, 100.0, 500.0):
                        for c0 in (1500.0, 1600.0):
                            if ns > np_pade:
                                continue
                            try:
                                p1, p2 = mod.compute_pade_coefficients(freq, c0, np_pade, ns=ns, dr=dr, ip=ip)
                            except (ValueError, ZeroDivisionError):
                                continue
                            if not (np.all(np.isfinite(p1)) and np.all(np.isfinite(p2))):
                                continue
                            a1 = np.zeros(8, complex); a2 = np.zeros(8, complex)
                            a1[:np_pade] = p1; a2[:np_pade] = p2
                            rows.append((np_pade, ns, ip, freq, dr, c0)); pd1s.append(a1); pd2s.append(a2)
    np.savez_compressed(HERE / "pade_ref.npz", params=np.array(rows, dtype=np.float64),
                        pd1=np.array(pd1s), pd2=np.array(pd2s))
    print(f"pade: {len(rows)} cases", flush=True)


def run_tlref(ref):
    """RAM v1.5's own Fortran TL line (the reference's tests/tl_ref.line)."""
    data = np.loadtxt(Path(ref) / "tests" / "tl_ref.line")
    np.savez_compressed(HERE / "ram_v15_fortran.npz", ranges=data[:, 0], tl=data[:, 1])
    print(f"tl_ref.line: {len(data)} ranges", flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True, help="path to the reference checkout")
    ap.add_argument("--one", help=argparse.SUPPRESS)
    ap.add_argument("cases", nargs="*")
    a = ap.parse_args()
    if a.one == "pade":
        run_pade(a.ref)
        return
    if a.one == "tlref":
        run_tlref(a.ref)
        return
    if a.one:
        run_case(a.one, a.ref)
        return
    names = a.cases or (["pade", "tlref"] + list(CASES))
    procs = [subprocess.Popen([sys.executable, __file__, "--ref", a.ref, "--one", n]) for n in names]
    rc = max(p.wait() for p in procs)
    sys.exit(rc)


if __name__ == "__main__":
    main()
