"""The C ABI library: loads, exports every declared symbol, host-only entry points.

No compute call here touches a GPU: cr_pade is host code, and cr_create
rejects invalid batches before any CUDA call.
"""
import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

from cupyram_b200 import _lib, compute_pade_coefficients
from golden_cases import GOLDEN, load_case
from cupyram_b200 import batch as B

HEADERS = sorted((Path(__file__).resolve().parent.parent / "include").glob("*.h"))


def declared_symbols():
    syms = set()
    for h in HEADERS:
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*(?:[A-Za-z_][\w\s\*]*?)\b(cr_\w+)\s*\(", text, flags=re.M):
            syms.add(m.group(1))
    return syms


def test_headers_declare_entry_points():
    syms = declared_symbols()
    for s in ("cr_create", "cr_run", "cr_march", "cr_pade", "cr_destroy", "cr_last_error"):
        assert s in syms


def test_library_exports_every_declared_symbol(lib_built):
    lib = ctypes.CDLL(str(lib_built))
    missing = [s for s in sorted(declared_symbols()) if not hasattr(lib, s)]
    assert not missing, missing


def test_abi_version(lib_built):
    assert _lib.load().cr_abi_version() == _lib.ABI_VERSION


def test_struct_layouts_match_header(lib_built):
    # sizes implied by the header's field lists
    assert _lib.RAY_DTYPE.itemsize == 136
    assert _lib.ENV_DTYPE.itemsize == 32
    assert ctypes.sizeof(_lib.CrBatch) == 64
    assert ctypes.sizeof(_lib.CrOutputs) == 32


def test_pade_matches_reference(lib_built):
    d = np.load(GOLDEN / "pade_ref.npz")
    worst = 0.0
    for row, p1, p2 in zip(d["params"], d["pd1"], d["pd2"]):
        np_, ns, ip, freq, dr, c0 = row
        a, c = compute_pade_coefficients(freq, c0, int(np_), ns=int(ns), dr=dr, ip=int(ip))
        n = int(np_)
        worst = max(worst, np.max(np.abs(a - p1[:n])), np.max(np.abs(c - p2[:n])))
    assert worst < 1e-8, worst


def test_pade_batch_matches_single_calls(lib_built):
    """compute_pade_coefficients_batch (cupyram/pade.py:276-317): [np, batch]
    arrays whose column b is the single call at c0_array[b]."""
    from cupyram_b200 import compute_pade_coefficients, compute_pade_coefficients_batch
    c0 = np.array([1480.0, 1500.0, 1525.0, 1550.0])
    for npd, ns, ip in ((4, 1, 1), (6, 2, 1), (8, 1, 2)):
        pd1, pd2 = compute_pade_coefficients_batch(75.0, c0, npd, ns, 20.0, ip)
        assert pd1.shape == pd2.shape == (npd, c0.size) and pd1.dtype == np.complex128
        for b, c in enumerate(c0):
            q1, q2 = compute_pade_coefficients(75.0, c, npd, ns=ns, dr=20.0, ip=ip)
            assert np.array_equal(pd1[:, b], q1) and np.array_equal(pd2[:, b], q2)


def test_pade_bad_arguments(lib_built):
    with pytest.raises(ValueError):
        compute_pade_coefficients(50.0, 1500.0, 0)
    with pytest.raises(ValueError):
        compute_pade_coefficients(50.0, 1500.0, 11)
    with pytest.raises(ValueError):
        compute_pade_coefficients(-50.0, 1500.0, 4)


def _desc(b, **over):
    rays = np.ascontiguousarray(b.rays.copy())
    for k, v in over.items():
        rays[k] = v
    d = _lib.CrBatch()
    d.n_rays, d.n_envs = len(rays), len(b.envs)
    d.rays, d.envs, d.pool = rays.ctypes.data, b.envs.ctypes.data, b.pool.ctypes.data
    d.pool_len, d.precision, d.compute_grids = b.pool.size, 0, 1
    d.line_len, d.grid_len = b.line_len, b.grid_len
    return d, rays


@pytest.mark.parametrize("field,value", [("np", 0), ("np", 11), ("ns", 3), ("nz", 1), ("dz", 0.0),
                                         ("env", 5), ("ndr", 0), ("line_off", 10**9), ("zs", 1e9)])
def test_create_rejects_invalid_batch(lib_built, field, value):
    args, kw, _ = load_case("pekeris_small")
    envs, p, zs, zr, pr = B.prepare(*args, dict(kw))
    b = B.build_batch(envs, p, zs, zr, pr, True)
    d, keep = _desc(b, **{field: value})
    h = ctypes.c_void_p()
    rc = _lib.load().cr_create(ctypes.byref(d), ctypes.byref(h))
    assert rc == _lib.CR_EINVAL
    assert not h.value
    assert _lib.global_error()


def test_null_arguments(lib_built):
    lib = _lib.load()
    assert lib.cr_create(None, None) == _lib.CR_EINVAL
    assert lib.cr_upload(None) == _lib.CR_EINVAL
    assert lib.cr_march(None) == _lib.CR_EINVAL
    lib.cr_destroy(None)


def test_header_constants_match_the_binding():
    """The host binding's copies of the header's #defines and enums."""
    text = (Path(__file__).resolve().parent.parent / "include" / "cupyram_b200.h").read_text()
    defines = {k: v.replace("u", "") for k, v in re.findall(r"#define\s+(CR_\w+)\s+\(?([0-9][0-9u *]*)\)?", text)}
    assert int(defines["CR_ABI_VERSION"]) == _lib.ABI_VERSION
    assert int(defines["CR_MAX_NP"]) == _lib.MAX_NP
    assert int(np.prod([int(x) for x in defines["CR_STATIC_SCRATCH_BYTES"].split("*")])) == _lib.STATIC_SCRATCH_BYTES
    enums = {k: int(v) for k, v in re.findall(r"\b(CR_[A-Z0-9_]+)\s*=\s*(\d+)", text)}
    for name in ("CR_OK", "CR_EINVAL", "CR_ECUDA", "CR_EPADE", "CR_ETIMEOUT", "CR_ENAN", "CR_ENOMEM", "CR_ESTATE",
                 "CR_PLAIN_C128", "CR_CHOSEN_C64R", "CR_CHOSEN_C64"):
        assert enums[name] == getattr(_lib, name), name


def test_create_without_a_device_fails_cleanly(lib_built):
    """A valid batch on a machine without a usable GPU: cr_create returns
    CR_ECUDA with the runtime's message, the binding raises, and the process
    carries on (the library never aborts)."""
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is visible")
    from cupyram_b200.engine import Engine
    from cupyram_b200._lib import EngineError
    args, kw, _ = load_case("pekeris_small")
    envs, p, zs, zr, pr = B.prepare(*args, dict(kw))
    b = B.build_batch(envs, p, zs, zr, pr, False)
    with pytest.raises(EngineError, match=r"status 2\].*cr_create"):
        Engine(b)


def test_peak_fma_arguments_and_no_device(lib_built):
    """cr_peak_fma (include/cupyram_b200_peaks.h) rejects bad arguments before
    any CUDA call, and without a usable GPU returns its CUDA status."""
    lib = _lib.load()
    t, ms = ctypes.c_double(), ctypes.c_double()
    assert lib.cr_peak_fma(1, 0, ctypes.byref(t), ctypes.byref(ms)) == 1
    assert lib.cr_peak_fma(1, 16, None, ctypes.byref(ms)) == 1
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        assert lib.cr_peak_fma(1, 16, ctypes.byref(t), ctypes.byref(ms)) == 2
