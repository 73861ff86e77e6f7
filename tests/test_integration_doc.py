"""The ctypes stub offered to the reference's maintainers (examples/ctypes_stub.py,
CPU): run against the built library, its structs must match the ABI and its
error path must raise the library's message."""
import ctypes
import importlib.util
from pathlib import Path

import numpy as np
import pytest

from cupyram_b200 import _lib

ROOT = Path(__file__).resolve().parent.parent


def _stub(lib_path):
    spec = importlib.util.spec_from_file_location("ctypes_stub", ROOT / "examples" / "ctypes_stub.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    mod.load(str(lib_path))
    return mod


def test_stub_structs_match_the_abi(lib_built):
    st = _stub(lib_built)
    assert st.RAY == _lib.RAY_DTYPE and st.ENV == _lib.ENV_DTYPE
    for mine, theirs in ((st.Batch, _lib.CrBatch), (st.Outputs, _lib.CrOutputs)):
        assert ctypes.sizeof(mine) == ctypes.sizeof(theirs)
        assert [(f[0], getattr(mine, f[0]).offset) for f in mine._fields_] == \
               [(f[0], getattr(theirs, f[0]).offset) for f in theirs._fields_]


def test_stub_raises_the_library_message(lib_built):
    st = _stub(lib_built)
    rays = np.zeros(1, st.RAY)  # nz = 0: rejected by cr_create before any device work
    envs = np.zeros(1, st.ENV)
    with pytest.raises(ValueError, match="cr_create"):
        st.march(rays, envs, np.zeros(4), 1, 0, compute_grids=False)
