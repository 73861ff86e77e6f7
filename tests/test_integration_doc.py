"""The ctypes stub that INTEGRATION.md offers the reference's maintainers (CPU):
extracted from the document and run against the built library, its structs
must match the ABI and its error path must raise the library's message."""
import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

from cupyram_b200 import _lib

ROOT = Path(__file__).resolve().parent.parent


def _stub(lib_path):
    text = (ROOT / "INTEGRATION.md").read_text()
    code = re.search(r"```python\n(# cupyram/_b200\.py.*?)```", text, re.S).group(1)
    code = code.replace('ctypes.CDLL("libcupyram_b200.so")', f"ctypes.CDLL({str(lib_path)!r})")
    ns = {}
    exec(compile(code, "INTEGRATION.md", "exec"), ns)
    return ns


def test_stub_structs_match_the_abi(lib_built):
    ns = _stub(lib_built)
    assert ns["RAY"] == _lib.RAY_DTYPE and ns["ENV"] == _lib.ENV_DTYPE
    for mine, theirs in ((ns["Batch"], _lib.CrBatch), (ns["Outputs"], _lib.CrOutputs)):
        assert ctypes.sizeof(mine) == ctypes.sizeof(theirs)
        assert [(f[0], getattr(mine, f[0]).offset) for f in mine._fields_] == \
               [(f[0], getattr(theirs, f[0]).offset) for f in theirs._fields_]


def test_stub_raises_the_library_message(lib_built):
    ns = _stub(lib_built)
    rays = np.zeros(1, ns["RAY"])  # nz = 0: rejected by cr_create before any device work
    envs = np.zeros(1, ns["ENV"])
    with pytest.raises(ValueError, match="cr_create"):
        ns["march"](rays, envs, np.zeros(4), 1, 0, compute_grids=False)
