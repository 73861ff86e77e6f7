"""Engine vs the oracle over the Pade parameters the reference accepts: every
lane count of the batched march (np 1..10, two terms per lane, odd np leaving
a lane slot without a term) and every stability setting (ns 0, 1, 2, with the
stability constraints lifted at rs = 1 km), on both march kernels.

np 1 with ns 2 is left out: its two stability constraints replace both
accuracy conditions, the Pade system is singular and the reference's
compute_pade_coefficients (cupyram/pade.py:240-256) returns NaN, as
compute_pade_coefficients does here.

Bars as in test_gpu_parity: TL line 1e-3 dB, complex pressure 1e-6 relative.
"""
import numpy as np
import pytest

from golden_cases import load_case
from cupyram_b200 import batch as B
from cupyram_b200.engine import Engine
from oracle import oracle

pytestmark = pytest.mark.gpu

CASES = [(npd, ns) for npd in (1, 2, 3, 5, 7, 9, 10) for ns in (0, 1, 2) if not (npd == 1 and ns == 2)]


@pytest.mark.parametrize("march", ["batched", "column"])
@pytest.mark.parametrize("npd,ns", CASES)
def test_pade_parameters_vs_oracle(cuda_device, monkeypatch, march, npd, ns):
    monkeypatch.setenv("CUPYRAM_B200_COL", "0" if march == "batched" else "1")
    args, kw, _ = load_case("pekeris_small")
    envs, p, zs, zr, pr = B.prepare(*args, dict(kw, np=npd, ns=ns, rs=1000.0))
    b = B.build_batch(envs, p, zs, zr, pr, False)
    with Engine(b) as eng:
        out = eng.run()
        st = eng.stats()
    assert st["rays_failed"] == 0
    assert st["column_rays"] == (b.n_rays if march == "column" else 0)
    ref = oracle.run(b, "plain")
    n = b.line_len
    d = np.abs(out["tll"][:n] - ref["tll"][:n])
    assert d.max() < 1e-3, d.max()
    cp = np.abs(out["cpl"][:n] - ref["cpl"][:n]).max() / np.abs(ref["cpl"][:n]).max()
    assert cp < 1e-6, cp
