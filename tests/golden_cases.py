"""Load the golden fixtures of tests/golden/ back into CuPyRAM arguments."""
from pathlib import Path

import numpy as np

GOLDEN = Path(__file__).resolve().parent / "golden"
CASES = ["ram_v15", "pekeris_small", "ragged_batch", "multifreq", "wedge_switch", "mini_munk"]
ARG_ORDER = ["freq", "zs", "zr", "z_ss", "rp_ss", "cw", "z_sb", "rp_sb", "cb", "rhob", "attn", "rbzb"]
INT_KW = {"np", "ns", "ndr", "ndz", "batch_size", "id"}


def load_case(name):
    """(args, kwargs, fixture) with args in CuPyRAM's positional order."""
    d = dict(np.load(GOLDEN / f"{name}.npz"))
    args = []
    for a in ARG_ORDER:
        if f"in_{a}_n" in d:
            n = int(d[f"in_{a}_n"])
            args.append([d[f"in_{a}_{i}"] for i in range(n)])
        else:
            v = d[f"in_{a}"]
            args.append(float(v) if v.ndim == 0 else (list(v) if a == "freq" else v))
    kw = {}
    for k, v in d.items():
        if k.startswith("kw_"):
            key = k[3:]
            kw[key] = int(v) if key in INT_KW else float(v)
    return args, kw, d
