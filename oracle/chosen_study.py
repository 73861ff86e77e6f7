"""Size of the chosen form's error, and of an FP32 inner loop's, on the CPU
(TEST INFRASTRUCTURE: runs the oracle's chosen-form models, not the engine).

    python oracle/chosen_study.py [n_munk_rays] [n_wedge_rays]

For full-range rays of the 4096-ray Munk batch and a sample of the wedge
batch (seed 2024), it prints the TL line error against the FP64 sum form
over cells with TL < 100 dB, per model:

* chosen      - the engine's chosen form (complex64 sweeps, FP64 combination);
* chosen_c32  - the same with the terms combined in FP32;
* chosen_f32  - also the elimination's coupling formed in FP32.
"""
import sys
import time
from pathlib import Path

import numpy as np

# run as a script, this folder would shadow the oracle package with its oracle.py
HERE = Path(__file__).resolve().parent
sys.path[:] = [p for p in sys.path if Path(p or ".").resolve() != HERE]
sys.path.insert(0, str(HERE.parent))
from oracle import oracle as O  # noqa: E402
from cupyram_b200 import workloads as W  # noqa: E402

MODELS = ("chosen", "chosen_c32", "chosen_f32")


def lines(batch, mode, rays):
    out = O.run(batch, mode, rays=rays)
    r = batch.rays[np.asarray(rays)]
    return [out["tll"][int(x["line_off"]): int(x["line_off"]) + int(x["nvr"])] for x in r]


def errors(ref, other):
    """Mean over rays of the RMS, and the max, of TL differences where the reference is below 100 dB."""
    rms, mx = [], []
    for a, b in zip(ref, other):
        d = (b - a)[a < 100.0]
        rms.append(np.sqrt(np.mean(d * d)))
        mx.append(np.abs(d).max())
    return float(np.mean(rms)), float(np.max(mx))


def study(name, batch, rays):
    t = time.time()
    ref = lines(batch, "sum", rays)
    print(f"{name}: {len(rays)} rays, {batch.rays['nz'][rays].astype(float) @ batch.rays['nr'][rays]:.2e} updates")
    for m in MODELS:
        rms, mx = errors(ref, lines(batch, m, rays))
        print(f"  {m:11s} RMS {rms:.4f} dB  max {mx:.3f} dB")
    print(f"  ({time.time() - t:.1f} s)")


def main():
    n_munk = int(sys.argv[1]) if len(sys.argv) > 1 else 8
    n_wedge = int(sys.argv[2]) if len(sys.argv) > 2 else 24
    munk = W.build(*W.munk_batch(4096, seed=2024), compute_grids=False)
    study("Munk, full range", munk, list(range(0, 4096, 4096 // n_munk))[:n_munk])
    wedge = W.build(*W.wedge_batch(10000, seed=2024), compute_grids=False)
    work = wedge.rays["nz"].astype(float) * wedge.rays["nr"]
    order = np.argsort(work)  # a sample of the lower 80 % of the work (CPU time)
    rays = [int(order[i]) for i in np.linspace(0, 7999, n_wedge).astype(int)]
    rays = [i for i in rays if np.floor(wedge.rays["zs"][i] / wedge.rays["dz"][i]) >= 1]
    study("wedge, sample", wedge, rays)


if __name__ == "__main__":
    main()
