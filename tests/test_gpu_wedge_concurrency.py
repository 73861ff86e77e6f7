"""Batched tiles marching beside column clusters: outputs are deterministic and the forms agree.

With column groups present the batched tiles go in one launch per lanes-per-ray
value, on their own streams, while the column clusters run on theirs.  Every
tile still marches alone in its warp, so:

* two plain marches of the same batch give bit-identical outputs (a stale row
  read by a bulk copy, or any other ordering fault, shows up as a mismatch);
* the refined form matches plain to rounding on every ray (its batched rays
  run the complex64 sweeps plus the FP64-residual step, its column rays the
  complex128 column kernel), so a fault in either form's batched march shows;
* the chosen form stays within its bar (RMS <= 0.1 dB, max <= 1 dB over cells
  with TL < 100 dB) on every ray.

The batch is 2000 rays of the benchmark's uneven wedge generator, at full range.
"""
import numpy as np
import pytest

from cupyram_b200 import workloads
from cupyram_b200.engine import Engine

pytestmark = pytest.mark.gpu

N_RAYS = 2000


@pytest.fixture(scope="module")
def wedge_batch():
    return workloads.build(*workloads.wedge_batch(N_RAYS, seed=2024), compute_grids=False)


def _march(b, form):
    with Engine(b, precision=form) as eng:
        out = eng.run()
        st = eng.stats()
    return out["tll"].copy(), st


def _per_ray_max(b, a, ref):
    r = b.rays
    mx = np.zeros(b.n_rays)
    for i in range(b.n_rays):
        s = slice(int(r["line_off"][i]), int(r["line_off"][i] + r["nvr"][i]))
        m = ref[s] < 100.0
        if np.any(m):
            mx[i] = np.max(np.abs(a[s][m] - ref[s][m]))
    return mx


def test_column_clusters_and_tiles_deterministic_and_forms_agree(cuda_device, wedge_batch):
    b = wedge_batch
    p1, st = _march(b, "plain")
    assert st["column_rays"] > 0, "the schedule must put some rays on the column kernel"
    assert st["kernel_launches"] > st["column_launches"], "and some on batched tiles"
    p2, _ = _march(b, "plain")
    assert np.array_equal(p1, p2), "two plain marches of one batch differ"
    rf, _ = _march(b, "refined")
    d = _per_ray_max(b, rf, p1)
    assert d.max() <= 1e-4, f"refined vs plain: ray {int(np.argmax(d))} off by {d.max():.3g} dB"
    ch, _ = _march(b, "chosen")
    d = _per_ray_max(b, ch, p1)
    assert d.max() <= 1.0, f"chosen vs plain: ray {int(np.argmax(d))} off by {d.max():.3g} dB"
    m = p1 < 100.0
    assert np.sqrt(np.mean((ch[m] - p1[m]) ** 2)) <= 0.1
