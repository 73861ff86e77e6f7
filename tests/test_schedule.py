"""The column policy's cost rule (cr_plan_columns), on the CPU.

cr_create sends a ray to the column-parallel kernel when its lockstep march in
a batched tile, (nz + 2)(nr + 4 + 4 x operator changes) x row_step_s, would
exceed 1.25 x the batch's balanced time, sum(nz nr) / updates_per_s - with
both costs measured on the device by the engine's tuner.  These tests fix the
costs and check the rule's choices.
"""
import numpy as np

from cupyram_b200 import batch as B
from cupyram_b200 import workloads
from cupyram_b200.engine import plan_columns

ROUND1 = (0.3e-6, 1.3e10)  # one B200's measured costs for the plain form


def _mixed(n_short=3500):
    """3500 short rays (nz 99, 59 steps) and two long ones (nz 299, 2999 steps)."""
    long_ids = {0, n_short // 2 + 1}
    is_long = [i in long_ids for i in range(n_short + 2)]
    n = len(is_long)
    rmax = np.array([30000.0 if L else 600.0 for L in is_long])
    dep = [200.0 if L else 40.0 for L in is_long]
    args = [np.full(n, 100.0), np.full(n, 10.0), np.full(n, 10.0),
            [np.array([0.0, 250.0 if L else 60.0]) for L in is_long], [np.array([0.0])] * n,
            [np.array([[1500.0], [1500.0]])] * n, [np.array([0.0, 20.0 if L else 10.0]) for L in is_long],
            [np.array([0.0])] * n, [np.array([[1700.0], [1700.0]])] * n, [np.array([[1.5], [1.5]])] * n,
            [np.array([[0.5], [0.5]])] * n, [np.array([[0.0, d], [r, d]]) for d, r in zip(dep, rmax)]]
    kw = dict(batch_size=n, per_ray=True, dz=1.0, dr=10.0, rmax=rmax, np=4, lyrw=2)
    envs, p, zs, zr, pr = B.prepare(*args, kw)
    return B.build_batch(envs, p, zs, zr, pr, False), sorted(long_ids)


def test_long_rays_leave_the_batched_kernel():
    b, longs = _mixed()
    col = plan_columns(b, *ROUND1)
    assert list(np.flatnonzero(col)) == longs


def test_choices_follow_the_measured_costs():
    """A slower batched throughput lengthens the balanced time: fewer rays leave;
    a slower tile (row step) makes more rays outlast it."""
    b, longs = _mixed()
    assert not plan_columns(b, ROUND1[0], ROUND1[1] / 1000.0).any()
    assert not plan_columns(b, ROUND1[0] / 1000.0, ROUND1[1]).any()
    assert plan_columns(b, ROUND1[0] * 1000.0, ROUND1[1]).all()


def test_rule_matches_its_formula():
    """The rule's boundary, computed here from the same formula."""
    b, _ = _mixed(600)
    r = b.rays
    work = float(np.sum(r["nz"].astype(float) * r["nr"]))
    lock = (r["nz"] + 2.0) * (r["nr"] + 4.0)  # flat bottoms, one profile: no operator changes
    for ups in (1e9, 3e9, 1e10):
        row = 1.25 * (work / ups) / np.sort(lock)[-2] * 1.0001  # just above the second-longest's boundary
        col = plan_columns(b, row, ups)
        assert np.array_equal(col, lock * row > 1.25 * work / ups)


def test_homogeneous_batch_stays_batched():
    """The 4096-ray Munk batch: every ray's lockstep march is close to the balanced
    time, so all stay batched; the same rays in a batch of 256 would leave the GPU
    idle on the batched kernel, so all go to the column kernel."""
    b = workloads.build(*workloads.munk_batch(4096, seed=9), compute_grids=False)
    assert not plan_columns(b, *ROUND1).any()
    small = workloads.build(*workloads.munk_batch(256, seed=9), compute_grids=False)
    assert plan_columns(small, *ROUND1).all()
