"""The column policy's cost rule (cr_plan_columns), on the CPU.

cr_create sends a ray to the column-parallel kernel when its lockstep march in
a batched tile, (nz + 2)(nr + 4 + 4 x operator changes) x row, would exceed
1.25 x the batch's balanced time, sum(nz nr) / updates_per_s; row is the larger
of a tile's row step alone and the pace at which the rays in flight (at most
slots x rays per tile) saturate the batched throughput - with the costs
measured on the device by the engine's tuner.  These tests fix the costs and
check the rule's choices.
"""
import numpy as np

from cupyram_b200 import batch as B
from cupyram_b200 import workloads
from cupyram_b200.engine import plan_columns

ROUND1 = (0.3e-6, 1.3e10)  # one B200's costs for the plain form: row step alone, updates/s
SLOTS = 835                # batched tiles a B200 holds at once


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
    """A slower tile alone makes more rays outlast the batch (at 1000x every ray
    does), and so does a faster batched throughput (a shorter balanced time: at
    10x every ray); a slower throughput lengthens the balanced time and the
    tiles' pace under load alike, so the long rays still leave and the short
    ones stay; at 1/1000 of the tile's row step the pace under load decides."""
    b, longs = _mixed()
    assert plan_columns(b, ROUND1[0] * 1000.0, ROUND1[1], SLOTS).all()
    assert plan_columns(b, ROUND1[0], ROUND1[1] * 10.0, SLOTS).all()
    assert list(np.flatnonzero(plan_columns(b, ROUND1[0], ROUND1[1] / 1000.0, SLOTS))) == longs
    assert list(np.flatnonzero(plan_columns(b, ROUND1[0] / 1000.0, ROUND1[1], SLOTS))) == longs


def test_rule_matches_its_formula():
    """The rule's boundary, computed here from the same formula."""
    b, _ = _mixed(600)
    r = b.rays
    work = float(np.sum(r["nz"].astype(float) * r["nr"]))
    lock = (r["nz"] + 2.0) * (r["nr"] + 4.0)  # flat bottoms, one profile: no operator changes
    per_tile = 32 // ((r["np"] + 1) // 2)
    for ups, slots in ((1e9, 0), (3e9, 10), (1e10, SLOTS)):
        in_flight = b.n_rays if slots <= 0 else min(b.n_rays, slots * per_tile.mean())
        for row0 in (1e-9, 1.25 * (work / ups) / np.sort(lock)[-2] * 1.0001):
            row = max(row0, in_flight / ups)
            col = plan_columns(b, row0, ups, slots)
            assert np.array_equal(col, lock * row > 1.25 * work / ups)


def test_homogeneous_batch_stays_batched():
    """The 4096-ray Munk batch: every ray's lockstep march is close to the balanced
    time, so all stay batched; the same rays in a batch of 256 would leave the GPU
    idle on the batched kernel, so all go to the column kernel."""
    b = workloads.build(*workloads.munk_batch(4096, seed=9), compute_grids=False)
    assert not plan_columns(b, *ROUND1, SLOTS).any()
    # a slower tile under load (its rays in flight saturating the throughput) does not change that
    assert not plan_columns(b, 1e-9, ROUND1[1], SLOTS).any()
    small = workloads.build(*workloads.munk_batch(256, seed=9), compute_grids=False)
    assert plan_columns(small, *ROUND1, SLOTS).all()
