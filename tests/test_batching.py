"""AsyncBatcher: the reference's prefetching pool (cupyram/batching.py:5-152).

Results come back in submission order whatever the order in which the workers
finish, at most max_prefetch tasks are in flight, worker errors reach the
iterating process, and share_object / load_shared_object /
cleanup_shared_object pass a read-only object to the workers through shared
memory.  The pool uses spawned processes.
"""
import numpy as np
import pytest

import batcher_workers as W
from golden_cases import load_case
from cupyram_b200 import AsyncBatcher
from cupyram_b200 import batch as B


def test_results_in_submission_order():
    # the early tasks sleep longest, so the workers finish them last
    tasks = [(i, 0.05 * (5 - i)) for i in range(6)]
    batcher = AsyncBatcher(iter(tasks), W.square_after, max_prefetch=3, max_workers=3)
    out, in_flight = [], []
    for res in batcher:
        in_flight.append(len(batcher._pending))
        out.append(res)
    assert [r[0] for r in out] == [i * i for i in range(6)]
    assert max(in_flight) <= 3
    assert len({r[1] for r in out}) > 1  # more than one worker process took part


def test_worker_error_reaches_the_caller():
    batcher = AsyncBatcher(((i, 2) for i in range(5)), W.fail_on, max_prefetch=2, max_workers=2)
    got = []
    with pytest.raises(ValueError, match="task 2 failed"):
        for r in batcher:
            got.append(r)
    assert got == [0, 1]


def test_empty_input_and_bad_arguments():
    assert list(AsyncBatcher(iter([]), W.fail_on)) == []
    with pytest.raises(ValueError):
        AsyncBatcher(iter([]), W.fail_on, max_prefetch=0)


def test_shared_object_round_trip():
    obj = {"a": np.arange(1000, dtype=np.float64)}
    name, size = AsyncBatcher.share_object(obj)
    try:
        assert np.array_equal(AsyncBatcher.load_shared_object(name, size)["a"], obj["a"])
        res = list(AsyncBatcher(((name, size, k) for k in (10, 100, 1000)), W.shared_sum, max_workers=2))
        assert res == [float(obj["a"][:k].sum()) for k in (10, 100, 1000)]
    finally:
        AsyncBatcher.cleanup_shared_object(name)
    AsyncBatcher.cleanup_shared_object(name)  # a second cleanup is harmless
    with pytest.raises(FileNotFoundError):
        AsyncBatcher.load_shared_object(name, size)


def test_batches_packed_in_workers_match_packing_in_process():
    args, kw, _ = load_case("ragged_batch")
    jobs = [(args, dict(kw, rmax=r)) for r in (1000.0, 2000.0, 3000.0)]
    got = list(AsyncBatcher(iter(jobs), W.pack_batch, max_prefetch=2, max_workers=2))
    for (a, k), b in zip(jobs, got):
        envs, p, zs, zr, pr = B.prepare(*a, dict(k))
        ref = B.build_batch(envs, p, zs, zr, pr, False)
        for f in ("rays", "envs", "pool"):
            assert getattr(b, f).tobytes() == getattr(ref, f).tobytes(), f
