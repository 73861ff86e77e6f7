"""The multi-GPU benchmark path on CPU: two gloo ranks on 127.0.0.1.

bench.py --gpus N runs one process per GPU, each marching its own seeded
batch of the same size (weak scaling, no data-path collective); the timings
are reduced as a maximum over ranks and the whole-job rate counts every
rank's updates.  This test runs those host-side pieces in two processes.
"""
import json
import os
import socket
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, outdir):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    sys.argv = ["bench.py", "--rays", "4", "--rmax", "1000", "--steps", "2"]
    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        a = bench.parse()
        batch, cfg = bench.workload(a, rank)
        # per-rank timings: the slowest rank sets the job's time
        t = bench.max_over_ranks(dist, [100.0 + 10.0 * rank, 50.0 - 5.0 * rank], device="cpu")
        total = bench.sum_over_ranks(dist, batch.point_updates, device="cpu")
        rate = bench.whole_job_rate(total, a.steps, t[0])
        res = {"seed": cfg["seed"], "updates": batch.point_updates, "n_rays": int(batch.n_rays),
               "freq0": float(batch.rays["freq"][0]), "t": t, "rate": rate}
        Path(outdir, f"rank{rank}.json").write_text(json.dumps(res))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_ranks_weak_scaling_and_max_timing(tmp_path):
    import torch.multiprocessing as mp
    world = 2
    mp.spawn(_rank, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    r = [json.loads(Path(tmp_path, f"rank{k}.json").read_text()) for k in range(world)]
    # each rank marches its own seeded batch of the same size
    assert r[0]["seed"] != r[1]["seed"] and r[0]["freq0"] != r[1]["freq0"]
    assert r[0]["n_rays"] == r[1]["n_rays"] == 4
    # the reduction is the element-wise maximum, identical on every rank
    assert r[0]["t"] == r[1]["t"] == [110.0, 50.0]
    # the whole job's rate counts both ranks' updates within the slowest rank's time
    assert np.isclose(r[0]["rate"], (r[0]["updates"] + r[1]["updates"]) * 2 / 0.110)
    assert r[0]["rate"] == r[1]["rate"]
