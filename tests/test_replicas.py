"""The multi-GPU path's host logic on CPU processes (gloo, world size 2):
each rank runs its own filter on its own counter stream, the data path has
no collective, and the job's time is the slowest rank's (all_reduce MAX),
exactly as bench.py does over NCCL with one GPU per rank."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    from vsmc_b200 import capi, replicas

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        rep = replicas.replica(rank)
        ox, oy = capi.cv_simulate(16, 7, stream_id=rep["stream_id"])
        elapsed = [0.5, 0.8, 0.3, 0.6][rank]  # this rank's timed region (s)
        slowest = replicas.max_over_ranks(elapsed, dist, device="cpu")
        value = replicas.job_throughput(world, 1 << 20, 10, slowest)
        np.savez(os.path.join(out, f"rank{rank}.npz"), stream_id=rep["stream_id"],
                 seed=rep["seed"], ox=ox, oy=oy, slowest=slowest, value=value)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2])
def test_replicas_over_gloo(tmp_path, world):
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world,
                       join=True, start_method="spawn")
    r = [np.load(tmp_path / f"rank{k}.npz") for k in range(world)]
    # every rank sees the slowest rank's time and reports the same job rate
    assert all(float(x["slowest"]) == 0.8 for x in r)
    assert all(float(x["value"]) == world * (1 << 20) * 10 / 0.8 for x in r)
    # one unit per rank: distinct counter streams, distinct observation series
    assert sorted(int(x["stream_id"]) for x in r) == list(range(world))
    assert len({int(x["seed"]) for x in r}) == 1
    assert not np.array_equal(r[0]["ox"], r[1]["ox"])


def test_replica_helpers_single_process():
    from vsmc_b200 import replicas

    assert replicas.max_over_ranks(1.25) == 1.25
    assert replicas.replica(3) == {"stream_id": 3, "seed": 101}
    assert replicas.job_throughput(4, 1000, 10, 2.0) == 4 * 1000 * 10 / 2.0
    with pytest.raises(ValueError):
        replicas.replica(-1)
    with pytest.raises(ValueError):
        replicas.job_throughput(1, 10, 1, 0.0)
