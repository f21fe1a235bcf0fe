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


def _batch_rank_main(rank, world, port, out):
    """One rank of a filter-partitioned batch: its share of a small batch of
    uneven filters, each run through the oracle (the CPU checker standing in
    for the device batch), the slowest rank's time, and the gathered
    per-filter log-evidence."""
    import datetime
    import time

    import torch.distributed as dist

    from oracle import oracle as O
    from vsmc_b200 import replicas

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        Ns, Ts = _batch_workload()
        parts = replicas.partition_filters([n * t for n, t in zip(Ns, Ts)], world)
        mine = parts[rank]
        t0 = time.perf_counter()
        logz = []
        for k in mine:
            ox, oy = O.cv_simulate(Ts[k], 1000 + k, stream=k)
            logz.append(O.cv_filter(Ns[k], Ts[k], 0, ox, oy, seed=101 + k, stream=k)["logz"])
        slowest = replicas.max_over_ranks(time.perf_counter() - t0, dist, device="cpu")
        got = replicas.gather_results(logz, dist, device="cpu")
        np.savez(os.path.join(out, f"batch{rank}.npz"), parts=np.array(
            [np.array(p + [-1] * (len(Ns) - len(p))) for p in parts]), mine=np.array(mine),
            slowest=slowest, got=np.array([x for g in got for x in g]),
            order=np.array([k for p in parts for k in p]))
    finally:
        dist.destroy_process_group()


def _batch_workload():
    rng = np.random.default_rng(3)
    Ns = [int(x) for x in np.exp(rng.uniform(np.log(64), np.log(1024), 9)).astype(int)]
    Ts = [int(x) for x in rng.integers(5, 20, 9)]
    return Ns, Ts


def test_partitioned_batch_over_gloo(tmp_path):
    """Two ranks split a batch of uneven filters by work: each filter runs on
    exactly one rank, the per-rank work is balanced, both ranks see the same
    slowest time, and the gathered results equal a single-process run of
    every filter."""
    from oracle import oracle as O
    from vsmc_b200 import replicas

    world = 2
    mp.start_processes(_batch_rank_main, args=(world, _free_port(), str(tmp_path)),
                       nprocs=world, join=True, start_method="spawn")
    r = [np.load(tmp_path / f"batch{k}.npz") for k in range(world)]
    Ns, Ts = _batch_workload()
    parts = replicas.partition_filters([n * t for n, t in zip(Ns, Ts)], world)
    assert sorted(k for p in parts for k in p) == list(range(len(Ns)))
    for k in range(world):
        assert list(r[k]["mine"]) == parts[k]
    assert float(r[0]["slowest"]) == float(r[1]["slowest"])
    work = [sum(Ns[k] * Ts[k] for k in p) for p in parts]
    assert max(work) - min(work) <= max(n * t for n, t in zip(Ns, Ts))
    want = {}
    for k in range(len(Ns)):
        ox, oy = O.cv_simulate(Ts[k], 1000 + k, stream=k)
        want[k] = O.cv_filter(Ns[k], Ts[k], 0, ox, oy, seed=101 + k, stream=k)["logz"]
    order = list(r[0]["order"])
    assert [want[k] for k in order] == list(r[0]["got"])
    assert np.array_equal(r[0]["got"], r[1]["got"])


def test_partition_filters_properties():
    from vsmc_b200 import replicas

    work = [5, 1, 9, 9, 2, 7, 3]
    for world in (1, 2, 3, 8):
        parts = replicas.partition_filters(work, world)
        assert len(parts) == world
        assert sorted(k for p in parts for k in p) == list(range(len(work)))
        assert replicas.partition_filters(work, world) == parts
    assert replicas.partition_filters(work, 2) == [[2, 4, 5], [0, 1, 3, 6]]
    with pytest.raises(ValueError):
        replicas.partition_filters(work, 0)
