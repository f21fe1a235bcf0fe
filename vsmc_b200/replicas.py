"""Host side of the multi-GPU run: independent filters spread over ranks.

Single filter: independent replicas, one per rank.  Batched filters: the
filter list is partitioned across ranks (each rank runs its share in one
batch on its own GPU), with no collective on the data path.

One filter's SMC step does not shard without an exchange step, so the
sharded unit is a whole filter.  Rank r runs its own filter of N particles
on its own counter stream (the fourth Philox counter word is the stream id,
so every rank's particle streams and observation series differ) with no
collective on the data path.  The only collective is the timing: each rank's
elapsed time is reduced with MAX, and the job's throughput is the units all
ranks processed divided by that time (weak scaling: per-rank work is fixed).

The helpers take the process group's module (torch.distributed, or None for
a single process) and the device its tensors live on, so the same code runs
over NCCL on GPUs and over gloo on CPU processes.
"""
from __future__ import annotations


def replica(rank: int, seed: int = 101) -> dict:
    """The filter rank `rank` runs: its counter stream and its seed.  The
    stream id separates the ranks' particle streams and observation series;
    the seed (the resample engine and the particle keys) is the same on
    every rank, as in a vSMC program started once per node."""
    if rank < 0:
        raise ValueError("rank must be >= 0")
    return {"stream_id": rank, "seed": seed}


def max_over_ranks(x: float, dist=None, device="cpu") -> float:
    """The largest of every rank's `x` (elapsed seconds or milliseconds):
    the job's time is its slowest rank's."""
    if dist is None:
        return float(x)
    import torch

    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(world: int, N: int, steps: int, seconds: float) -> float:
    """Particle-steps per second of the whole job: world filters of N
    particles, `steps` steps each, in the slowest rank's time."""
    if seconds <= 0.0:
        raise ValueError("elapsed time must be positive")
    return world * N * steps / seconds


def partition_filters(work, world: int) -> list:
    """Filter indices of each rank for a batch whose filter k costs work[k]
    (particles x steps): longest processing time first, each filter to the
    rank with the least work so far (ties to the lower rank), then each
    rank's list in ascending filter order.  Deterministic, so every rank
    computes the same partition without a collective; every filter goes to
    exactly one rank."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(work)), key=lambda k: (-int(work[k]), k))
    load = [0] * world
    parts = [[] for _ in range(world)]
    for k in order:
        r = min(range(world), key=lambda q: (load[q], q))
        parts[r].append(k)
        load[r] += int(work[k])
    return [sorted(p) for p in parts]


def gather_results(values, dist=None, device="cpu"):
    """Every rank's list of per-filter results (equal-length float lists are
    not required): all_gather of a padded tensor, returned as a list per
    rank.  Used for the job's results, never on the timed data path."""
    if dist is None:
        return [list(values)]
    import torch

    world = dist.get_world_size()
    n = torch.tensor([len(values)], dtype=torch.int64, device=device)
    ns = [torch.zeros_like(n) for _ in range(world)]
    dist.all_gather(ns, n)
    m = int(max(int(x.item()) for x in ns))
    t = torch.full((max(m, 1),), float("nan"), dtype=torch.float64, device=device)
    if values:
        t[: len(values)] = torch.tensor(list(values), dtype=torch.float64, device=device)
    ts = [torch.zeros_like(t) for _ in range(world)]
    dist.all_gather(ts, t)
    return [ts[r][: int(ns[r].item())].tolist() for r in range(world)]
