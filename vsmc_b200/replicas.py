"""Host side of the multi-GPU run: independent filter replicas, one per rank.

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
