"""Host logic of the multi-GPU replica runs: one process per GPU, each solving its own
systems with no exchange on the data path.

The reference splits one lattice over ranks (mp.cpp); here a lattice fits one GPU, so N GPUs
run N independent replicas (different sources, or different configurations), and the only
collectives are the barrier that brackets a timed region and the maximum of its duration
over the ranks.  Works with any torch.distributed backend (NCCL on the GPUs, gloo on CPU)."""
from __future__ import annotations

SEED_STRIDE = 7919


def rank_seed(seed: int, rank: int) -> int:
    """the seed of rank `rank`'s inputs: distinct per rank, reproducible per (seed, rank)"""
    return int(seed) + SEED_STRIDE * int(rank)


def barrier(dist=None, synchronize=None):
    """all ranks meet (when distributed), then the local device drains"""
    if dist is not None:
        dist.barrier()
    if synchronize is not None:
        synchronize()


def max_over_ranks(value: float, dist=None, device: str = "cpu") -> float:
    """the largest of the ranks' values (a duration: the job ends with its slowest rank)"""
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_time_per_solve(ms_max: float, world: int) -> float:
    """whole-job time per solve: `world` solves run concurrently in `ms_max`"""
    if world < 1:
        raise ValueError("world must be >= 1")
    return ms_max / world
