"""Multi-GPU form of the commitment path: independent replicas, one process per GPU.

Commitment jobs share nothing, so N GPUs run N independent job streams (weak scaling) with no
data-path collective; the only cross-rank step is the timing reduction (max over ranks), done
through torch.distributed (NCCL on GPUs, gloo in the CPU tests).
"""
from __future__ import annotations


def rank_seed(seed: str, rank: int) -> str:
    """Seed of the synthetic inputs of one rank's replica."""
    return "%s-rank%d" % (seed, rank)


def shard_jobs(jobs: list, rank: int, world: int) -> list:
    """Jobs of one rank when a batch is spread over ranks: round-robin by descending cost keeps
    the per-rank work balanced for uneven batches."""
    order = sorted(range(len(jobs)), key=lambda i: -job_cost(jobs[i]))
    return [jobs[i] for k, i in enumerate(order) if k % world == rank]


def job_cost(job) -> float:
    log_n, cols, log_lde = job[0], job[1], job[2]
    n, f = 1 << log_n, 1 << log_lde
    return 472.0 * (f * n * ((cols + 7) // 8) + f * n) + 1.5 * (1 + f) * cols * n * 0.5 * log_n


def max_over_ranks(value: float, device=None) -> float:
    """Max of `value` over all ranks of the default process group (identity when not
    initialised)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return value
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(units_per_rank: float, world: int, seconds_max: float) -> float:
    """Whole-job rate: every rank processed units_per_rank in at most seconds_max."""
    return units_per_rank * world / seconds_max
