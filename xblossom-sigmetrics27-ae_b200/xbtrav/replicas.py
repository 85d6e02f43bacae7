"""Multi-GPU layout of the traversal: replicas, one process per GPU.

Sources are independent, so each rank holds the whole graph and traverses
its own seeded source set; no data crosses between ranks.  The only
collectives are the ones that report the job: the slowest rank's time and
the total work.  bench.py uses these helpers under torchrun (NCCL);
tests/test_replicas_cpu.py runs them on two gloo ranks.
"""
from __future__ import annotations

RANK_SEED_STRIDE = 7919  # seeds of different ranks' source sets


def rank_seed(seed: int, rank: int) -> int:
    """Seed of rank `rank`'s source set (rank 0 uses seed itself)."""
    return seed + RANK_SEED_STRIDE * rank


def _reduce(dist, x: float, op, device) -> float:
    if dist is None:
        return float(x)
    import torch

    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=op)
    return float(t.item())


def max_over_ranks(dist, x: float, device="cpu") -> float:
    return _reduce(dist, x, None if dist is None else dist.ReduceOp.MAX, device)


def sum_over_ranks(dist, x: float, device="cpu") -> float:
    return _reduce(dist, x, None if dist is None else dist.ReduceOp.SUM, device)


def whole_job_gteps(dist, edges_local: float, ms_local: float, device="cpu") -> tuple[float, float]:
    """(GTEPS of the whole job, its time in ms): all ranks' processed edges
    over the slowest rank's time."""
    ms = max_over_ranks(dist, ms_local, device)
    edges = sum_over_ranks(dist, edges_local, device)
    return edges / (ms / 1e3) / 1e9, ms
