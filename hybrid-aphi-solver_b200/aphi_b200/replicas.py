"""Frequency replicas over several GPUs, one process per GPU.

The path does not shard: a factorization runs on one GPU. Several GPUs each
solve their own sweep (independent frequencies of the same mesh) with no data
exchange. The only collectives are the barriers around timed regions and the
max-over-ranks reduction of their times, since the whole job is as fast as its
slowest rank. The backend is whatever the process group was initialised with:
NCCL on GPUs, gloo on CPU for the tests.
"""
from __future__ import annotations

import os

import numpy as np


def dist_env() -> tuple[int, int, int]:
    """(rank, world size, local rank) from the launcher's environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def rank_omegas(rank: int, nfreq: int, f_lo: float, f_hi: float) -> np.ndarray:
    """Rank `rank`'s sweep: nfreq log-spaced frequencies in [f_lo, f_hi] (rad/s),
    scaled by 1 + 1e-3 * rank so that every rank solves different systems."""
    return 2 * np.pi * np.geomspace(f_lo, f_hi, nfreq) * (1.0 + 1e-3 * rank)


def _group():
    import torch.distributed as dist
    return dist if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1 else None


def barrier() -> None:
    """Every rank reaches this point before any continues (no-op alone)."""
    d = _group()
    if d is not None:
        d.barrier()


def max_over_ranks(values, device=None) -> list[float]:
    """Element-wise maximum of per-rank values across the process group, in
    one collective (the values themselves when there is no group)."""
    v = [float(x) for x in values]
    d = _group()
    if d is None:
        return v
    import torch
    t = torch.tensor(v, dtype=torch.float64, device=device)
    d.all_reduce(t, op=d.ReduceOp.MAX)
    return [float(x) for x in t.tolist()]


def job_rate(world: int, units_per_rank: float, ms: float) -> float:
    """Whole-job throughput: every rank's units over the slowest rank's time (ms)."""
    return world * units_per_rank / (ms / 1000.0)
