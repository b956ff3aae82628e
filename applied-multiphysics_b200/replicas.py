"""Host logic for running the solver on several GPUs of one node, one process per GPU.

The supernodal factorization of one matrix runs on one GPU; what shards is a batch of independent matrices (the
batched 2D heat set: 256 problems of uneven size). Ranks split such a batch with no data-path collective; the only
collectives are the timing reductions (max over ranks) and the count of units processed. For a single system every
rank solves its own replica.
"""
from __future__ import annotations

import datetime
import os
from dataclasses import dataclass
from typing import Sequence


@dataclass(frozen=True)
class RankInfo:
    rank: int
    world: int
    local_rank: int

    @staticmethod
    def from_env() -> "RankInfo":
        return RankInfo(int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
                        int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str, timeout_s: float = 120.0):
    """Join the process group (MASTER_ADDR / MASTER_PORT / RANK / WORLD_SIZE from the environment) with a short
    timeout, so that a rank that never arrives ends the others' next collective with an error."""
    import torch.distributed as dist

    if not dist.is_initialized():
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return dist


def shard_batch(costs: Sequence[float], world: int) -> list[list[int]]:
    """Split independent problems over `world` ranks: longest-processing-time first, each to the least-loaded rank
    (ties to the lower rank), then each rank's list in increasing index. Deterministic, so every rank computes the
    same assignment without communicating."""
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    load = [0.0] * world
    parts: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        parts[r].append(i)
        load[r] += float(costs[i])
    return [sorted(p) for p in parts]


def _reduce(value: float, op_name: str, device) -> float:
    import torch
    import torch.distributed as dist

    if not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=getattr(dist.ReduceOp, op_name))
    return float(t.item())


def max_over_ranks(value: float, device="cpu") -> float:
    """Max of a per-rank time over all ranks (every rank must call it, in the same order)."""
    return _reduce(value, "MAX", device)


def sum_over_ranks(value: float, device="cpu") -> float:
    """Sum of a per-rank count over all ranks (every rank must call it, in the same order)."""
    return _reduce(value, "SUM", device)
