"""Replica bookkeeping of a multi-GPU run (one process per GPU, torch.distributed).

The fused kNN path shards by query rows with no data-path exchange: each rank runs an
independent replica on its own seeded query set against the same references. A timed step is
bracketed by a barrier on every rank; the reported step time is the maximum over ranks and the
whole-job throughput is the evaluations of all ranks divided by that time.
"""
from __future__ import annotations

import numpy as np


def replica_queries(rank: int, world: int, n_points: int, n_queries: int,
                    default: np.ndarray | None = None, seed: int = 1000) -> np.ndarray:
    """Query rows of this rank: the workload's own list on a single process, otherwise a
    seeded permutation prefix per rank (independent replicas, weak scaling)."""
    from rnn_b200 import workloads as W
    if world == 1 and default is not None:
        return np.ascontiguousarray(default[:n_queries], dtype=np.int32)
    return W.permutation(seed + rank, n_points)[:n_queries].astype(np.int32)


def barrier() -> None:
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.barrier()


def max_over_ranks(value: float, device=None) -> float:
    """Maximum of `value` over all ranks (the value itself on a single process). Uses the
    process group's backend: CUDA tensors for NCCL, CPU tensors for gloo."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64,
                     device=device if device is not None else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(evals_per_rank: float, world: int, max_ms: float) -> float:
    """Whole-job evaluations per second: all ranks' work over the slowest rank's time."""
    return evals_per_rank * world / (max_ms * 1e-3)
