"""Replicas across GPUs: one process per GPU, each solving the same batch (weak scaling).

The slab-stepping path does not shard: one solve is a sequential chain of slab steps, and
independent solves need no exchange. N GPUs therefore run N independent replicas; the only
collective steps are the timing ones: a barrier around the timed region and the maximum of the
per-rank device times, from which the whole-job throughput is N × solves / max time.
"""

from __future__ import annotations

import os
from datetime import timedelta


def init(backend: str = "nccl", timeout_s: float = 600.0):
    """Joins the process group named by the torchrun environment (RANK, WORLD_SIZE, MASTER_*);
    returns (dist module or None for one process, rank, world size, local rank)."""
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    if ws <= 1:
        return None, 0, 1, 0
    import torch
    import torch.distributed as dist

    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    kwargs = {}
    if backend == "nccl":
        torch.cuda.set_device(local)
        kwargs["device_id"] = torch.device("cuda", local)
    dist.init_process_group(backend, timeout=timedelta(seconds=timeout_s), **kwargs)
    return dist, rank, ws, local


def max_over_ranks(dist, x: float) -> float:
    """The largest x over all ranks (x itself for one process)."""
    if dist is None:
        return x
    import torch

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(dist) -> None:
    if dist is not None:
        dist.barrier()


def throughput(world_size: int, solves_per_rank: int, step_ms_max: float) -> float:
    """Whole-job solves/s: every rank solves its batch in at most step_ms_max."""
    return world_size * solves_per_rank / (step_ms_max * 1e-3)
