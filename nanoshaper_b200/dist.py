"""Multi-process plumbing of the benchmark: one process per GPU, independent replicas.

The surface path has no cross-GPU exchange (structures are independent), so ranks only agree on
timing: the slowest rank's time per step, and the whole job's throughput as all ranks' units over
that time.  The same code runs over NCCL on GPUs and over gloo on the CPU (tests).
"""
from __future__ import annotations

import os
from datetime import timedelta


def env() -> tuple[int, int, int]:
    """(world size, rank, local rank) from the torchrun environment (1, 0, 0 without it)."""
    return int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")), int(os.environ.get("LOCAL_RANK", "0"))


def init(backend: str, timeout_s: float = 300.0):
    """Process group from the environment, or None for a single process."""
    world, _, _ = env()
    if world <= 1:
        return None
    import torch.distributed as dist
    dist.init_process_group(backend, timeout=timedelta(seconds=timeout_s))
    return dist


def max_over_ranks(pg, x: float) -> float:
    """The largest value over all ranks (the slowest replica's time)."""
    if pg is None:
        return float(x)
    import torch
    dev = "cuda" if pg.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def throughput(units_per_rank: float, world: int, ms_per_step: float) -> float:
    """Whole-job units per second: every rank processes units_per_rank per step and the step time
    is the slowest rank's."""
    return world * units_per_rank * 1000.0 / ms_per_step


def barrier(pg) -> None:
    if pg is not None:
        pg.barrier()


def close(pg) -> None:
    if pg is not None:
        pg.destroy_process_group()
