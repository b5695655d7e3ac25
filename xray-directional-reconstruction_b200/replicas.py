"""Replica-parallel runs: one process per GPU, each reconstructing its own
specimen; no collective touches the data path.

The reference runs on one GPU and its reconstructions are independent per
specimen, so the multi-GPU form here is N independent replicas (weak
scaling).  The only collectives are the run's bookkeeping: a barrier around
the timed region and a MAX reduction of per-rank device times, so the
whole-job time is the slowest rank's.
"""
from __future__ import annotations

import os
from datetime import timedelta


def rank_env():
    """(rank, world size, local rank) from the torch.distributed launcher's
    environment; (0, 1, 0) when launched as a single process."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def specimen_seed(base: int, rank: int) -> int:
    """Each replica reconstructs a different seeded specimen."""
    return base + rank


def init(backend: str, timeout_s: float = 120.0) -> None:
    """Process group over 127.0.0.1 rendezvous (MASTER_ADDR/PORT from the
    launcher) with a short timeout, so a rank that never arrives ends the
    others' next collective with an error instead of a hang."""
    import torch.distributed as dist
    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    dist.init_process_group(backend, timeout=timedelta(seconds=timeout_s))


def barrier() -> None:
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        dist.barrier()


def max_over_ranks(values, device="cpu"):
    """Element-wise MAX of a list of floats over all ranks (every rank gets it)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.cpu().tolist()]


def whole_job_rate(units_per_rank: float, world: int, t_max_ms: float) -> float:
    """Units per second of the whole job: every rank processed
    units_per_rank, the job took the slowest rank's time."""
    return world * units_per_rank / (t_max_ms / 1e3)


def finish() -> None:
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        dist.barrier()
        dist.destroy_process_group()
