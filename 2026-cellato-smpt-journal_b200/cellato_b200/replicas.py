"""Multi-GPU runs as independent replicas: one process per GPU, each running the
same workload on its own grids.  The bit-plane path has no exchange step (each
grid, batch or request stays on one GPU), so the only collectives are a barrier
around the timed region and a max over the ranks' device times; nothing crosses
NVLink on the data path.

The process group is NCCL when CUDA is available and gloo otherwise (the CPU
tests run two gloo ranks).  The rendezvous comes from the environment that
torch.distributed.run sets (RANK, WORLD_SIZE, MASTER_ADDR, MASTER_PORT).
"""
from __future__ import annotations

import datetime
import os


def world_from_env() -> tuple[int, int]:
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1"))


def init(timeout_s: float = 120.0, backend: str | None = None) -> tuple[int, int]:
    """Joins the process group when WORLD_SIZE > 1; returns (rank, world).
    backend: None = NCCL with CUDA, gloo without."""
    import torch
    rank, world = world_from_env()
    if world > 1 and not torch.distributed.is_initialized():
        backend = backend or ("nccl" if torch.cuda.is_available() else "gloo")
        if backend == "nccl":
            torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        torch.distributed.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return rank, world


def _device():
    import torch
    if torch.distributed.is_initialized() and torch.distributed.get_backend() == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def barrier() -> None:
    import torch
    if torch.distributed.is_initialized():
        torch.distributed.barrier()


def max_over_ranks(x: float) -> float:
    """The largest value over the ranks (a time: the slowest rank sets the job's)."""
    import torch
    if not torch.distributed.is_initialized():
        return x
    t = torch.tensor([x], dtype=torch.float64, device=_device())
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x: float) -> float:
    """The sum over the ranks (units of work that differ per rank)."""
    import torch
    if not torch.distributed.is_initialized():
        return x
    t = torch.tensor([x], dtype=torch.float64, device=_device())
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.SUM)
    return float(t.item())


def job_rate(units_per_rank: float, world: int, max_ms: float) -> float:
    """Whole-job throughput: the units all ranks processed over the slowest
    rank's time, per second."""
    return units_per_rank * world / (max_ms * 1e-3)


def shutdown() -> None:
    import torch
    if torch.distributed.is_initialized():
        torch.distributed.destroy_process_group()
