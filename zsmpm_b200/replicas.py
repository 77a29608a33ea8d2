"""One process per GPU running independent replicas of the substep.

The MPM substep has no exchange step between independent systems, so N GPUs run N replicas
(or N shards of a batch of independent scenes) with no data-path collective.  The process group
is used only to line the ranks up before and after the timed region and to take the slowest
rank's device time, from which the whole-job throughput is computed.  NCCL on GPUs; gloo on CPU
(the tests run two gloo ranks).
"""
from __future__ import annotations

import datetime
import os


def world() -> tuple[int, int, int]:
    """(world size, rank, local rank) from the torchrun environment (1, 0, 0 without it)."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str = "nccl", timeout_s: int = 120) -> tuple[int, int, int]:
    ws, rank, local = world()
    if ws > 1:
        import torch.distributed as dist
        if not dist.is_initialized():
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return ws, rank, local


def _device():
    import torch.distributed as dist
    return "cuda" if dist.get_backend() == "nccl" else "cpu"


def max_over_ranks(x: float) -> float:
    """The maximum of x over all ranks (x itself with one rank)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return x
    t = torch.tensor([x], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier() -> None:
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.barrier()


def throughput(units_per_rank: int, steps: int, max_ms: float, world_size: int) -> float:
    """Whole-job units per second: every rank processed units_per_rank per step; the job took
    the slowest rank's time."""
    return units_per_rank * steps * world_size / (max_ms * 1e-3)


def shard(n_items: int, rank: int, world_size: int) -> range:
    """Contiguous share of n_items (e.g. scenes of a batch) for one rank."""
    base, extra = divmod(n_items, world_size)
    lo = rank * base + min(rank, extra)
    return range(lo, lo + base + (1 if rank < extra else 0))


def finish() -> None:
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        dist.destroy_process_group()
