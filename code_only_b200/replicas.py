"""One process per GPU running independent solves (replicas).

The FMG path is solved on one GPU; with N GPUs every rank solves its own
hierarchy and no data crosses between ranks.  The only collectives are the
timing ones: a barrier on both sides of the timed region and a max over ranks
of the elapsed time, so that the reported throughput is all ranks' solves
divided by the slowest rank's time.  NCCL carries them on GPUs; gloo on CPU
(tests).  A rank that fails raises on every rank at the next collective
(bounded by the process-group timeout) instead of hanging.
"""
from __future__ import annotations

import datetime
import os
from dataclasses import dataclass
from typing import Callable, Optional


@dataclass
class RankInfo:
    rank: int = 0
    world: int = 1
    local: int = 0
    backend: Optional[str] = None


def setup(backend: Optional[str] = None, timeout_s: float = 600.0) -> RankInfo:
    """Initialises the process group from RANK/WORLD_SIZE/LOCAL_RANK (torchrun)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if world <= 1:
        return RankInfo()
    import torch
    import torch.distributed as dist
    rank = int(os.environ["RANK"])
    local = int(os.environ.get("LOCAL_RANK", rank))
    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    if backend is None:
        backend = "nccl" if torch.cuda.is_available() else "gloo"
    kw = {}
    if backend == "nccl":
        torch.cuda.set_device(local)
        kw["device_id"] = torch.device("cuda", local)
    dist.init_process_group(backend, rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=timeout_s), **kw)
    return RankInfo(rank, world, local, backend)


def _device(info: RankInfo):
    import torch
    return torch.device("cuda", info.local) if info.backend == "nccl" else torch.device("cpu")


def barrier(info: RankInfo) -> None:
    if info.world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(info: RankInfo, x: float) -> float:
    if info.world <= 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=_device(info))
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(info: RankInfo, x: float) -> float:
    if info.world <= 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=_device(info))
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def timed_replicas(info: RankInfo, step: Callable[[], None], steps: int, warmup: int,
                   clock: Callable[[Callable[[], None], int], float]) -> dict:
    """Runs `warmup` untimed and `steps` timed calls of `step` on every rank.
    `clock(fn, k)` returns the milliseconds k calls of fn take on this rank
    (CUDA events on GPUs).  Returns the weak-scaling throughput."""
    for _ in range(warmup):
        step()
    barrier(info)
    ms = clock(step, steps)
    barrier(info)
    ms_max = max_over_ranks(info, ms)
    solves = sum_over_ranks(info, float(steps))
    return {"ms_per_step": ms_max / steps, "solves_per_s": solves * 1e3 / ms_max, "world": info.world}


def teardown(info: RankInfo) -> None:
    if info.world > 1:
        import torch.distributed as dist
        if dist.is_initialized():
            dist.destroy_process_group()
