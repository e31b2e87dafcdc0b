"""Replica parallelism for the projection benchmark.

The projection does not shard across GPUs here: each rank (one process per
GPU) projects its own replica of the workload and ranks never exchange
grid data.  The only collectives are the timing barrier and a max over ranks
of the device-measured time; throughput is all ranks' solves divided by the
slowest rank's time.
"""
from __future__ import annotations

import datetime
import os
from dataclasses import dataclass


@dataclass
class Ranks:
    rank: int
    world: int
    local_rank: int
    backend: str | None

    @property
    def distributed(self) -> bool:
        return self.world > 1


def from_env() -> Ranks:
    return Ranks(int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
                 int(os.environ.get("LOCAL_RANK", "0")), None)


def init(ranks: Ranks, backend: str, device=None, timeout_s: float = 120.0) -> Ranks:
    """Join the process group (NCCL on GPUs, gloo on CPU) with a short timeout
    so that ranks waiting on a lost peer end with an error."""
    if ranks.world > 1:
        import torch.distributed as dist
        kw = {"timeout": datetime.timedelta(seconds=timeout_s)}
        if device is not None and backend == "nccl":
            kw["device_id"] = device
        dist.init_process_group(backend, **kw)
        ranks.backend = backend
    return ranks


def barrier(ranks: Ranks):
    if ranks.world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(ranks: Ranks, value: float, device=None) -> float:
    if ranks.world == 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64, device=device if ranks.backend == "nccl" else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def throughput(ranks: Ranks, units_per_rank: int, ms_max: float) -> float:
    """Whole-job units per second from the slowest rank's milliseconds."""
    return ranks.world * units_per_rank / (ms_max / 1e3)


def finish(ranks: Ranks):
    if ranks.world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
