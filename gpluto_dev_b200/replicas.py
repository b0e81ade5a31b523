"""Replica mode for several GPUs of one node: one process per GPU, each
advancing its own independent grid(s); no data-path collective.

The Godunov step of one grid never crosses GPUs (every configuration fits
one B200), so the multi-GPU run is N independent replicas.  The process
group exists only for the timing discipline: a barrier on both sides of the
timed region and the maximum of the ranks' times, from which the whole-job
rate is taken (zone updates of all ranks / slowest rank's time).

The same functions run over NCCL on the GPUs and over gloo on the CPU, where
the tests exercise them with two ranks.
"""
from __future__ import annotations

import datetime
import os
from dataclasses import dataclass


@dataclass
class Ranks:
    world: int
    rank: int
    local: int
    dist: object = None          # torch.distributed when world > 1
    device: str = "cpu"          # device of the reduction tensors

    def barrier(self) -> None:
        if self.dist is not None:
            self.dist.barrier()

    def max_over_ranks(self, x: float) -> float:
        """Largest value of `x` over the ranks (every rank receives it)."""
        if self.dist is None:
            return float(x)
        import torch
        t = torch.tensor([float(x)], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def close(self) -> None:
        if self.dist is not None:
            self.barrier()
            self.dist.destroy_process_group()
            self.dist = None


def from_env() -> tuple[int, int, int]:
    """(WORLD_SIZE, RANK, LOCAL_RANK) as set by torch.distributed.run."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str = "nccl", timeout_s: float = 300.0) -> Ranks:
    """Join the process group of a torchrun launch (nothing for one rank).

    With NCCL each rank binds its GPU (LOCAL_RANK) and the reductions run on
    it; the short timeout turns a rank that never joins into an error on the
    others instead of a hang."""
    world, rank, local = from_env()
    r = Ranks(world, rank, local)
    if world > 1:
        import torch
        import torch.distributed as dist
        kw = {}
        if backend == "nccl":
            torch.cuda.set_device(local)
            kw["device_id"] = torch.device("cuda", local)
            r.device = "cuda"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s), **kw)
        r.dist = dist
    return r


def whole_job_rate(world: int, units_per_rank: float, steps: int, t_ms: float) -> float:
    """Units (zone updates) of all ranks per second, in millions, over the
    slowest rank's time `t_ms` for `steps` steps."""
    return world * units_per_rank * steps / (t_ms * 1e-3) / 1e6


def replica_seed(base: int, rank: int, per_rank: int = 1) -> int:
    """Seed of rank `rank`'s first grid: replicas integrate different data."""
    return base + rank * per_rank
