"""One process per GPU, each running its own replica of the case.

The per-step solver path has no data exchange between GPUs (every rank steps
its own copy of the case; nothing crosses NVLink on the data path), so the
only collectives are the timing barrier and the max-over-ranks reduction of
the measured time.  The backend is NCCL on GPUs and gloo on CPU (tests).
"""
from __future__ import annotations

import datetime
import os
from dataclasses import dataclass
from typing import Optional


@dataclass
class Replicas:
    rank: int = 0
    world: int = 1
    local: int = 0
    dist: Optional[object] = None  # torch.distributed when world > 1
    device: str = "cpu"

    def barrier(self) -> None:
        import torch

        if self.dist is not None:
            self.dist.barrier()
        if self.device.startswith("cuda"):
            torch.cuda.synchronize()

    def max_over_ranks(self, v: float) -> float:
        """The largest of every rank's v (timing: the slowest replica sets the job time)."""
        if self.dist is None:
            return float(v)
        import torch

        t = torch.tensor([float(v)], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def aggregate_rate(self, units_per_rank: float, seconds_max: float) -> float:
        """Whole-job throughput: every rank processed units_per_rank in at most seconds_max."""
        return self.world * units_per_rank / seconds_max

    def close(self) -> None:
        if self.dist is not None:
            self.dist.barrier()
            self.dist.destroy_process_group()
            self.dist = None


def from_env(backend: Optional[str] = None, timeout_s: int = 300) -> Replicas:
    """Reads RANK / WORLD_SIZE / LOCAL_RANK (torchrun) and joins the process group
    when WORLD_SIZE > 1.  backend defaults to nccl with CUDA, else gloo."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    import torch

    cuda = torch.cuda.is_available()
    if cuda:
        torch.cuda.set_device(local)
    device = f"cuda:{local}" if cuda else "cpu"
    r = Replicas(rank=rank, world=world, local=local, device=device)
    if world > 1:
        import torch.distributed as dist

        be = backend or ("nccl" if cuda else "gloo")
        if be == "gloo":
            r.device = "cpu"
        dist.init_process_group(be, timeout=datetime.timedelta(seconds=timeout_s))
        r.dist = dist
    return r
