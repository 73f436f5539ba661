"""One process per GPU, each running its own replica of the workload (the
dedispersion path shards by beam or DM range with no data exchange): rank
discovery from the torchrun environment, a barrier, and the maximum of a
per-rank time over all ranks (whole-job time = slowest replica)."""
from __future__ import annotations

import datetime
import os
from dataclasses import dataclass


@dataclass
class Replicas:
    world: int
    rank: int
    local: int
    backend: str

    @classmethod
    def from_env(cls, backend: str = "nccl", timeout_s: int = 600) -> "Replicas":
        import torch
        import torch.distributed as dist
        world = int(os.environ.get("WORLD_SIZE", "1"))
        rank = int(os.environ.get("RANK", "0"))
        local = int(os.environ.get("LOCAL_RANK", "0"))
        if backend == "nccl":
            torch.cuda.set_device(local)
        if world > 1:
            kw = {"timeout": datetime.timedelta(seconds=timeout_s)}
            if backend == "nccl":
                kw["device_id"] = torch.device("cuda", local)
            dist.init_process_group(backend, **kw)
        return cls(world, rank, local, backend)

    def barrier(self) -> None:
        if self.world > 1:
            import torch.distributed as dist
            dist.barrier()

    def max_over_ranks(self, x: float) -> float:
        if self.world == 1:
            return x
        import torch
        import torch.distributed as dist
        dev = "cuda" if self.backend == "nccl" else "cpu"
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def close(self) -> None:
        if self.world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
