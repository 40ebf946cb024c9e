"""Independent problem replicas, one process per GPU.

Multigrid problems shard across GPUs only as whole problems (no exchange
inside a V-cycle is needed for a problem that fits one GPU), so a multi-GPU
run is N independent solves: rank r solves its own seeded problem, and the
only collectives are the barriers around a timed region and the max over
ranks of its device time.  The job's aggregate time per solve is that max
divided by the number of ranks (N solves finish within it).

Launched by torch.distributed.run (RANK, LOCAL_RANK, WORLD_SIZE, MASTER_*
from the environment); a single process needs no launcher.
"""
from __future__ import annotations

import os
from datetime import timedelta


class Replicas:
    def __init__(self, backend: str = "nccl", timeout_s: float = 300.0):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.backend = backend
        self.device = None
        if self.world > 1:
            import torch
            import torch.distributed as dist
            kw = {}
            if backend == "nccl":
                self.device = torch.device("cuda", self.local)
                kw["device_id"] = self.device
            dist.init_process_group(backend, timeout=timedelta(seconds=timeout_s), **kw)

    def barrier(self):
        if self.world > 1:
            import torch.distributed as dist
            dist.barrier()

    def max(self, v: float) -> float:
        """Max of v over the ranks (every rank gets it)."""
        if self.world == 1:
            return float(v)
        import torch
        import torch.distributed as dist
        t = torch.tensor([float(v)], dtype=torch.float64, device=self.device or "cpu")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def seed(self, base: int) -> int:
        """This rank's problem seed: one independent problem per rank."""
        return base + self.rank

    def per_solve(self, t_max: float) -> float:
        """Aggregate time per solve of the job: N solves within t_max."""
        return t_max / self.world

    @property
    def is_root(self) -> bool:
        return self.rank == 0

    def close(self):
        if self.world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
