"""One process per GPU, each advancing its own independent problems (replicas).

The finite-volume step has no data exchange between problems once the whole domain of
each problem is resident on one GPU (the reference's 2x1 host ghost exchange,
hydro2d/main.cxx:349-378, becomes in-kernel periodic addressing). Several GPUs therefore
run independent replicas or disjoint shares of a request stream; the only collectives
are the timing reduction (max over ranks) and barriers around the timed region.
"""
from __future__ import annotations

import os
from datetime import timedelta


class Replicas:
    """Rank bookkeeping for torchrun-style launches (RANK, WORLD_SIZE, LOCAL_RANK,
    MASTER_ADDR/PORT in the environment). `backend` is "nccl" on GPUs, "gloo" on CPU."""

    def __init__(self, backend: str = "nccl", timeout_s: float = 300.0, env=None):
        env = os.environ if env is None else env
        self.rank = int(env.get("RANK", "0"))
        self.world = int(env.get("WORLD_SIZE", "1"))
        self.local = int(env.get("LOCAL_RANK", "0"))
        self.backend = backend
        self.dist = None
        if self.world > 1:
            import torch.distributed as dist

            if not dist.is_initialized():
                dist.init_process_group(backend, timeout=timedelta(seconds=timeout_s))
            self.dist = dist

    @property
    def device(self) -> str:
        return "cuda" if self.backend == "nccl" else "cpu"

    def max_over_ranks(self, x: float) -> float:
        if self.dist is None:
            return float(x)
        import torch

        t = torch.tensor([float(x)], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def sum_over_ranks(self, x: float) -> float:
        if self.dist is None:
            return float(x)
        import torch

        t = torch.tensor([float(x)], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM)
        return float(t.item())

    def barrier(self):
        if self.dist is not None:
            if self.backend == "nccl":
                import torch

                self.dist.barrier(device_ids=[torch.cuda.current_device()])
            else:
                self.dist.barrier()
        if self.backend == "nccl":
            import torch

            torch.cuda.synchronize()

    def share(self, items):
        """This rank's share of a stream of independent items (round robin)."""
        return list(items)[self.rank::self.world]

    def close(self):
        if self.dist is not None and self.dist.is_initialized():
            self.dist.destroy_process_group()
        self.dist = None
