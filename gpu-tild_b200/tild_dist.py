"""Multi-GPU plumbing for replicas and ensembles: one process per GPU, no data-path collective.

Independent systems never exchange anything (a single system's FFT stays on one GPU), so the
only cross-rank traffic is timing and result bookkeeping: a barrier around the timed region, the
maximum of the per-rank times, and sums of processed particle-steps.  torch.distributed is the
plumbing (NCCL between GPUs, gloo on CPU for tests).
"""
from __future__ import annotations

import os
from datetime import timedelta
from typing import List, Sequence


def shard(sizes: Sequence[int], rank: int, world: int) -> List[int]:
    """Indices of the systems this rank runs: greedy longest-processing-time assignment by size
    (deterministic: ties broken by index), so every rank gets a near-equal particle count."""
    order = sorted(range(len(sizes)), key=lambda i: (-int(sizes[i]), i))
    load = [0] * world
    owner = [0] * len(sizes)
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        owner[i] = r
        load[r] += int(sizes[i])
    return [i for i in range(len(sizes)) if owner[i] == rank]


class Group:
    """Process-group wrapper used by bench.py; a no-op for a single process."""

    def __init__(self, backend: str = "nccl", timeout_s: int = 120):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", str(self.rank)))
        self.dist = None
        self.device = None
        if self.world > 1:
            import torch
            import torch.distributed as dist
            if backend == "nccl":
                torch.cuda.set_device(self.local)
                self.device = torch.device("cuda", self.local)
            else:
                self.device = torch.device("cpu")
            dist.init_process_group(backend, timeout=timedelta(seconds=timeout_s))
            self.dist = dist

    def barrier(self):
        if self.dist is not None:
            self.dist.barrier()

    def _reduce(self, v: float, op) -> float:
        if self.dist is None:
            return v
        import torch
        t = torch.tensor([float(v)], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=op)
        return float(t.item())

    def max(self, v: float) -> float:
        return self._reduce(v, None if self.dist is None else self.dist.ReduceOp.MAX)

    def sum(self, v: float) -> float:
        return self._reduce(v, None if self.dist is None else self.dist.ReduceOp.SUM)

    def gather_lists(self, items: list) -> list:
        """Concatenation of every rank's list (all ranks receive it)."""
        if self.dist is None:
            return list(items)
        out = [None] * self.world
        self.dist.all_gather_object(out, list(items))
        return [x for part in out for x in part]

    def close(self):
        if self.dist is not None:
            self.dist.destroy_process_group()
            self.dist = None
