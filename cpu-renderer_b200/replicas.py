"""Replicated rendering over N processes, one per GPU (the torchrun environment).

Camera samples are independent of each other and the scene is read-only, so each rank renders
its own replica of the workload with its own sample streams (seed + rank) and nothing crosses
between ranks on the data path. The only collectives are the barriers that bracket a timed
region and one max-reduction of each rank's time: a whole-job rate is the samples all ranks
rendered over the slowest rank's time.

The process group gets a short timeout, so a rank that never arrives (it failed, or exited
early) ends the others' next collective with an error instead of a hang.
"""
import os
from datetime import timedelta


def dist_env():
    """(rank, world size, local rank) from the launcher's environment (1 process: 0, 1, 0)."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class Replicas:
    """The ranks of one replicated run. backend "nccl" (one GPU per rank, reductions on the
    device) or "gloo" (host tensors; the CPU tests of this plumbing)."""

    def __init__(self, backend="nccl", device=None, timeout_s=120):
        self.rank, self.world, self.local = dist_env()
        self.backend = backend
        self.device = device
        self.distributed = self.world > 1
        if self.distributed:
            import torch.distributed as dist
            kw = {"device_id": device} if backend == "nccl" and device is not None else {}
            dist.init_process_group(backend, timeout=timedelta(seconds=timeout_s), **kw)

    def seed(self, base):
        """The sample-stream seed of this rank's replica."""
        return base + self.rank

    def _sync_device(self):
        if self.device is not None and getattr(self.device, "type", None) == "cuda":
            import torch
            torch.cuda.synchronize(self.device)

    def barrier(self):
        """Every rank's queued device work is done and every rank has arrived."""
        self._sync_device()
        if self.distributed:
            import torch.distributed as dist
            dist.barrier()

    def max_over_ranks(self, x):
        """The largest of the ranks' values of x (a time: the slowest rank's)."""
        import torch
        on_device = self.backend == "nccl" and self.device is not None
        t = torch.tensor([float(x)], dtype=torch.float64, device=self.device if on_device else "cpu")
        if self.distributed:
            import torch.distributed as dist
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def whole_job_rate(self, units_per_rank, seconds, scale=1e-6):
        """Units all ranks processed per second of the slowest rank (scaled, default to millions)."""
        slowest = self.max_over_ranks(seconds)
        if not slowest > 0:
            raise ValueError("the slowest rank's time must be positive")
        return self.world * units_per_rank / slowest * scale

    def close(self):
        if self.distributed:
            import torch.distributed as dist
            dist.barrier()
            dist.destroy_process_group()
            self.distributed = False
