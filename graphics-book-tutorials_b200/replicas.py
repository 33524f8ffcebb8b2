"""Replica group for multi-GPU runs: one process per GPU, launched by torchrun.

The path tracer has no cross-GPU exchange: every (pixel, sample) path is independent and every
job owns its film, so N GPUs run N replicas (each holds its own resident scene and renders its
own work) and only scalars cross ranks -- a barrier around the timed region and the max over
ranks of the device time, as the whole-job figure. No data-path collective, no peer memory.

The backend is NCCL on GPUs and gloo on CPU (multi-process tests); a single process (no
WORLD_SIZE in the environment, or 1) gets a no-op group.
"""
import datetime
import os


class ReplicaGroup:
    def __init__(self, backend: str = "nccl", timeout_s: float = 120.0, device=None):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local_rank = int(os.environ.get("LOCAL_RANK", "0"))
        self.backend = backend
        self.device = device
        self._dist = None
        if self.world > 1:
            import torch.distributed as dist
            os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
            self._dist = dist

    @property
    def active(self) -> bool:
        return self._dist is not None

    def _tensor(self, x: float):
        import torch
        dev = self.device if self.device is not None else ("cuda" if self.backend == "nccl" else "cpu")
        return torch.tensor([float(x)], dtype=torch.float64, device=dev)

    def barrier(self) -> None:
        if self._dist is not None:
            self._dist.barrier()

    def max(self, x: float) -> float:
        """Max over ranks (every rank gets it); the identity in a single process."""
        if self._dist is None:
            return float(x)
        t = self._tensor(x)
        self._dist.all_reduce(t, op=self._dist.ReduceOp.MAX)
        return float(t.item())

    def sum(self, x: float) -> float:
        if self._dist is None:
            return float(x)
        t = self._tensor(x)
        self._dist.all_reduce(t, op=self._dist.ReduceOp.SUM)
        return float(t.item())

    def close(self) -> None:
        if self._dist is not None:
            self._dist.destroy_process_group()
            self._dist = None


def whole_job_rate(units_per_rank: float, steps: int, world: int, max_seconds: float) -> float:
    """Units per second of the whole job: every rank processed units_per_rank per step, and the job
    took as long as its slowest rank (max over ranks of the device time)."""
    if max_seconds <= 0.0:
        raise ValueError("max_seconds must be positive")
    return units_per_rank * steps * world / max_seconds
