"""Replicas across GPUs: one process per GPU, each dedispersing its own chunks.

astroflow's dedispersion runs one chunk on one GPU (`target_id`,
src/core/dedispered.cu:997-1001) and independent chunks or beams need no
exchange, so multi-GPU use is replicas only: no data-path collective.  The
process group exists for the job's bookkeeping: a barrier around timed
regions, the slowest rank's time (max over ranks) and the whole job's
throughput.  Ranks come from the launcher's environment (RANK, LOCAL_RANK,
WORLD_SIZE, MASTER_ADDR, MASTER_PORT; torchrun sets them).
"""
from __future__ import annotations

import datetime
import os


class Replicas:
    def __init__(self, backend: str = "nccl", timeout_s: float = 300.0):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", str(self.rank)))
        self.backend = backend
        self.pg = None
        if self.world > 1:
            import torch.distributed as dist

            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
            self.pg = dist

    @property
    def device(self) -> str:
        return f"cuda:{self.local}" if self.backend == "nccl" else "cpu"

    def chunk_seed(self, base: int) -> int:
        """Each rank works on its own chunk."""
        return base + self.rank

    def barrier(self) -> None:
        if self.pg:
            if self.backend == "nccl":
                self.pg.barrier(device_ids=[self.local])
            else:
                self.pg.barrier()

    def _reduce(self, v: float, op) -> float:
        if not self.pg:
            return v
        import torch

        t = torch.tensor([v], dtype=torch.float64, device=self.device)
        self.pg.all_reduce(t, op=op)
        return float(t.item())

    def max(self, v: float) -> float:
        """The largest value over ranks (the slowest rank's time)."""
        return self._reduce(v, self.pg.ReduceOp.MAX if self.pg else None)

    def sum(self, v: float) -> float:
        return self._reduce(v, self.pg.ReduceOp.SUM if self.pg else None)

    def job_rate(self, units_per_rank: float, seconds_per_rank: float) -> float:
        """Whole-job throughput: the units all ranks processed over the slowest rank's time."""
        return self.sum(units_per_rank) / self.max(seconds_per_rank)

    def close(self) -> None:
        if self.pg:
            self.pg.destroy_process_group()
            self.pg = None
