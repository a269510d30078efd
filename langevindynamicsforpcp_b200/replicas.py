"""Replicas over GPUs: one process per GPU, launched by torchrun.

Trajectories are independent and the reference's only cross-rank traffic is
an end-of-run reduction of a few KB (MPIKernel, src/mpiKernel.cpp), so N GPUs
run N replicas: each rank integrates its own trajectories (job ids offset by
rank, so the Philox streams differ), nothing is exchanged on the data path,
and a timing is the maximum over ranks.  RANK, WORLD_SIZE and LOCAL_RANK come
from the launcher's environment; rendezvous on MASTER_ADDR / MASTER_PORT.
"""
from __future__ import annotations

import os
from datetime import timedelta

JOB_ID_STRIDE = 1000   # job ids of rank r: r * JOB_ID_STRIDE + job index


class Replicas:
    def __init__(self, backend: str = "nccl", timeout_s: float = 120.0):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local_rank = int(os.environ.get("LOCAL_RANK", str(self.rank)))
        self.backend = backend
        self.dist = None
        if self.world > 1:
            import torch.distributed as dist
            dist.init_process_group(backend, timeout=timedelta(seconds=timeout_s))
            self.dist = dist

    @property
    def job_id_base(self) -> int:
        return self.rank * JOB_ID_STRIDE

    def barrier(self) -> None:
        if self.dist:
            self.dist.barrier()

    def max_over_ranks(self, value: float) -> float:
        """The maximum of value over all ranks (the step time of the job)."""
        if not self.dist:
            return value
        import torch
        dev = f"cuda:{self.local_rank}" if self.backend == "nccl" else "cpu"
        t = torch.tensor([value], dtype=torch.float64, device=dev)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def close(self) -> None:
        if self.dist:
            self.dist.destroy_process_group()
            self.dist = None
