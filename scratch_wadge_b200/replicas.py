"""Multi-GPU runs as independent replicas: one process per GPU, each running
its own solve (the reference's time step exchanges no data within a rank,
rk_step in euler.c:3610-3670, and this path is single-rank by design), so
ranks only agree on choices and combine timings:

* ``init``            — the process group over the launcher's environment
                        (RANK, WORLD_SIZE, LOCAL_RANK, MASTER_*) with a short
                        timeout, or None for a single process;
* ``agree``           — every rank takes the same boolean choice (true if any
                        rank proposes true), so all ranks run the same kernels;
* ``all_max``         — the slowest rank's time (whole-job time);
* ``job_throughput``  — units all ranks processed / whole-job time.

Every rank calls these in the same order (they are collectives).  The
collectives run on CUDA tensors over NCCL, or on CPU tensors over gloo.
"""

from __future__ import annotations

import datetime
import os


def env():
    """(world_size, rank, local_rank) from the launcher's environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str = "nccl", timeout_s: float = 120.0):
    ws, _, _ = env()
    if ws <= 1:
        return None
    import torch.distributed as dist
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return dist


def _device(pg):
    return "cuda" if pg.get_backend() == "nccl" else "cpu"


def all_max(pg, x: float) -> float:
    if pg is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=_device(pg))
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def agree(pg, flag: bool) -> bool:
    return all_max(pg, 1.0 if flag else 0.0) > 0.0


def job_throughput(world_size: int, units_per_rank: float, seconds_max: float) -> float:
    """weak scaling: every rank processes units_per_rank in at most seconds_max"""
    return world_size * units_per_rank / seconds_max


def finish(pg):
    if pg is not None:
        pg.barrier()
        pg.destroy_process_group()
