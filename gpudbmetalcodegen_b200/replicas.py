"""Replica plumbing for `bench.py --gpus N` (one process per GPU).

The hot path does not shard: every rank runs the same query on its own GPU
over its own copy of the tables, with no collective on the data path. The
ranks only meet to start the timed region together (a barrier) and to
report the slowest rank's time (an all-reduce MAX), so the printed
throughput is the whole job's rows over the slowest replica's time.
"""
from __future__ import annotations

import datetime
import os
from typing import Optional, Sequence, Tuple


def dist_info() -> Tuple[int, int, int]:
    """(world size, rank, local rank) from the launcher's environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str = "nccl", timeout_s: float = 300.0):
    """The process group of a multi-rank run, or None for one rank. A short
    timeout makes ranks that wait on a missing peer fail instead of hang."""
    world, _, _ = dist_info()
    if world <= 1:
        return None
    import torch.distributed as dist
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return dist


def barrier(pg) -> None:
    if pg is not None:
        pg.barrier()


def max_over_ranks(pg, values: Sequence[float], device: Optional[str] = None) -> list:
    """Element-wise maximum of `values` over all ranks (every rank gets it).
    `device` is where the reduction tensor lives: "cuda" for NCCL, "cpu"
    for gloo."""
    vals = [float(v) for v in values]
    if pg is None:
        return vals
    import torch
    dev = device or ("cuda" if pg.get_backend() == "nccl" else "cpu")
    t = torch.tensor(vals, dtype=torch.float64, device=dev)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return [float(x) for x in t.tolist()]


def shutdown(pg) -> None:
    if pg is not None:
        pg.destroy_process_group()
