"""Replica runs on several GPUs of one node (``bench.py --gpus N``).

The hot path is replicated, not partitioned: every rank runs the same workload on its own
GPU, with no collective on the data path.  Ranks only meet to start their timed regions
together (a barrier) and to report one time for the job: the maximum over ranks of each
rank's device-timed seconds.  ``torch.distributed`` carries both, over NCCL between GPUs or
gloo on the host (the tests).
"""
from __future__ import annotations

import os

import torch


def rank_world():
    """(rank, local_rank, world_size) from the launcher's environment (1 process: 0, 0, 1)."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("LOCAL_RANK", "0")),
            int(os.environ.get("WORLD_SIZE", "1")))


def barrier(world):
    if world > 1:
        torch.distributed.barrier()


def max_over_ranks(values, world, device="cpu"):
    """Element-wise maximum over ranks of a list of floats (identity for one process)."""
    if world <= 1:
        return [float(v) for v in values]
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return t.tolist()
