"""Replica runs: one process per GPU, each running its own VMC.

The reference has no multi-device path (its VMC runs on one device), and one VMC step does not
shard across GPUs without an all-reduce of a P-vector per CG iteration, so several GPUs run
independent replicas: every rank builds its own chains and network from ``replica_seed(seed,
rank)`` and steps them with no collective on the data path.  The only collectives are on the
measurement side: a barrier before the timed region and the maximum over ranks of the timed
device milliseconds, from which the whole-job throughput (all ranks' samples over the slowest
rank's time) is formed.  These helpers take the process group's backend into account (NCCL
reduces a device tensor, gloo a host tensor), so the same code runs under ``torchrun`` on GPUs and
in multi-process CPU tests.
"""

from __future__ import annotations

import datetime
import os


def rank_env():
    """(rank, world_size, local_rank) from the launcher's environment (1 process: (0, 1, 0))."""
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("LOCAL_RANK", "0"))


def replica_seed(seed: int, rank: int) -> int:
    """Seed of rank `rank`'s replica: distinct chains, sampler streams and initial parameters."""
    return int(seed) + int(rank)


def init_group(world: int, backend: str = "nccl", timeout_s: float = 120.0):
    """The default process group when world > 1 (else None), with a short timeout so that ranks
    waiting for a rank that has gone end with an error."""
    if world <= 1:
        return None
    import torch.distributed as dist
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return dist


def _device(dist):
    return "cuda" if dist.get_backend() == "nccl" else "cpu"


def max_over_ranks(x: float, dist=None) -> float:
    """max of x over all ranks (x itself without a process group)."""
    if dist is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=_device(dist))
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(units_per_rank_step: float, steps: int, total_ms: float, world: int) -> float:
    """Whole-job units per second: every rank processed units_per_rank_step per step for `steps`
    steps; total_ms is the slowest rank's timed device milliseconds (max over ranks)."""
    if total_ms <= 0:
        raise ValueError("total_ms must be positive")
    return float(world) * float(units_per_rank_step) * int(steps) / (float(total_ms) / 1e3)


def finish(dist=None):
    """Barrier, then tear the process group down (every rank takes the same steps)."""
    if dist is None:
        return
    dist.barrier()
    dist.destroy_process_group()
