"""Multi-GPU host logic: one process per GPU, independent work per rank.

The hot path has no data exchange between lattices, so N GPUs run N replicas (one
lattice each, or a share of a batch of independent lattices); the only collectives are the
barrier around the timed region and the max of the per-rank times.  The reference instead
splits one lattice over n_core_dims^4 MPI ranks with frozen block faces
(src/mpi/MpiTopology.cpp:7-24, src/geometry/GeometryCB.cpp:33-56).
"""
from __future__ import annotations

import os


def env_rank():
    """(rank, world_size, local_rank) from the launcher's environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str = "nccl", timeout_s: float = 300.0):
    """Initialise torch.distributed from the environment (no-op for one process).  Returns
    the torch.distributed module or None."""
    rank, world, local = env_rank()
    if world <= 1:
        return None
    import datetime

    import torch
    import torch.distributed as dist

    kw = {"timeout": datetime.timedelta(seconds=timeout_s)}
    if backend == "nccl":
        torch.cuda.set_device(local)
        kw["device_id"] = torch.device("cuda", local)
    dist.init_process_group(backend, **kw)
    return dist


def max_over_ranks(x: float, dist=None, device: str = "cpu") -> float:
    """The slowest rank's value (the timing rule for multi-GPU numbers)."""
    if dist is None:
        return float(x)
    import torch

    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x: float, dist=None, device: str = "cpu") -> float:
    if dist is None:
        return float(x)
    import torch

    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def replica_seed(base: int, rank: int) -> int:
    """Independent Philox key per replica (seed + 1000 * rank; the reference seeds each MPI
    rank with seed + rank, src/bin/gauge_hb_ncb.cpp:28)."""
    return int(base) + 1000 * int(rank)


def shard(costs, world: int):
    """Partition independent items (lattices, jobs) over `world` ranks by cost: largest
    first onto the least-loaded rank (LPT).  Returns a list of index lists, one per rank;
    deterministic for equal inputs."""
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    loads = [0.0] * world
    parts = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (loads[k], k))
        parts[r].append(i)
        loads[r] += costs[i]
    return [sorted(p) for p in parts]
