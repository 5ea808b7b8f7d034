"""Multi-GPU layout of the solve: replicas only.

Instances (wavelength x polarisation x geometry) are independent, which is
the reference's own parallelism (one process per wavelength, main.cpp:27-36).
Each rank (one process per GPU) solves its own instances with no data-path
collective; the only cross-rank traffic is the barrier and the max-over-ranks
of the timed interval, so throughput = all ranks' instances / the slowest
rank's time.  These helpers are the host-side logic of that layout; they run
with any torch.distributed backend (NCCL on the GPUs, gloo in the CPU tests).
"""
from __future__ import annotations


def replica_wavelength(base_nm: float, rank: int, step_nm: float = 5.0) -> float:
    """Wavelength solved by `rank` when every rank solves one replica of the
    same geometry: the base wavelength shifted by `step_nm` per rank."""
    return float(base_nm) + step_nm * int(rank)


def shard(items, rank: int, world: int):
    """The instances of a batch that `rank` solves: round-robin, so uneven
    grid sizes spread over the ranks."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank must be in [0, world)")
    return list(items)[rank::world]


def max_over_ranks(value: float, device=None) -> float:
    """The largest `value` over all ranks (the job's time is the slowest
    rank's); the value itself when no process group is initialised."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float, device=None) -> float:
    """The sum of `value` over all ranks (the value itself without a group)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def throughput(units_local: float, ms_local: float, device=None) -> tuple[float, float]:
    """(whole-job units/s, slowest rank's ms): the units of all ranks over the
    slowest rank's time (ranks may hold uneven shares)."""
    units = sum_over_ranks(units_local, device)
    ms_max = max_over_ranks(ms_local, device)
    return units * 1e3 / ms_max, ms_max
