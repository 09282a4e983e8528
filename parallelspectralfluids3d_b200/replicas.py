"""Multi-GPU layout: independent replicas, one process per GPU.

Rollouts are independent and a step has no exchange between them, so N GPUs
run N replicas of the engine with no collective inside the step.  The only
communication is host-side bookkeeping around a measurement: splitting the
instances (or requests) between ranks and combining the ranks' device times
(the slowest rank defines the job's time).  The reference has no multi-GPU
path at all (it drives one OpenCL queue, Solver/SolverImpl/psfsolvergpu.cpp).
"""

from __future__ import annotations


def shard(items, rank: int, world: int):
    """Items of one rank: round-robin over ranks, so uneven items spread evenly."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside world of size {world}")
    return [x for i, x in enumerate(items) if i % world == rank]


def slowest(values, device=None):
    """Element-wise maximum over ranks of a list of floats (identity when not distributed)."""
    import torch
    import torch.distributed as td

    vals = [float(v) for v in values]
    if not (td.is_available() and td.is_initialized()) or td.get_world_size() == 1:
        return vals
    t = torch.tensor(vals, dtype=torch.float64, device=device)
    td.all_reduce(t, op=td.ReduceOp.MAX)
    return [float(x) for x in t.cpu().tolist()]


def job_rate(units_per_rank: int, ms_per_rank: float, device=None) -> float:
    """Whole-job rate (units/s): all ranks' units over the slowest rank's time."""
    import torch.distributed as td

    world = td.get_world_size() if td.is_available() and td.is_initialized() else 1
    (ms,) = slowest([ms_per_rank], device=device)
    return world * units_per_rank / (ms / 1e3)
