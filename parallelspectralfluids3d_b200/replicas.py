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


def gather_objects(obj):
    """Every rank's ``obj`` in rank order (host-side; ``[obj]`` when not distributed)."""
    import torch.distributed as td

    if not (td.is_available() and td.is_initialized()) or td.get_world_size() == 1:
        return [obj]
    out = [None] * td.get_world_size()
    td.all_gather_object(out, obj)
    return out


def combine_serving(records):
    """Whole-job serving figures from every rank's completions.

    Each record holds the rank's ``requests`` (request indices it completed),
    ``latencies`` (seconds), ``steps`` (instance-steps completed) and the
    ``first`` submission / ``last`` completion times on the host's monotonic
    clock, which all processes on a node share.  The job's rate is all
    instance-steps over the span from the first submission to the last
    completion on any rank.
    """
    import numpy as np

    done = [i for r in records for i in r["requests"]]
    if len(done) != len(set(done)):
        raise RuntimeError("a request was completed by more than one rank")
    lat = np.array([x for r in records for x in r["latencies"]], dtype=np.float64)
    steps = sum(int(r["steps"]) for r in records)
    first = min(r["first"] for r in records)
    last = max(r["last"] for r in records)
    return {"completed": len(done), "requests": sorted(done), "instance_steps": steps,
            "instance_steps_per_s": steps / max(last - first, 1e-12), "span_s": last - first,
            "p50_latency_s": float(np.percentile(lat, 50)) if lat.size else None,
            "p99_latency_s": float(np.percentile(lat, 99)) if lat.size else None,
            "per_rank_completed": [len(r["requests"]) for r in records]}
