"""Multi-GPU host logic on CPU: two gloo ranks (no GPU, no collective in a step)."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from parallelspectralfluids3d_b200 import replicas


def test_shard_covers_every_item_once():
    items = list(range(17))
    parts = [replicas.shard(items, r, 3) for r in range(3)]
    assert sorted(x for p in parts for x in p) == items
    assert max(len(p) for p in parts) - min(len(p) for p in parts) <= 1
    with pytest.raises(ValueError):
        replicas.shard(items, 3, 3)


def test_single_process_is_identity():
    assert replicas.slowest([1.5, 2.0]) == [1.5, 2.0]
    assert replicas.job_rate(100, 50.0) == pytest.approx(2000.0)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out):
    import datetime

    import torch.distributed as td

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    td.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=30))
    try:
        mine = replicas.shard(list(range(10)), rank, world)
        # Rank 1 is the slow one: the job's time is its time.
        ms = 40.0 if rank == 1 else 25.0
        rate = replicas.job_rate(len(mine), ms)
        both = replicas.slowest([ms, float(rank)])
        out.put((rank, mine, rate, both))
    finally:
        td.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_time():
    world = 2
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    res = [out.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    assert res[0][1] == [0, 2, 4, 6, 8] and res[1][1] == [1, 3, 5, 7, 9]
    for _, mine, rate, both in res:
        assert rate == pytest.approx(2 * 5 / 0.040)
        assert both == [40.0, 1.0]


def _serve_rank(rank, world, port, out):
    """A CPU stand-in for one rank's engine: it serves its round-robin share of a
    Poisson request stream (each request takes steps x 10 us) and rank 0
    combines every rank's completions."""
    import datetime
    import time

    import numpy as np
    import torch.distributed as td

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    td.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=30))
    try:
        rng = np.random.default_rng(7)
        arrivals = np.cumsum(rng.exponential(1 / 2000.0, 40))
        reqs = [dict(index=i, t=float(t), steps=int(rng.integers(50, 1001))) for i, t in enumerate(arrivals)]
        mine = replicas.shard(reqs, rank, world)
        t0 = time.monotonic()
        lat, first, last = [], None, None
        for q in mine:
            wait = q["t"] - (time.monotonic() - t0)
            if wait > 0:
                time.sleep(wait)
            submit = time.monotonic()
            time.sleep(q["steps"] * 1e-5)
            end = time.monotonic()
            first = submit if first is None else first
            last = end
            lat.append(end - submit)
        rec = {"requests": [q["index"] for q in mine], "latencies": lat, "steps": sum(q["steps"] for q in mine),
               "first": first, "last": last}
        recs = replicas.gather_objects(rec)
        job = replicas.combine_serving(recs)
        out.put((rank, job, sum(q["steps"] for q in reqs)))
    finally:
        td.destroy_process_group()


def test_two_gloo_ranks_serve_a_sharded_request_stream():
    world = 2
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_serve_rank, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    res = [out.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for _, job, total in res:
        assert job["requests"] == list(range(40))  # every request served once, by one rank
        assert job["per_rank_completed"] == [20, 20]
        assert job["instance_steps"] == total
        assert job["instance_steps_per_s"] == pytest.approx(total / job["span_s"])
        assert 0 < job["p50_latency_s"] <= job["p99_latency_s"]


def test_combine_serving_rejects_a_request_served_twice():
    recs = [{"requests": [0, 1], "latencies": [0.1, 0.2], "steps": 10, "first": 0.0, "last": 1.0},
            {"requests": [1], "latencies": [0.1], "steps": 5, "first": 0.5, "last": 2.0}]
    with pytest.raises(RuntimeError):
        replicas.combine_serving(recs)
