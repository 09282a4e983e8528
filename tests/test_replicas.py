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
