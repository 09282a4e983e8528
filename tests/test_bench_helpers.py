"""Host-side helpers of bench.py that its numbers rely on (no GPU).

* The serving request stream: only the arrival times depend on the rate, so
  runs at 200 and 2000 requests/s serve the same requests (the serving form
  reuses one plain-path sample and one set of FP64 references for both).
* Slot assignment of batched workloads and the per-rank sharding of instances.
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import bench  # noqa: E402
from parallelspectralfluids3d_b200 import replicas  # noqa: E402


def _params(reqs):
    return [(q["basis"], q["n"], q["steps"], q["P"], q["seed"]) for q in reqs]


def test_request_stream_depends_on_the_rate_only_through_arrival_times():
    slow = bench.serve_requests(60.0, rate=200.0, seed=7)
    fast = bench.serve_requests(6.0, rate=2000.0, seed=7)
    k = min(len(slow), len(fast))
    assert k > 10000
    assert _params(slow[:k]) == _params(fast[:k])
    t_slow = np.array([q["t"] for q in slow[:k]])
    t_fast = np.array([q["t"] for q in fast[:k]])
    np.testing.assert_allclose(t_fast * 10.0, t_slow, rtol=1e-12)


def test_request_stream_follows_the_configured_distributions():
    reqs = bench.serve_requests(60.0, rate=200.0, seed=7)
    assert 11000 < len(reqs) < 13000  # Poisson(200/s) over 60 s
    n = np.array([q["n"] for q in reqs])
    steps = np.array([q["steps"] for q in reqs])
    P = np.array([q["P"] for q in reqs])
    assert n.min() >= 64 and n.max() <= 384
    assert steps.min() >= 50 and steps.max() <= 1000
    assert P.min() >= 10_000 and P.max() <= 1_000_000
    assert 1.8e5 < P.mean() < 2.5e5  # log-uniform on [1e4, 1e6]: mean 2.15e5
    assert set(q["basis"] for q in reqs) == {0, 1, 2}


def test_assign_slots_numbers_instances_per_basis():
    insts = [{"basis": b} for b in (0, 1, 0, 2, 0, 1)]
    counts = bench.assign_slots(insts, 3)
    assert counts == [3, 2, 1]
    assert [x["slot"] for x in insts] == [0, 0, 1, 0, 2, 1]
    assert bench.assign_slots([], 2) == [1, 1]


def test_shards_cover_every_instance_once():
    items = list(range(517))
    shards = [replicas.shard(items, r, 4) for r in range(4)]
    assert sorted(x for s in shards for x in s) == items
    assert max(len(s) for s in shards) - min(len(s) for s in shards) <= 1
