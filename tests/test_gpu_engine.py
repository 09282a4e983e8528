"""Serving engine (include/psf_engine.h): continuous batching of rollouts.

Requests are submitted from another thread while earlier ones run, with
fewer slots than requests so that admission waits for slots to free up.  Each
result must match the FP64 oracle (the batched path's tolerances: relative
L2 error of w <= 1e-4, particles within 2e-3 voxel) and must be the same
alone as in the mix (within 1e-12 relative; the products of one rollout do
not depend on the other columns of the batch).
"""
import threading
import time

import numpy as np
import pytest

from oracle import oracle as O
from parallelspectralfluids3d_b200 import _lib as L
from parallelspectralfluids3d_b200.engine import Engine
from parallelspectralfluids3d_b200.fixture import initial_coefficients, initial_particles

from conftest import rel_err

pytestmark = pytest.mark.gpu

W_TOL = 1e-4
P_TOL_VOX = 2e-3
MIX_TOL = 1e-12

# (basis index, n_modes, steps, particles, seed, dt, integrator)
REQS = [
    (0, 37, 23, 300, 1, 0.02, L.PSF_RK4),
    (1, 13, 9, 128, 2, 0.04, L.PSF_RK1),
    (0, 20, 14, 700, 3, 0.03, L.PSF_RK4),
    (0, 37, 5, 0, 4, 0.02, L.PSF_RK4),
    (1, 8, 30, 512, 5, 0.02, L.PSF_RK4),
    (0, 11, 17, 256, 6, 0.05, L.PSF_RK1),
    (1, 13, 12, 999, 7, 0.01, L.PSF_RK4),
]


def _inputs(bases, q):
    g, n, steps, P, seed, dt, integ = q
    w0 = initial_coefficients(n, seed)
    parts = initial_particles(bases[g], P, seed + 70) if P else None
    params = L.make_params(dt=dt, integrator=integ, seed=seed, precision=L.PSF_PRECISION_BF16X2)
    return w0, parts, params


def _submit(engine, bases, q):
    w0, parts, params = _inputs(bases, q)
    return engine.submit(q[0], w0, q[2], params, particles=parts)


def _oracle(bases, q):
    g, n, steps, P, seed, dt, integ = q
    w0, parts, _ = _inputs(bases, q)
    return O.OracleRollout(bases[g].truncate(n), w0, parts, dt=dt, integrator=integ, seed=seed).step(steps)


@pytest.fixture(scope="module")
def bases(small_bases):
    return [small_bases["sphere12x10x9"], small_bases["box576"]]


def test_engine_continuous_batching_matches_oracle_and_alone(bases):
    with Engine(bases, slots=[2, 2], max_particles=1024, chunk_steps=4) as eng:
        ids = [None] * len(REQS)

        def producer():
            # Five at once (more than the four slots), the rest while those run.
            for i, q in enumerate(REQS):
                ids[i] = _submit(eng, bases, q)
                if i >= 4:
                    time.sleep(0.003)

        th = threading.Thread(target=producer)
        th.start()
        th.join()
        eng.drain(120)
        results = [eng.collect(rid) for rid in ids]
        st = eng.stats()
    assert st["completed"] == len(REQS)
    assert st["instance_steps"] == sum(q[2] for q in REQS)
    assert st["budget_refusals"] > 0  # more requests than slots: some had to wait
    for q, (w, p, info) in zip(REQS, results):
        assert info["status"] == 0 and info["t_submit"] <= info["t_admit"] <= info["t_done"]
        ref = _oracle(bases, q)
        assert rel_err(w, ref.w) <= W_TOL, q
        if q[3]:
            assert np.abs(p[:, :3] - ref.pos).max() / bases[q[0]].h <= P_TOL_VOX, q
    # The same requests alone in an engine of their own.
    for i in (0, 4):
        with Engine(bases, slots=[1, 1], max_particles=1024, chunk_steps=4) as eng:
            rid = _submit(eng, bases, REQS[i])
            assert eng.wait(rid, 60)
            w, p, _ = eng.collect(rid)
        assert rel_err(w, results[i][0]) <= MIX_TOL
        assert np.abs(p[:, :3] - results[i][1][:, :3]).max() <= MIX_TOL
        assert np.array_equal(p[:, 3], results[i][1][:, 3])


def test_engine_staged_and_unstaged_placements_match_alone(bases):
    # Six full-size requests picked in one round: the pinned staging holds
    # four of them, the other two are placed from their own copies.  Each
    # rollout retires while others still run, read beside the running chunk.
    qs = [(g, (20 + 3 * i) if g == 0 else (8 + i), 6 + 3 * i, 1024, 20 + i, 0.02, L.PSF_RK4)
          for i, g in enumerate((0, 1, 0, 1, 0, 1))]
    with Engine(bases, slots=[3, 3], max_particles=1024, chunk_steps=4) as eng:
        ids = [_submit(eng, bases, q) for q in qs]
        eng.drain(120)
        results = [eng.collect(rid) for rid in ids]
    for i, q in enumerate(qs):
        w, p, info = results[i]
        assert info["status"] == 0
        with Engine(bases, slots=[1, 1], max_particles=1024, chunk_steps=4) as eng:
            rid = _submit(eng, bases, q)
            assert eng.wait(rid, 60)
            w1, p1, _ = eng.collect(rid)
        assert rel_err(w, w1) <= MIX_TOL, q
        assert np.abs(p[:, :3] - p1[:, :3]).max() <= MIX_TOL, q
        assert np.array_equal(p[:, 3], p1[:, 3]), q
    ref = _oracle(bases, qs[0])
    assert rel_err(results[0][0], ref.w) <= W_TOL
    assert np.abs(results[0][1][:, :3] - ref.pos).max() / bases[0].h <= P_TOL_VOX


def test_engine_budget_admits_one_rollout_at_a_time(bases):
    qs = [(0, 37, 6, 300, s, 0.02, L.PSF_RK4) for s in range(4)]
    one = 300 * 20 + 24 * int(np.prod(bases[0].dims)) + 16 * bases[0].n_modes
    with Engine(bases, slots=[4, 1], max_particles=1024, hbm_budget_bytes=int(1.5 * one), chunk_steps=2) as eng:
        ids = [_submit(eng, bases, q) for q in qs]
        eng.drain(60)
        infos = [eng.collect(r)[2] for r in ids]
        st = eng.stats()
    infos.sort(key=lambda x: x["t_admit"])
    for a, b in zip(infos, infos[1:]):
        assert b["t_admit"] >= a["t_done"] - 1e-9
    assert st["budget_refusals"] > 0 and st["rollout_bytes"] == 0


def test_engine_rejects_requests_it_can_never_run(bases):
    with Engine(bases, slots=[1, 1], max_particles=100, chunk_steps=2) as eng:
        p = L.make_params(dt=0.01)
        with pytest.raises(L.PSFError):
            eng.submit(2, np.ones(4), 5, p)  # unknown basis
        with pytest.raises(L.PSFError):
            eng.submit(1, np.ones(bases[1].n_modes + 1), 5, p)  # too many modes
        with pytest.raises(L.PSFError):
            eng.submit(0, np.ones(4), 5, p, particles=np.zeros((101, 4), np.float32))  # too many particles
        with pytest.raises(L.PSFError):
            eng.submit(0, np.ones(4), 0, p)  # no steps
