"""Parity at the configurations' large mode counts and particle loads.

N = 256 and N = 384 are the tile shapes of the precision and serving
configurations (256 is two 128-row MMA tiles and four 64-wide K chunks; 384
is three of each, and three 128-column chunks in the plain contraction).
They run here on a 14^3 box, whose basis the GPU precompute builds in
seconds, against the FP64 oracle on the same basis (psfsolver.cpp:34-224).
The batched tracer also runs at the 32^3 + sphere size with 262,144
particles per instance, where a step's particles no longer sit in a few
warps' worth of cells.  Bars as in test_gpu_parity.py (plain FP32) and
test_gpu_batch.py (BF16 hi/lo).
"""
import numpy as np
import pytest

from oracle import oracle as O
from parallelspectralfluids3d_b200 import _lib as L
from parallelspectralfluids3d_b200.batch import Batch
from parallelspectralfluids3d_b200.domain import box_domain, sphere_obstacle_domain
from parallelspectralfluids3d_b200.fixture import initial_coefficients, initial_particles

from conftest import rel_err
from test_gpu_parity import P_TOL_VOX, W_TOL, run_pair

pytestmark = pytest.mark.gpu

BATCH_W_TOL = 1e-4
BATCH_P_TOL_VOX = 2e-3


@pytest.fixture(scope="session")
def box14_n384(make_basis):
    return make_basis(box_domain(14), 384)


@pytest.mark.parametrize("n", [256, 384])
def test_plain_path_at_large_mode_counts(box14_n384, n):
    b = box14_n384.truncate(n)
    ctx, ref = run_pair(b, 50, dt=0.005, P=2048, seed_w=n, seed_p=n + 1)
    assert rel_err(ctx.get_state(), ref.w) <= W_TOL
    assert np.abs(ctx.get_particles()[:, :3] - ref.pos).max() / b.h <= P_TOL_VOX


def test_batched_path_at_large_mode_counts(box14_n384):
    b = box14_n384
    specs = [(0, 384, 11), (1, 256, 12), (2, 300, 13), (3, 256, 14)]  # (slot, N, seed)
    steps, dt = 40, 0.005
    params = {s: L.make_params(dt=dt, integrator=L.PSF_RK4, seed=seed, precision=L.PSF_PRECISION_BF16X2)
              for s, _, seed in specs}
    with Batch([b], slots=4, max_particles=2048) as batch:
        for slot, n, seed in specs:
            batch.set_instance(0, slot, initial_coefficients(n, seed), params[slot],
                               particles=initial_particles(b, 2048, seed + 100))
        batch.step(steps)
        batch.sync()
        assert batch.device_status() == 0
        for slot, n, seed in specs:
            ref = O.OracleRollout(b.truncate(n), initial_coefficients(n, seed), initial_particles(b, 2048, seed + 100),
                                  dt=dt, integrator=4, seed=seed).step(steps)
            assert rel_err(batch.get_state(0, slot), ref.w) <= BATCH_W_TOL, (slot, n)
            p = batch.get_particles(0, slot)
            assert np.abs(p[:, :3] - ref.pos).max() / b.h <= BATCH_P_TOL_VOX, (slot, n)


def test_batched_tracer_at_the_sphere32_size(make_basis):
    """Two instances of 262,144 particles each on the 32^3 + sphere r=8 basis (N = 128)."""
    b = make_basis(sphere_obstacle_domain(32, 8.0), 128)
    steps, dt, P = 20, 0.005, 262144
    with Batch([b], slots=2, max_particles=P) as batch:
        for slot in range(2):
            batch.set_instance(0, slot, initial_coefficients(128, 2 + slot),
                               L.make_params(dt=dt, integrator=L.PSF_RK4, seed=slot,
                                             precision=L.PSF_PRECISION_BF16X2),
                               particles=initial_particles(b, P, 3 + slot))
        batch.step(steps)
        batch.sync()
        for slot in range(2):
            ref = O.OracleRollout(b, initial_coefficients(128, 2 + slot), initial_particles(b, P, 3 + slot), dt=dt,
                                  integrator=4, seed=slot).step(steps)
            assert rel_err(batch.get_state(0, slot), ref.w) <= BATCH_W_TOL
            d = np.abs(batch.get_particles(0, slot)[:, :3] - ref.pos).max(axis=1) / b.h
            assert d.max() <= BATCH_P_TOL_VOX and np.percentile(d, 99) <= 1e-4
