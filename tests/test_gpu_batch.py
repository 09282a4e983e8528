"""Batched BF16 hi/lo tensor-core path (include/psf_batch.h) against the FP64 oracle.

Every slot is checked against an FP64 rollout of the reference step on its
own prefix basis.  Tolerances for the compensated BF16 products (each operand
carries 16 significant bits, products accumulate in FP32): relative L2 error
of w <= 1e-4 (the bar stated for this form), particles within 2e-3 voxel,
face velocities within 1e-4 of max |u|.
"""
import numpy as np
import pytest

from oracle import oracle as O
from parallelspectralfluids3d_b200 import _lib as L
from parallelspectralfluids3d_b200.batch import Batch
from parallelspectralfluids3d_b200.fixture import initial_coefficients, initial_particles

from conftest import rel_err

pytestmark = pytest.mark.gpu

W_TOL = 1e-4
P_TOL_VOX = 2e-3
U_TOL = 1e-4

# (slot, n_modes, dt, flags, viscosity, integrator, particles, seed)
SPECS = [
    (0, 37, 0.02, L.PSF_FLAG_RENORM, 0.0, L.PSF_RK4, 300, 1),
    (1, 20, 0.03, L.PSF_FLAG_RENORM | L.PSF_FLAG_FORCING, 0.0, L.PSF_RK1, 500, 2),
    (2, 11, 0.05, L.PSF_FLAG_RENORM | L.PSF_FLAG_DECAY_NEG, 0.05, L.PSF_RK4, 257, 3),
    (4, 37, 0.01, 0, 0.0, L.PSF_RK4, 700, 4),
    (5, 30, 0.02, L.PSF_FLAG_RENORM, 0.02, L.PSF_RK1, 0, 5),
]


def _instance(b, spec):
    slot, n, dt, flags, visc, integ, P, seed = spec
    w0 = initial_coefficients(n, seed)
    parts = initial_particles(b, P, seed + 50) if P else None
    f = None
    if flags & L.PSF_FLAG_FORCING:
        f = np.zeros(n)
        f[0] = 0.1 / dt
    params = L.make_params(dt=dt, viscosity=visc, integrator=integ, flags=flags, seed=seed)
    return w0, parts, f, params


def _oracle(b, spec, steps):
    slot, n, dt, flags, visc, integ, P, seed = spec
    w0, parts, f, _ = _instance(b, spec)
    oflags = (O.FLAG_RENORM if flags & L.PSF_FLAG_RENORM else 0) | (
        O.FLAG_DECAY_NEG if flags & L.PSF_FLAG_DECAY_NEG else 0)
    return O.OracleRollout(b.truncate(n), w0, parts, dt=dt, viscosity=visc, flags=oflags, integrator=integ,
                           seed=seed, forcing=f).step(steps)


def _fill(batch, b, specs, basis=0):
    for spec in specs:
        w0, parts, f, params = _instance(b, spec)
        batch.set_instance(basis, spec[0], w0, params, particles=parts, forcing=f)


def test_batch_slots_match_oracle(small_bases):
    b = small_bases["sphere12x10x9"]
    steps = 20
    with Batch([b], slots=6, max_particles=1024) as batch:
        _fill(batch, b, SPECS)
        batch.step(steps)
        batch.sync()
        assert batch.device_status() == 0
        for spec in SPECS:
            ref = _oracle(b, spec, steps)
            w = batch.get_state(0, spec[0])
            assert rel_err(w, ref.w) <= W_TOL, (spec, rel_err(w, ref.w))
            if spec[6]:
                p = batch.get_particles(0, spec[0])
                err = np.abs(p[:, :3] - ref.pos).max() / b.h
                assert err <= P_TOL_VOX, (spec, err)
                assert np.array_equal(p[:, 3], ref.life)
            assert batch.get_steps(0, spec[0]) == steps


def test_batch_one_step_velocity_field(small_bases):
    b = small_bases["sphere12x10x9"]
    spec = SPECS[0]
    with Batch([b], slots=3, max_particles=512) as batch:
        _fill(batch, b, [spec])
        batch.step(1)
        u = batch.get_velocity(0, spec[0])
    ref = _oracle(b, spec, 1)
    assert np.abs(u - ref.u).max() <= U_TOL * np.abs(ref.u).max()
    mask = np.ones(b.n_faces, bool)
    mask[b.active_faces] = False
    assert np.all(u[mask] == 0)


def test_alone_equals_in_the_mix(small_bases):
    """A rollout gives the same result alone in a batch and among other rollouts."""
    b = small_bases["sphere12x10x9"]
    target = SPECS[0]
    results = []
    for others in ([], [s for s in SPECS if s[0] != target[0]]):
        with Batch([b], slots=6, max_particles=1024) as batch:
            _fill(batch, b, [target] + others)
            batch.step(15)
            results.append((batch.get_state(0, target[0]), batch.get_particles(0, target[0])))
    (w_a, p_a), (w_m, p_m) = results
    assert np.array_equal(w_a, w_m)
    assert np.array_equal(p_a, p_m)


@pytest.mark.parametrize("cols", [64, 128, 256])
def test_kernel_variants_agree(small_bases, cols):
    b = small_bases["sphere12x10x9"]
    outs = []
    for c in (0, cols):
        with Batch([b], slots=6, max_particles=1024, autotune=False, gemm_columns=c) as batch:
            _fill(batch, b, SPECS[:3])
            batch.step(10)
            outs.append(np.concatenate([batch.get_state(0, s[0]) for s in SPECS[:3]]))
    assert np.array_equal(outs[0], outs[1])


def test_two_bases_in_one_batch(small_bases):
    b1, b2 = small_bases["sphere12x10x9"], small_bases["box576"]
    s1 = (1, 25, 0.02, L.PSF_FLAG_RENORM, 0.0, L.PSF_RK4, 400, 7)
    s2 = (0, 13, 0.04, L.PSF_FLAG_RENORM, 0.0, L.PSF_RK4, 333, 8)
    with Batch([b1, b2], slots=[2, 3], max_particles=[512, 512]) as batch:
        _fill(batch, b1, [s1], basis=0)
        _fill(batch, b2, [s2], basis=1)
        batch.step(12)
        for bb, spec, gi in ((b1, s1, 0), (b2, s2, 1)):
            ref = _oracle(bb, spec, 12)
            assert rel_err(batch.get_state(gi, spec[0]), ref.w) <= W_TOL
            p = batch.get_particles(gi, spec[0])
            assert np.abs(p[:, :3] - ref.pos).max() / bb.h <= P_TOL_VOX


def test_clear_and_reuse_slot(small_bases):
    b = small_bases["sphere12x10x9"]
    with Batch([b], slots=2, max_particles=1024) as batch:
        _fill(batch, b, [SPECS[0]])
        batch.step(5)
        batch.clear_instance(0, 0)
        batch.step(3)  # empty batch steps are no-ops for the cleared slot
        spec = (0,) + SPECS[3][1:]
        _fill(batch, b, [spec])
        batch.step(10)
        ref = _oracle(b, spec, 10)
        assert rel_err(batch.get_state(0, 0), ref.w) <= W_TOL
        assert batch.get_steps(0, 0) == 10


def test_batch_argument_errors(small_bases):
    b = small_bases["box6"]
    with Batch([b], slots=2, max_particles=100) as batch:
        w0 = initial_coefficients(b.n_modes, 0)
        with pytest.raises(L.PSFError):
            batch.set_instance(0, 2, w0, L.make_params())  # slot out of range
        with pytest.raises(L.PSFError):
            batch.set_instance(0, 0, np.zeros(b.n_modes + 1), L.make_params())  # too many modes
        with pytest.raises(L.PSFError):
            batch.set_instance(0, 0, w0, L.make_params(), particles=np.zeros((300, 4), np.float32))
        with pytest.raises(L.PSFError):
            batch.get_state(0, 1)  # empty slot


def test_step_limit_freezes_a_slot(small_bases):
    """A slot with a step limit stops there while the others go on."""
    b = small_bases["sphere12x10x9"]
    spec_a, spec_b = SPECS[0], SPECS[3]
    with Batch([b], slots=6, max_particles=1024) as batch:
        w0, parts, f, params = _instance(b, spec_a)
        batch.set_instance(0, spec_a[0], w0, params, particles=parts, forcing=f, steps=7)
        _fill(batch, b, [spec_b])
        batch.step(12)
        assert batch.get_steps(0, spec_a[0]) == 7
        assert batch.get_steps(0, spec_b[0]) == 12
        ra, rb = _oracle(b, spec_a, 7), _oracle(b, spec_b, 12)
        assert rel_err(batch.get_state(0, spec_a[0]), ra.w) <= W_TOL
        assert np.abs(batch.get_particles(0, spec_a[0])[:, :3] - ra.pos).max() / b.h <= P_TOL_VOX
        assert rel_err(batch.get_state(0, spec_b[0]), rb.w) <= W_TOL


def test_particle_pool_admission(small_bases):
    """Instances take ranges of a shared particle pool; a full pool refuses, a freed range is reused."""
    b = small_bases["sphere12x10x9"]
    with Batch([b], slots=6, max_particles=1024, particle_pool=1536) as batch:
        assert batch.pool_free() == (1536, 1536)
        _fill(batch, b, [SPECS[0], SPECS[3]])  # 300 -> 512 and 700 -> 768 particles
        assert batch.pool_free()[0] == 1536 - 512 - 768
        w0, parts, f, params = _instance(b, SPECS[1])  # 500 particles: no room
        with pytest.raises(L.PSFError) as e:
            batch.set_instance(0, SPECS[1][0], w0, params, particles=parts, forcing=f)
        assert e.value.code == -3
        batch.clear_instance(0, SPECS[0][0])
        batch.set_instance(0, SPECS[1][0], w0, params, particles=parts, forcing=f)
        batch.step(5)
        ref = _oracle(b, SPECS[1], 5)
        assert rel_err(batch.get_state(0, SPECS[1][0]), ref.w) <= W_TOL
        assert np.abs(batch.get_particles(0, SPECS[1][0])[:, :3] - ref.pos).max() / b.h <= P_TOL_VOX


def test_multi_tile_shapes_match_oracle(medium_basis):
    """N = 160 (2 a-tiles, 3 K chunks), 40 slots (MMA N = 48, a partial 32-column epilogue chunk)."""
    b = medium_basis
    specs = [(0, 160, 0.01, L.PSF_FLAG_RENORM, 0.0, L.PSF_RK4, 400, 21),
             (17, 100, 0.02, L.PSF_FLAG_RENORM, 0.0, L.PSF_RK4, 0, 22),
             (33, 129, 0.01, L.PSF_FLAG_RENORM | L.PSF_FLAG_FORCING, 0.0, L.PSF_RK1, 300, 23),
             (39, 33, 0.02, L.PSF_FLAG_RENORM, 0.01, L.PSF_RK4, 0, 24)]
    with Batch([b], slots=40, max_particles=512) as batch:
        _fill(batch, b, specs)
        for i in range(40):
            if i not in (s[0] for s in specs):
                w0 = initial_coefficients(int(40 + (i * 7) % 120), 100 + i)
                batch.set_instance(0, i, w0, L.make_params(dt=0.01, integrator=L.PSF_RK4))
        batch.step(15)
        for spec in specs:
            ref = _oracle(b, spec, 15)
            assert rel_err(batch.get_state(0, spec[0]), ref.w) <= W_TOL, spec
            if spec[6]:
                p = batch.get_particles(0, spec[0])
                assert np.abs(p[:, :3] - ref.pos).max() / b.h <= P_TOL_VOX, spec
        u = batch.get_velocity(0, specs[0][0])
    ref1 = _oracle(b, specs[0], 15)
    assert np.abs(u - ref1.u).max() <= U_TOL * np.abs(ref1.u).max()


@pytest.mark.parametrize("ksplit", [2, 4])
def test_contraction_k_splits_agree(medium_basis, ksplit):
    """Splitting the contraction's K range per tile changes only the FP32 summation order."""
    b = medium_basis
    specs = [(0, 160, 0.01, L.PSF_FLAG_RENORM, 0.0, L.PSF_RK4, 0, 31), (5, 77, 0.02, L.PSF_FLAG_RENORM, 0.0, L.PSF_RK4, 0, 32)]
    outs = []
    for ks in (1, ksplit):
        with Batch([b], slots=8, max_particles=256, autotune=False, ksplit=ks) as batch:
            assert batch.info()["contraction_ksplit"] == ks
            _fill(batch, b, specs)
            batch.step(10)
            outs.append([batch.get_state(0, s[0]) for s in specs])
    for spec, w1, w2 in zip(specs, outs[0], outs[1]):
        assert rel_err(w2, w1) <= 1e-6
        assert rel_err(w2, _oracle(b, spec, 10).w) <= W_TOL


def test_fused_step_equals_three_launches(medium_basis):
    """One cooperative launch (contraction, state update, reconstruction) against three launches."""
    b = medium_basis
    specs = [(0, 160, 0.01, L.PSF_FLAG_RENORM, 0.0, L.PSF_RK4, 300, 41),
             (3, 90, 0.02, L.PSF_FLAG_RENORM | L.PSF_FLAG_DECAY_NEG, 0.03, L.PSF_RK1, 200, 42)]
    outs = []
    for fused in (True, False):
        with Batch([b], slots=5, max_particles=512, fused=fused, autotune=False) as batch:
            assert batch.info()["kernels_per_step"] == (2 if fused else 4)
            _fill(batch, b, specs)
            batch.step(12)
            assert batch.device_status() == 0
            outs.append([(batch.get_state(0, s[0]), batch.get_particles(0, s[0])) for s in specs])
    for spec, (w1, p1), (w2, p2) in zip(specs, outs[0], outs[1]):
        assert rel_err(w1, w2) <= 1e-10
        assert np.abs(p1[:, :3] - p2[:, :3]).max() / b.h <= 1e-5
        assert rel_err(w1, _oracle(b, spec, 12).w) <= W_TOL
