"""GPU path (through the C ABI) against the FP64 oracle.

Tolerances: the FP32 plain path stays within 1e-5
relative on w after 100 steps and within 1e-4 voxel on particle positions on
the 16^3 / N = 64 workload; small domains use the same bars.
"""
import numpy as np
import pytest

from oracle import oracle as O
from parallelspectralfluids3d_b200 import _lib as L
from parallelspectralfluids3d_b200.fixture import initial_coefficients, initial_particles
from parallelspectralfluids3d_b200.solver import Context

from conftest import rel_err

pytestmark = pytest.mark.gpu

W_TOL = 1e-5       # relative L2 error of w
P_TOL_VOX = 1e-4   # max particle position error, in voxels
U_TOL = 2e-6       # face velocity error relative to max |u|


def run_pair(b, steps, integrator=L.PSF_RK4, dt=0.01, P=2048, seed_w=0, seed_p=1, flags=L.PSF_FLAG_RENORM,
             visc=0.0, forcing=None, lifetime=np.inf, seed=0):
    w0 = initial_coefficients(b.n_modes, seed_w)
    parts = initial_particles(b, P, seed_p, lifetime=lifetime)
    params = L.make_params(dt=dt, viscosity=visc, lifetime=lifetime, integrator=integrator, flags=flags, seed=seed)
    ctx = Context(b, params)
    if forcing is not None:
        ctx.set_forcing(forcing)
        params.flags |= L.PSF_FLAG_FORCING
        ctx.set_params(params)
    ctx.set_state(w0)
    ctx.set_particles(parts)
    ctx.step(steps)
    ctx.sync()
    oflags = (O.FLAG_RENORM if flags & L.PSF_FLAG_RENORM else 0) | (O.FLAG_DECAY_NEG if flags & L.PSF_FLAG_DECAY_NEG else 0)
    ref = O.OracleRollout(b, w0, parts, dt=dt, viscosity=visc, flags=oflags, integrator=integrator,
                          lifetime=lifetime, seed=seed, forcing=forcing)
    ref.step(steps)
    return ctx, ref


@pytest.mark.parametrize("integrator", [L.PSF_RK1, L.PSF_RK4])
def test_c1_100_steps(c1_basis, integrator):
    ctx, ref = run_pair(c1_basis, 100, integrator=integrator, P=4096)
    w = ctx.get_state()
    assert rel_err(w, ref.w) <= W_TOL
    err_vox = np.abs(ctx.get_particles()[:, :3] - ref.pos).max() / c1_basis.h
    assert err_vox <= P_TOL_VOX
    u = ctx.get_velocity()
    assert np.abs(u - ref.u).max() <= U_TOL * np.abs(ref.u).max()


@pytest.mark.parametrize("name", ["box6", "sphere10", "box576", "sphere12x10x9"])
def test_small_domains(small_bases, name):
    b = small_bases[name]
    ctx, ref = run_pair(b, 25, dt=0.05, P=1000)
    assert rel_err(ctx.get_state(), ref.w) <= W_TOL
    assert np.abs(ctx.get_particles()[:, :3] - ref.pos).max() / b.h <= P_TOL_VOX


def test_one_step_velocity_field_and_state(c1_basis):
    ctx, ref = run_pair(c1_basis, 1, P=0)
    assert rel_err(ctx.get_state(), ref.w) <= 1e-7
    u = ctx.get_velocity()
    assert np.abs(u - ref.u).max() <= U_TOL * np.abs(ref.u).max()
    # Wall faces stay exactly zero.
    mask = np.ones(c1_basis.n_faces, bool)
    mask[c1_basis.active_faces] = False
    assert np.all(u[mask] == 0)


@pytest.mark.parametrize("flags", [0, L.PSF_FLAG_RENORM, L.PSF_FLAG_RENORM | L.PSF_FLAG_DECAY_NEG])
def test_flags_viscosity_forcing(small_bases, flags):
    b = small_bases["sphere12x10x9"]
    f = np.zeros(b.n_modes)
    f[0] = 0.1 / 0.02
    ctx, ref = run_pair(b, 20, dt=0.02, P=500, flags=flags, visc=0.05, forcing=f)
    assert rel_err(ctx.get_state(), ref.w) <= W_TOL


def test_respawn_is_deterministic_and_matches(small_bases):
    b = small_bases["sphere10"]
    ctx, ref = run_pair(b, 12, dt=0.05, P=777, lifetime=4.0, seed=1234)
    got = ctx.get_particles()
    exp = ref.particles()
    assert np.array_equal(got[:, 3], exp[:, 3])
    assert np.abs(got[:, :3] - exp[:, :3]).max() / b.h <= P_TOL_VOX


def test_graph_replay_equals_single_steps(small_bases):
    b = small_bases["box576"]
    w0 = initial_coefficients(b.n_modes, 9)
    parts = initial_particles(b, 300, 9)
    outs = []
    for chunks in ([10], [1] * 10, [3, 7]):
        ctx = Context(b, L.make_params(dt=0.05))
        ctx.set_state(w0)
        ctx.set_particles(parts)
        for c in chunks:
            ctx.step(c)
        outs.append((ctx.get_state(), ctx.get_particles()))
        ctx.close()
    for w, p in outs[1:]:
        assert np.array_equal(w, outs[0][0]) and np.array_equal(p, outs[0][1])


def test_errors_are_status_codes(c1_basis):
    ctx = Context(c1_basis, L.make_params())
    with pytest.raises(L.PSFError) as e:
        ctx.step(1)  # no state yet
    assert e.value.code == -5
    with pytest.raises(L.PSFError):
        ctx.set_state(np.zeros(3))
    bad = L.make_params(integrator=3)
    with pytest.raises(L.PSFError):
        ctx.set_params(bad)
    ctx.close()


def test_profiled_steps_equal_graph_steps(small_bases):
    """psf_profile_step runs a step kernel by kernel; mixed with graph steps it gives the same states."""
    b = small_bases["sphere12x10x9"]
    w0 = initial_coefficients(b.n_modes, 4)
    parts = initial_particles(b, 400, 4)
    outs = []
    for plan in (["g"] * 6, ["p", "g", "p", "p", "g", "p"]):
        ctx = Context(b, L.make_params(dt=0.03))
        ctx.set_state(w0)
        ctx.set_particles(parts)
        for k in plan:
            ctx.step(1) if k == "g" else ctx.profile_step()
        outs.append((ctx.get_state(), ctx.get_particles(), ctx.get_velocity()))
        ctx.close()
    for a, c in zip(outs[0], outs[1]):
        assert np.array_equal(a, c)


def test_changes_between_steps_take_effect_at_the_next_step(small_bases):
    """Each step's state update is prepared one step ahead; changing the time step,
    the forcing or the state between steps must still act from the next step on."""
    b = small_bases["sphere12x10x9"]
    w0 = initial_coefficients(b.n_modes, 6)
    w1 = initial_coefficients(b.n_modes, 7)
    f = np.zeros(b.n_modes)
    f[1] = 0.5
    ctx = Context(b, L.make_params(dt=0.02))
    ctx.set_state(w0)
    ctx.step(3)
    ctx.set_params(L.make_params(dt=0.05))
    ctx.step(2)
    ctx.set_forcing(f)
    ctx.set_params(L.make_params(dt=0.05, flags=L.PSF_FLAG_RENORM | L.PSF_FLAG_FORCING))
    ctx.step(2)
    got_a = ctx.get_state()
    ctx.set_state(w1)
    assert np.array_equal(ctx.get_state(), w1)
    ctx.step(4)
    got_b = ctx.get_state()
    ctx.close()
    ref = O.OracleRollout(b, w0, None, dt=0.02, reconstruct=False).step(3)
    ref.dt = 0.05
    ref.step(2)
    ref.force = np.ascontiguousarray(f)
    ref.flags |= O.FLAG_FORCING
    ref.step(2)
    assert rel_err(got_a, ref.w) <= W_TOL
    ref_b = O.OracleRollout(b, w1, None, dt=0.05, forcing=f, reconstruct=False).step(4)
    assert rel_err(got_b, ref_b.w) <= W_TOL


def test_lean_bootstrap_and_steady_steps_agree(small_bases):
    """Re-setting the state before every step (each step then runs the lean graph) gives the
    same states, particles and velocity field as stepping on (bootstrap, then steady graphs)."""
    b = small_bases["sphere12x10x9"]
    w0 = initial_coefficients(b.n_modes, 8)
    parts = initial_particles(b, 500, 8)
    outs = []
    for reset in (False, True):
        ctx = Context(b, L.make_params(dt=0.03))
        ctx.set_state(w0)
        ctx.set_particles(parts)
        for _ in range(9):
            if reset:
                ctx.set_state(ctx.get_state())
            ctx.step(1)
        outs.append((ctx.get_state(), ctx.get_particles(), ctx.get_velocity()))
        ctx.close()
    for a, c in zip(outs[0], outs[1]):
        assert np.array_equal(a, c)


def test_resetting_particles_every_step_keeps_results(small_bases):
    """Setting the particles back before every step (the cell order is then reused, and re-sorted
    every 8th time) gives the same particles as stepping on without setting them."""
    b = small_bases["sphere12x10x9"]
    w0 = initial_coefficients(b.n_modes, 12)
    parts = initial_particles(b, 700, 12)
    outs = []
    for reset in (False, True):
        ctx = Context(b, L.make_params(dt=0.03))
        ctx.set_state(w0)
        ctx.set_particles(parts)
        for _ in range(12):
            if reset:
                ctx.set_particles(ctx.get_particles())
            ctx.step(1)
        outs.append((ctx.get_state(), ctx.get_particles()))
        ctx.close()
    assert np.array_equal(outs[0][0], outs[1][0]) and np.array_equal(outs[0][1], outs[1][1])


def test_end_to_end_loop_with_lookahead_at_set_particles(small_bases):
    """The end-to-end pattern (set state, set particles, step, read both back) queues the lean
    step's contraction and reconstruction at psf_set_particles.  It must give the same results
    as stepping on, and a setter between psf_set_particles and the step must still act."""
    b = small_bases["sphere12x10x9"]
    w0 = initial_coefficients(b.n_modes, 14)
    w1 = initial_coefficients(b.n_modes, 15)
    parts = initial_particles(b, 600, 14)
    f = np.zeros(b.n_modes)
    f[2] = 0.3
    outs = []
    for loop in (False, True):
        ctx = Context(b, L.make_params(dt=0.03))
        ctx.set_state(w0)
        ctx.set_particles(parts)
        for _ in range(10):
            if loop:
                w, p = ctx.get_state(), ctx.get_particles()
                ctx.set_state(w)
                ctx.set_particles(p)
            ctx.step(1)
        outs.append((ctx.get_state(), ctx.get_particles(), ctx.get_velocity()))
        ctx.close()
    for a, c in zip(outs[0], outs[1]):
        assert np.array_equal(a, c)

    # Setters after the queued lookahead: a new state, new forcing and time step.
    ctx = Context(b, L.make_params(dt=0.03))
    ctx.set_state(w0)
    ctx.set_particles(parts)
    u_before = ctx.get_velocity()
    ctx.set_state(w1)
    ctx.set_particles(parts)
    assert np.array_equal(ctx.get_velocity(), u_before)  # the visible field is unchanged until a step
    ctx.set_state(w0)
    ctx.step(2)
    got_a = ctx.get_state()
    ctx.set_state(w1)
    ctx.set_particles(parts)
    ctx.set_forcing(f)
    ctx.set_params(L.make_params(dt=0.05, flags=L.PSF_FLAG_RENORM | L.PSF_FLAG_FORCING))
    ctx.step(3)
    got_b = ctx.get_state()
    ctx.close()
    ref_a = O.OracleRollout(b, w0, None, dt=0.03, reconstruct=False).step(2)
    assert rel_err(got_a, ref_a.w) <= W_TOL
    ref_b = O.OracleRollout(b, w1, None, dt=0.05, forcing=f, reconstruct=False).step(3)
    assert rel_err(got_b, ref_b.w) <= W_TOL


def test_off_centre_box_matches_oracle(small_bases):
    """A box that is not centred on the origin: the tracer's index coordinate (the reference's
    (min + extent + p) / h) and its weight coordinate (p - min) / h then differ, and the GPU takes
    the branch that computes both; it must still follow the oracle.  With the two coordinates
    apart, the interpolant jumps where the index coordinate crosses a cell boundary, so an FP32
    (GPU) against FP64 (oracle) rounding of that coordinate can send a particle sitting on such a
    boundary to another cell: the bar holds for 99 % of the particles, and the w bar for all."""
    import dataclasses

    b0 = small_bases["sphere12x10x9"]
    off = np.array([0.3, -0.2, 0.1], dtype=b0.aabb_min.dtype)
    b = dataclasses.replace(b0, aabb_min=b0.aabb_min + off, aabb_max=b0.aabb_max + off)
    for integrator in (L.PSF_RK1, L.PSF_RK4):
        ctx, ref = run_pair(b, 40, integrator=integrator, dt=0.02, P=1500, seed_w=21, seed_p=22)
        assert rel_err(ctx.get_state(), ref.w) <= W_TOL
        err = np.abs(ctx.get_particles()[:, :3] - ref.pos).max(axis=1) / b.h
        ctx.close()
        assert np.percentile(err, 99) <= P_TOL_VOX, (np.percentile(err, 99), err.max())
        assert np.mean(err > P_TOL_VOX) <= 0.01, (np.mean(err > P_TOL_VOX), err.max())
