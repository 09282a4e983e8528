"""The FP64 oracle against independent NumPy restatements and known answers."""
import numpy as np
import pytest

from oracle import oracle as O
from parallelspectralfluids3d_b200.fixture import initial_coefficients, initial_particles


def np_velocity(b, dom, u, p):
    """Vectorised restatement of psfsolver.cpp:80-212 (with sign-string lookups)."""
    nx, ny, nz = b.dims
    h = b.h
    mn = b.aabb_min.astype(np.float64)
    shift = (b.aabb_min + (b.aabb_max - b.aabb_min)).astype(np.float32).astype(np.float64)
    cl = lambda v, n: np.clip(v, 0, n - 1)
    t = lambda v: np.trunc(v).astype(np.int64)
    xO, yO, zO = (cl(t((shift[i] + p[:, i]) / h), n) for i, n in enumerate((nx, ny, nz)))
    xM, yM, zM = (cl(t((shift[i] + p[:, i] - h / 2) / h), n) for i, n in enumerate((nx, ny, nz)))
    xP, yP, zP = (cl(t((shift[i] + p[:, i] + h / 2) / h), n) for i, n in enumerate((nx, ny, nz)))
    V, XF, YF, ZF = dom.voxel_index, dom.xface_index, dom.yface_index, dom.zface_index
    s = dom.face_signum
    mix = lambda a, c, w: a * (1 - w) + c * w

    def tri(vals, nrm):
        a = mix(vals[0], vals[1], nrm[:, 1]); c = mix(vals[2], vals[3], nrm[:, 1])
        d = mix(vals[4], vals[5], nrm[:, 1]); e = mix(vals[6], vals[7], nrm[:, 1])
        return mix(mix(a, c, nrm[:, 0]), mix(d, e, nrm[:, 0]), nrm[:, 2])

    uu = u.astype(np.float64)
    v1, v2, v3, v4 = V(xO, yM, zM), V(xO, yP, zM), V(xO, yM, zP), V(xO, yP, zP)
    X = [-s(v1, 4) * uu[XF(xO, yM, zM)], -s(v2, 4) * uu[XF(xO, yP, zM)],
         s(v1, 5) * uu[XF(xO + 1, yM, zM)], s(v2, 5) * uu[XF(xO + 1, yP, zM)],
         -s(v3, 4) * uu[XF(xO, yM, zP)], -s(v4, 4) * uu[XF(xO, yP, zP)],
         s(v3, 5) * uu[XF(xO + 1, yM, zP)], s(v4, 5) * uu[XF(xO + 1, yP, zP)]]
    cfx = np.stack([mn[0] + h * xO, mn[1] + h * yM + h / 2, mn[2] + h * zM + h / 2], 1)
    w1, w2, w3, w4 = V(xM, yO, zM), V(xP, yO, zM), V(xM, yO, zP), V(xP, yO, zP)
    Y = [-s(w1, 2) * uu[YF(xM, yO, zM)], s(w1, 3) * uu[YF(xM, yO + 1, zM)],
         -s(w2, 2) * uu[YF(xP, yO, zM)], s(w2, 3) * uu[YF(xP, yO + 1, zM)],
         -s(w3, 2) * uu[YF(xM, yO, zP)], s(w3, 3) * uu[YF(xM, yO + 1, zP)],
         -s(w4, 2) * uu[YF(xP, yO, zP)], s(w4, 3) * uu[YF(xP, yO + 1, zP)]]
    cfy = np.stack([mn[0] + h * xM + h / 2, mn[1] + h * yO, mn[2] + h * zM + h / 2], 1)
    z1, z2, z3, z4 = V(xM, yM, zO), V(xP, yM, zO), V(xM, yP, zO), V(xP, yP, zO)
    Z = [s(z1, 0) * uu[ZF(xM, yM, zO)], s(z3, 0) * uu[ZF(xM, yP, zO)],
         s(z2, 0) * uu[ZF(xP, yM, zO)], s(z4, 0) * uu[ZF(xP, yP, zO)],
         -s(z1, 1) * uu[ZF(xM, yM, zO + 1)], -s(z3, 1) * uu[ZF(xM, yP, zO + 1)],
         -s(z2, 1) * uu[ZF(xP, yM, zO + 1)], -s(z4, 1) * uu[ZF(xP, yP, zO + 1)]]
    cfz = np.stack([mn[0] + h * xM + h / 2, mn[1] + h * yM + h / 2, mn[2] + h * zO], 1)
    return np.stack([tri(X, (p - cfx) / h), tri(Y, (p - cfy) / h), tri(Z, (p - cfz) / h)], 1)


def test_contraction_matches_einsum(small_bases):
    b = small_bases["sphere12x10x9"]
    w = initial_coefficients(b.n_modes, 3)
    assert np.allclose(O.contract(b.C, w), np.einsum("kaj,a,j->k", b.C, w, w), rtol=1e-13, atol=1e-18)


def test_coefficient_step_matches_numpy(small_bases):
    b = small_bases["box576"]
    w0 = initial_coefficients(b.n_modes, 5)
    f = np.linspace(-1, 1, b.n_modes)
    for flags in (O.FLAG_RENORM, O.FLAG_RENORM | O.FLAG_DECAY_NEG, 0):
        r = O.OracleRollout(b, w0, dt=0.05, viscosity=0.3, flags=flags, forcing=f)
        r.step(1)
        w = w0.copy()
        e1 = w @ w
        w = w + 0.05 * np.einsum("kaj,a,j->k", b.C, w, w)
        if flags & O.FLAG_RENORM:
            w *= np.sqrt(e1 / (w @ w))
        sgn = -1.0 if flags & O.FLAG_DECAY_NEG else 1.0
        w *= np.exp(sgn * 0.3 * b.lam * 0.05)
        w += 0.05 * f
        assert np.allclose(r.w, w, rtol=1e-13, atol=1e-16)
        u = np.zeros(b.n_faces, dtype=np.float32)
        u[b.active_faces] = (b.phi @ r.w).astype(np.float32)
        assert np.array_equal(r.u, u)


@pytest.mark.parametrize("integrator", [1, 4])
@pytest.mark.parametrize("name", ["box6", "sphere10", "sphere12x10x9"])
def test_tracer_matches_numpy_restatement(small_bases, name, integrator):
    b = small_bases[name]
    dom = b.domain().build()
    rng = np.random.default_rng(7)
    u = rng.standard_normal(b.n_faces).astype(np.float32)
    parts = initial_particles(b, 500, 11)
    # Include points on the box faces and corners (clamped offsets).
    parts[:6, :3] = np.array([b.aabb_min, b.aabb_max, [0, 0, 0], b.aabb_min * 0.99,
                              [b.aabb_min[0], 0, b.aabb_max[2]], b.aabb_max * 0.999])
    r = O.OracleRollout(b, np.zeros(b.n_modes), parts, dt=0.02, integrator=integrator)
    r.u[:] = u
    r.trace()
    p = parts[:, :3].astype(np.float64)
    lo, hi = b.aabb_min.astype(np.float64), b.aabb_max.astype(np.float64)
    if integrator == 1:
        v = np_velocity(b, dom, u, p)
    else:
        k1 = np_velocity(b, dom, u, p)
        k2 = np_velocity(b, dom, u, np.clip(p + 0.01 * k1, lo, hi))
        k3 = np_velocity(b, dom, u, np.clip(p + 0.01 * k2, lo, hi))
        k4 = np_velocity(b, dom, u, np.clip(p + 0.02 * k3, lo, hi))
        v = (k1 + 2 * k2 + 2 * k3 + k4) / 6
    expect = np.clip(p + 0.02 * v, lo, hi)
    assert np.allclose(r.pos, expect, rtol=0, atol=1e-12)


def test_zero_state_keeps_particles_still(small_bases):
    b = small_bases["sphere10"]
    parts = initial_particles(b, 256, 2, lifetime=5.0)
    # Renormalisation of a zero state is 0/0 in the reference too, so it is off here.
    r = O.OracleRollout(b, np.zeros(b.n_modes), parts, dt=0.1, integrator=4, lifetime=5.0, flags=0)
    r.step(3)
    out = r.particles()
    assert np.array_equal(out[:, :3], parts[:, :3])
    assert np.array_equal(out[:, 3], parts[:, 3] - 3)


def test_uniform_field_moves_particles_exactly():
    from parallelspectralfluids3d_b200.domain import box_domain
    from parallelspectralfluids3d_b200.fixture import Basis

    dom = box_domain(8).build()
    b = Basis(dom.dims, dom.h, dom.aabb_min, dom.aabb_max, dom.interior_faces.astype(np.int32),
              np.ones(1), np.zeros(1), np.zeros((len(dom.interior_faces), 1)), np.zeros((1, 1, 1)),
              dom.sign_bits, dom.inside.ravel().astype(np.uint8))
    u = np.zeros(dom.n_faces, dtype=np.float32)
    s = dom.tracer_face_sign()
    u[dom.face_axis == 0] = 0.5 * s[dom.face_axis == 0]  # read back as +0.5 on every x face
    parts = np.array([[0.0, 0.1, -0.2, np.inf], [-0.3, 0.0, 0.3, np.inf]], dtype=np.float32)
    for integ in (1, 4):
        r = O.OracleRollout(b, np.zeros(1), parts, dt=0.1, integrator=integ)
        r.u[:] = u
        r.trace()
        assert np.allclose(r.pos[:, 0], parts[:, 0] + 0.05, atol=1e-7)
        assert np.allclose(r.pos[:, 1:], parts[:, 1:3], atol=1e-7)


def test_energy_is_renormalised(c1_basis):
    w0 = initial_coefficients(c1_basis.n_modes, 0)
    r = O.OracleRollout(c1_basis, w0, dt=0.01)
    r.step(20)
    assert abs(r.w @ r.w - 1.0) < 1e-12


def test_respawn_formula():
    from parallelspectralfluids3d_b200.domain import box_domain
    from parallelspectralfluids3d_b200.fixture import Basis

    dom = box_domain(4).build()
    b = Basis(dom.dims, dom.h, dom.aabb_min, dom.aabb_max, dom.interior_faces.astype(np.int32),
              np.ones(1), np.zeros(1), np.zeros((len(dom.interior_faces), 1)), np.zeros((1, 1, 1)),
              dom.sign_bits, dom.inside.ravel().astype(np.uint8))
    parts = np.zeros((64, 4), dtype=np.float32)  # life 0 -> respawn
    r = O.OracleRollout(b, np.zeros(1), parts, lifetime=60.0, seed=99)
    r.step_index = 17
    r.trace()
    h = lambda i, k: O.lib().psfo_hash(99, 17, i, k) % 1024
    for i in range(64):
        assert r.pos[i, 0] == np.float32((h(i, 1) / 1024.0 - 0.5) * 0.25)
        assert r.pos[i, 1] == np.float32(np.float32(-0.5) + np.float32(0.2))
        assert r.pos[i, 2] == np.float32((h(i, 3) / 1024.0 - 0.5) * 0.25)
        assert r.life[i] == np.float32(60.0 * (h(i, 2) / 1024.0))


def test_fp32_position_mode_stores_float_positions(small_bases):
    """positions="f32" rounds the state to FP32 after every step, as the reference's
    glm::vec4 particle buffer does; with FP64 positions the state is not float-exact."""
    from parallelspectralfluids3d_b200.fixture import initial_coefficients, initial_particles

    b = small_bases["sphere10"]
    w0 = initial_coefficients(b.n_modes, 0)
    parts = initial_particles(b, 300, 1)
    r32 = O.OracleRollout(b, w0, parts, dt=0.05, integrator=4, positions="f32").step(5)
    r64 = O.OracleRollout(b, w0, parts, dt=0.05, integrator=4).step(5)
    assert np.array_equal(r32.pos, r32.pos.astype(np.float32).astype(np.float64))
    assert not np.array_equal(r64.pos, r64.pos.astype(np.float32).astype(np.float64))
    assert np.abs(r32.pos - r64.pos).max() < 1e-5
    with pytest.raises(ValueError):
        O.OracleRollout(b, w0, parts, positions="f16")
