"""Particle density volume and ray march on the GPU (through the C ABI) against
the oracle restatement: bit-identical counts, FP16 density and image."""
import numpy as np
import pytest

from oracle import volume_oracle as VO
from parallelspectralfluids3d_b200 import _lib as L
from parallelspectralfluids3d_b200 import volume
from parallelspectralfluids3d_b200.fixture import initial_coefficients, initial_particles
from parallelspectralfluids3d_b200.solver import Context

from test_volume import MN, MX, cloud

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("res", [16, 33])
def test_density_matches_oracle(res):
    p = cloud(300000, seed=3, sigma=0.12)
    p[:50, 1] = 0.9  # outside the box
    vol = volume.Volume(res)
    try:
        vol.splat(p, MN, MX)
        got = vol.density()
        want = VO.density(VO.histogram(p, MN, MX, res))
        assert np.array_equal(got.view(np.uint16), want.view(np.uint16))
        # the counts are cleared for the next frame: a second splat gives the same density
        vol.splat(p, MN, MX)
        assert np.array_equal(vol.density().view(np.uint16), want.view(np.uint16))
    finally:
        vol.close()


@pytest.mark.parametrize("eye,light", [((0.3, 0.4, 1.6), (1.0, 2.0, 1.5)), ((-1.2, 0.2, -0.9), (-0.5, 1.0, 0.2))])
def test_render_matches_oracle(eye, light):
    p = cloud(500000, seed=4, sigma=0.1)
    vol = volume.Volume(24)
    try:
        vol.splat(p, MN, MX)
        view = volume.make_view(40, 28, eye=eye, light=light)
        got = vol.render(view)
        want = VO.render(VO.density(VO.histogram(p, MN, MX, 24)), view, MN, MX)
        assert got.shape == want.shape
        assert np.array_equal(got, want), f"{int(np.sum(got != want))} values differ"
        assert want[..., 3].min() < 0.9  # the image is not empty
        s, r = vol.profile(view, 2)
        assert s > 0.0 and r > 0.0
    finally:
        vol.close()


def test_splat_from_a_solver_context(make_basis):
    from parallelspectralfluids3d_b200.domain import sphere_obstacle_domain

    b = make_basis(sphere_obstacle_domain(16, 4), 32)
    ctx = Context(b, L.make_params(dt=0.01))
    vol = volume.Volume(32)
    try:
        ctx.set_state(initial_coefficients(b.n_modes, 0))
        ctx.set_particles(initial_particles(b, 20000, 1))
        ctx.step(5)
        vol.splat_context(ctx)
        dev = vol.density()
        host = ctx.get_particles()
        want = VO.density(VO.histogram(host, b.aabb_min, b.aabb_max, 32))
        assert np.array_equal(dev.view(np.uint16), want.view(np.uint16))
        with pytest.raises(L.PSFError) as e:
            vol.profile(volume.make_view(8, 8, eye=(0, 0, 2)))
        assert e.value.code == -5  # profiling needs a host splat
    finally:
        vol.close()
        ctx.close()


def test_render_before_splat_and_bad_sizes():
    vol = volume.Volume(8)
    try:
        with pytest.raises(L.PSFError) as e:
            vol.render(volume.make_view(4, 4, eye=(0, 0, 2)))
        assert e.value.code == -5
        with pytest.raises(L.PSFError):
            vol.splat(cloud(10), MX, MN)  # max < min
    finally:
        vol.close()
