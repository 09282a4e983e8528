"""Particle density volume and ray march on CPU: the oracle restatement of the
reference's drawParticles compute path (Solver/SolverImpl/psfsolvergpu.cpp:876-1022)
against known answers, and the C ABI's argument checks (no device needed)."""
import ctypes as ct

import numpy as np
import pytest

from oracle import volume_oracle as VO
from parallelspectralfluids3d_b200 import _lib as L
from parallelspectralfluids3d_b200 import volume

MN = np.array([-0.5, -0.5, -0.5], np.float32)
MX = -MN


def cloud(n, seed=0, sigma=0.15):
    rng = np.random.default_rng(seed)
    xyz = rng.normal(0.0, sigma, (n, 3))
    return np.concatenate([xyz, np.full((n, 1), 50.0)], 1).astype(np.float32)


def test_histogram_counts_particles_in_the_box_once():
    p = cloud(20000)
    p[:100, 0] = 0.75     # outside: dropped
    p[100:110, 2] = -0.5  # on the lower face: cell 0
    h = VO.histogram(p, MN, MX, 16)
    inside = np.all((p[:, :3] >= MN) & (p[:, :3] < MX), axis=1)
    assert h.sum() == inside.sum()
    cells = np.floor((p[inside, :3] - MN) / (MX - MN) * 16).astype(int)
    want = np.zeros((16, 16, 16), np.int64)
    np.add.at(want, (cells[:, 2], cells[:, 1], cells[:, 0]), 1)
    assert np.array_equal(h, want)


def test_density_is_count_over_a_million_in_fp16():
    h = np.arange(4 ** 3, dtype=np.int32).reshape(4, 4, 4) * 977
    d = VO.density(h)
    assert d.dtype == np.float16
    assert np.array_equal(d, (h.astype(np.float32) / np.float32(1e6)).astype(np.float16))


def test_exp_polynomial_is_accurate_on_the_unit_interval():
    ys = np.linspace(0.0, 1.0, 257, dtype=np.float32)
    got = np.array([VO.exp_neg_unit(y) for y in ys])
    assert np.max(np.abs(got - np.exp(-ys.astype(np.float64))) / np.exp(-ys.astype(np.float64))) < 5e-7


def test_empty_volume_is_transparent():
    d = np.zeros((8, 8, 8), np.float16)
    img = VO.render(d, volume.make_view(12, 8, eye=(0.2, 0.3, 1.5)), MN, MX)
    assert np.all(img[..., :3] == 0.0) and np.all(img[..., 3] == 1.0)


def test_dense_blob_absorbs_the_rays_through_it():
    d = VO.density(VO.histogram(cloud(400000, sigma=0.08), MN, MX, 16))
    img = VO.render(d, volume.make_view(16, 16, eye=(0.0, 0.0, 1.5)), MN, MX)
    centre, corner = img[8, 8], img[0, 0]
    assert centre[3] < 0.5 and centre[0] > 0.0  # light scattered, transmittance reduced
    assert corner[3] == 1.0                     # a ray that misses the blob keeps all of it
    assert np.all((img >= 0.0) & (img <= 1.0))


def test_look_at_matches_the_glm_convention():
    m = volume.look_at((0.0, 0.0, 2.0), (0.0, 0.0, 0.0)).reshape(4, 4).T  # back to row-major
    assert np.allclose(m @ np.array([0.0, 0.0, 0.0, 1.0]), [0.0, 0.0, -2.0, 1.0])
    assert np.allclose(m[:3, :3], np.eye(3))


def test_c_abi_argument_checks_without_a_device():
    lib = L.load()
    out = ct.c_void_p()
    assert lib.psf_volume_create(0, 1, ct.byref(out)) == -6
    assert lib.psf_volume_create(0, 4096, ct.byref(out)) == -6
    assert lib.psf_volume_create(0, 64, None) == -1
    assert lib.psf_volume_destroy(None) == -1
    assert lib.psf_volume_splat(None, None, 0, None, None) == -1
    assert lib.psf_volume_render(None, None, None, 0) == -1
    assert lib.psf_volume_splat_context(None, None) == -1
