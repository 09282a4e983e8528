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


# ------------------------------------------------------------ literal ray march
def _literal_pixel(vol, view, mn, mx, px, py):
    """volume.frag (Resources/Effects/Volume/volume.frag:27-98) for one pixel, restated line by line
    in FP32 scalars (numpy float32 rounds every operation to nearest), with the trilinear
    clamp-to-border sampler and the exp polynomial of the oracle."""
    f = np.float32
    R = vol.shape[0]
    mn = [f(x) for x in mn]
    mx = [f(x) for x in mx]
    V = np.asarray(view["view"], np.float32).reshape(16)
    cam = [f(x) for x in view["camera"]]
    light = [f(x) for x in view["light"]]
    Wd, Ht = view["width"], view["height"]
    ext = [f(mx[a] - mn[a]) for a in range(3)]
    vox = f(f(f(ext[0] / f(R)) * f(ext[1] / f(R))) * f(ext[2] / f(R)))
    step = f(ext[0] / f(256))
    lview = [f(f(f(f(V[i] * light[0]) + f(V[4 + i] * light[1])) + f(V[8 + i] * light[2])) + f(V[12 + i] * f(1)))
             for i in range(3)]

    def texel(x, y, z):
        if x < 0 or y < 0 or z < 0 or x >= R or y >= R or z >= R:
            return f(0)
        return f(vol[z, y, x])

    def lerp(a, b, t):
        return f(f(f(f(1) - t) * a) + f(t * b))

    def sample(p):
        u = [f(f(p[a] * f(R)) - f(0.5)) for a in range(3)]
        fl = [f(np.floor(u[a])) for a in range(3)]
        if not all(fl[a] >= -1 and fl[a] < R for a in range(3)):
            return f(0)
        w = [f(u[a] - fl[a]) for a in range(3)]
        x, y, z = (int(fl[a]) for a in range(3))
        c00 = lerp(texel(x, y, z), texel(x + 1, y, z), w[0])
        c10 = lerp(texel(x, y + 1, z), texel(x + 1, y + 1, z), w[0])
        c01 = lerp(texel(x, y, z + 1), texel(x + 1, y, z + 1), w[0])
        c11 = lerp(texel(x, y + 1, z + 1), texel(x + 1, y + 1, z + 1), w[0])
        return lerp(lerp(c00, c10, w[1]), lerp(c01, c11, w[1]), w[2])

    def exp_neg(y):
        r = f(1)
        for k in range(12, 0, -1):
            r = f(f(1) + f(f(f(-y) / f(k)) * r))
        return r

    def length(x, y, z):
        return f(np.sqrt(f(f(f(x * x) + f(y * y)) + f(z * z))))

    r0 = f(f(f(f(2) * f(f(px) + f(0.5))) / f(Wd)) - f(1))
    r1 = f(f(f(f(2) * f(f(py) + f(0.5))) / f(Ht)) - f(1))
    r0 = f(r0 * f(f(Wd) / f(Ht)))
    r2 = f(-1.792590986919304)
    d = [f(f(f(f(r0 * V[4 * j]) + f(r1 * V[4 * j + 1])) + f(r2 * V[4 * j + 2])) + f(f(0) * V[4 * j + 3]))
         for j in range(3)]
    tt = [f(f(f(1) / d[a]) * f(mx[a] - cam[a])) for a in range(3)]
    tb = [f(f(f(1) / d[a]) * f(mn[a] - cam[a])) for a in range(3)]
    tmin = [min(tt[a], tb[a]) for a in range(3)]
    tmax = [max(tt[a], tb[a]) for a in range(3)]
    t0 = max(f(0), max(max(tmin[0], tmin[1]), max(tmin[0], tmin[2])))
    t1 = min(min(tmax[0], tmax[1]), min(tmax[0], tmax[2]))
    pos = [f(f(f(cam[a] + f(d[a] * t0)) - mn[a]) / ext[a]) for a in range(3)]
    stop = [f(f(f(cam[a] + f(d[a] * t1)) - mn[a]) / ext[a]) for a in range(3)]
    ray = [f(stop[a] - pos[a]) for a in range(3)]
    rl = length(*ray)
    sv = [f(f(step * ray[a]) / rl) for a in range(3)]
    trans, le = f(1), [f(0), f(0), f(0)]
    steps = 1024
    while rl > 0 and steps > 0:
        s = f(sample(pos) / vox)
        if s > f(0.001):
            lx, ly, lz = (f(lview[a] - pos[a]) for a in range(3))
            ll = length(lx, ly, lz)
            lv = [f(f(step * c) / ll) for c in (lx, ly, lz)]
            lp = list(pos)
            sd = f(0)
            for _ in range(128):
                lp = [f(lp[a] + lv[a]) for a in range(3)]
                sd = f(sd + f(sample(lp) / vox))
                if sd > f(6.907755278982137):
                    break
            dens = min(max(f(s * step), f(0)), f(1))
            e = exp_neg(min(max(f(sd * step), f(0)), f(1)))
            sh = [f(f(1) * e), f(f(0.5) * e), f(f(0) * e)]
            le = [f(le[a] + f(f(sh[a] * dens) * trans)) for a in range(3)]
            trans = f(trans * f(f(1) - dens))
            if trans < f(0.01):
                break
            le = [min(max(x, f(0)), f(1)) for x in le]
            trans = min(max(trans, f(0)), f(1))
        rl = f(rl - step)
        pos = [f(pos[a] + sv[a]) for a in range(3)]
        steps -= 1
    return np.array(le + [trans], np.float32)


def test_oracle_ray_march_matches_a_literal_restatement():
    d = VO.density(VO.histogram(cloud(200000, sigma=0.1), MN, MX, 12))
    view = volume.make_view(10, 8, eye=(0.3, 0.4, 1.6))
    img = VO.render(d, view, MN, MX)
    assert img[4, 5, 3] < 0.9 and img[4, 5, 0] > 0.0  # the centre ray crosses the cloud
    for py, px in [(4, 5), (3, 4), (0, 0), (7, 9), (5, 2)]:
        want = _literal_pixel(d, view, MN, MX, px, py)
        assert np.array_equal(img[py, px], want), (py, px, img[py, px], want)
