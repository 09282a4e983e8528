"""Mesh voxeliser on CPU: the oracle restatement of the reference's slice map
(Graphics/Model/Model.cpp:203-451) against known answers, and the C ABI's
grid and argument checks (no device needed)."""
import ctypes as ct

import numpy as np
import pytest

from oracle import voxel_oracle as VO
from parallelspectralfluids3d_b200 import _lib as L
from parallelspectralfluids3d_b200 import voxel
from parallelspectralfluids3d_b200._lib_voxel import VoxelMesh


def centres(dims, mn, res):
    W, H, D = dims
    z, y, x = np.meshgrid(np.arange(D), np.arange(H), np.arange(W), indexing="ij")
    return np.stack([mn[0] + (x + 0.5) * res, mn[1] + (y + 0.5) * res, mn[2] + (z + 0.5) * res], -1)


def tessellated_box(lo, hi, n):
    """Box whose faces are split into n x n quads (shared interior edges everywhere)."""
    lo = np.asarray(lo, np.float64)
    hi = np.asarray(hi, np.float64)
    verts, tris = [], []
    for axis in range(3):
        for side in (0, 1):
            a, b = [k for k in range(3) if k != axis]
            base = len(verts)
            for i in range(n + 1):
                for j in range(n + 1):
                    p = np.empty(3)
                    p[axis] = hi[axis] if side else lo[axis]
                    p[a] = lo[a] + (hi[a] - lo[a]) * i / n
                    p[b] = lo[b] + (hi[b] - lo[b]) * j / n
                    verts.append(p)
            for i in range(n):
                for j in range(n):
                    q = [base + i * (n + 1) + j, base + (i + 1) * (n + 1) + j, base + (i + 1) * (n + 1) + j + 1,
                         base + i * (n + 1) + j + 1]
                    tris += [(q[0], q[1], q[2]), (q[0], q[2], q[3])]
    return np.array(verts, np.float32), np.array(tris, np.uint32)


def test_grid_follows_the_reference_aabb():
    # The AABB starts at the origin (Graphics/AABB/AABB.cpp:3-7), so a mesh away from it still includes it.
    v, _ = voxel.box_mesh([0.25, 0.25, 0.25], [0.75, 0.5, 1.0])
    dims, mn, mx = VO.grid(v, 0.125)
    assert np.allclose(mn, 0.0) and np.allclose(mx, [0.75, 0.5, 1.0])
    assert dims == (6, 4, 8)
    d2, mn2, mx2 = voxel.grid(v, 0.125)
    assert d2 == dims and np.array_equal(mn2, mn) and np.array_equal(mx2, mx)


@pytest.mark.parametrize("mode", [VO.REFERENCE, VO.GEOMETRIC])
def test_box_filling_its_aabb_is_all_inside(mode):
    v, t = voxel.box_mesh([-0.5, -0.5, -0.5], [0.5, 0.5, 0.5])
    m = VO.voxelize(v, t, 1 / 16, mode)
    assert m.shape == (16, 16, 16) and m.all()


@pytest.mark.parametrize("mode", [VO.REFERENCE, VO.GEOMETRIC])
def test_shared_edges_cover_each_pixel_once(mode):
    # Splitting every face into many triangles must not change the result:
    # pixel centres on shared edges belong to exactly one triangle.
    lo, hi = [-0.4, -0.3, -0.35], [0.3, 0.4, 0.25]
    v1, t1 = voxel.box_mesh(lo, hi)
    v2, t2 = tessellated_box(lo, hi, 7)
    for res in (0.05, 0.0437, 1 / 32):
        a = VO.voxelize(v1, t1, res, mode)
        b = VO.voxelize(v2, t2, res, mode)
        assert np.array_equal(a, b)


def test_geometric_sphere_matches_centre_test():
    r = 0.4
    v, t = voxel.icosphere(5, r)
    res = 2 * r / 40
    m = VO.voxelize(v, t, res, VO.GEOMETRIC)
    dims, mn, _ = VO.grid(v, res, VO.GEOMETRIC)
    c = centres(dims, mn, res)
    rad = np.linalg.norm(c, axis=-1)
    # the inscribed polyhedron differs from the sphere only in a thin shell
    sure_in, sure_out = rad < r * 0.995, rad > r
    assert m[sure_in].all() and not m[sure_out].any()


def test_nested_boxes_leave_a_shell():
    vo, to = voxel.box_mesh([-0.5] * 3, [0.5] * 3)
    vi, ti = voxel.box_mesh([-0.25] * 3, [0.25] * 3)
    v = np.concatenate([vo, vi])
    t = np.concatenate([to, ti[:, ::-1] + len(vo)])
    m = VO.voxelize(v, t, 1 / 16, VO.GEOMETRIC)
    inner = np.zeros_like(m, dtype=bool)
    inner[4:12, 4:12, 4:12] = True
    assert np.array_equal(m.astype(bool), ~inner)


def test_reference_mode_counts_slices_from_the_top():
    # A box occupying the lower part of its AABB (which reaches up to z = 0 at the origin):
    # the reference's projection negates z, so its slab shows at the top of the index range.
    v, t = voxel.box_mesh([-0.5, -0.5, -1.0], [0.5, 0.5, -0.5])
    res = 1 / 16
    ref = VO.voxelize(v, t, res, VO.REFERENCE)
    geo = VO.voxelize(v, t, res, VO.GEOMETRIC)
    assert ref.shape == geo.shape == (16, 16, 16)
    assert geo[:8].all() and not geo[8:].any()
    assert np.array_equal(ref, geo[::-1])


def test_reference_mode_layers_follow_the_provoking_vertex():
    # Depth 200 needs two 128-slice layers.  Each triangle writes its mask only into the
    # layer of its last vertex (voxel.geom), with at most 128 bits; bits past the depth are dropped.
    v, t = voxel.box_mesh([-0.05, -0.05, -1.0], [0.05, 0.05, 0.0])
    res = 1 / 200
    m = VO.voxelize(v, t, res, VO.REFERENCE)
    assert m.shape[0] == 200
    # top and bottom faces: the top face (z = 0) lies in layer 0 with an empty mask; the bottom
    # face (z = -1, 200 slices down) lies in layer 1 and sets slices 128..199 of every column
    # it covers; the side faces draw nothing (zero area in xy).
    col = m[:, m.shape[1] // 2, m.shape[2] // 2]
    assert not col[:128].any() and col[128:].all()


def test_degenerate_and_out_of_range():
    v, t = voxel.box_mesh([-0.5] * 3, [0.5] * 3)
    t_deg = np.concatenate([t, np.array([[0, 0, 1], [2, 2, 2]], np.uint32)])
    assert np.array_equal(VO.voxelize(v, t, 0.1), VO.voxelize(v, t_deg, 0.1))
    with pytest.raises(ValueError):
        VO.voxelize(v, np.array([[0, 1, 8]], np.uint32), 0.1)
    empty = VO.voxelize(v, np.zeros((0, 3), np.uint32), 0.1)
    assert not empty.any()


def test_c_abi_grid_and_argument_checks_without_a_device():
    lib = L.load()
    v, t = voxel.icosphere(2, 0.5)
    m = VoxelMesh(v.ctypes.data_as(ct.POINTER(ct.c_float)), len(v), t.ctypes.data_as(ct.POINTER(ct.c_uint32)),
                  len(t))
    dims = np.zeros(3, np.int32)
    aabb = np.zeros(6, np.float32)
    for mode in (0, 1):
        assert lib.psf_voxel_grid(ct.byref(m), 0.05, mode, L.ptr(dims, ct.c_int32), L.ptr(aabb, ct.c_float)) == 0
        d, mn, mx = VO.grid(v, 0.05, mode)
        assert tuple(dims) == d and np.array_equal(aabb[:3], mn) and np.array_equal(aabb[3:], mx)
    assert lib.psf_voxel_grid(ct.byref(m), 0.0, 0, L.ptr(dims, ct.c_int32), L.ptr(aabb, ct.c_float)) == -1
    assert lib.psf_voxel_grid(ct.byref(m), 0.05, 7, L.ptr(dims, ct.c_int32), L.ptr(aabb, ct.c_float)) == -1
    assert lib.psf_voxel_grid(ct.byref(m), 1e-4, 0, L.ptr(dims, ct.c_int32), L.ptr(aabb, ct.c_float)) == -6
    assert lib.psf_voxel_grid(None, 0.05, 0, L.ptr(dims, ct.c_int32), L.ptr(aabb, ct.c_float)) == -1
    bad = v.copy()
    bad[3, 1] = np.nan
    mb = VoxelMesh(bad.ctypes.data_as(ct.POINTER(ct.c_float)), len(bad), None, 0)
    assert lib.psf_voxel_grid(ct.byref(mb), 0.05, 0, L.ptr(dims, ct.c_int32), L.ptr(aabb, ct.c_float)) == -1
    assert lib.psf_voxelizer_profile(None, 1, None) == -1
    assert lib.psf_voxelizer_destroy(None) == -1


def test_voxelised_mesh_builds_a_domain():
    v, t = voxel.icosphere(3, 0.45)
    res = 0.9 / 12
    m = VO.voxelize(v, t, res, VO.GEOMETRIC)
    dims, mn, mx = VO.grid(v, res, VO.GEOMETRIC)
    d = voxel.to_domain(m, dims, res, mn, mx, name="sphere12").build()
    assert d.dims == dims and d.inside.sum() == m.sum()
    assert d.n_voxels == m.size


# ------------------------------------------------------------ literal slice map
def _literal_slice_map(v, t, res):
    """The reference's slice map, restated literally in Python for small meshes: every covered
    pixel centre builds the RGBA32UI mask of voxel.frag (bits [0, z) over r, g, b, a, one bit at a
    time) in the layer of the triangle's last vertex (voxel.geom), XORs it into the texel
    (GL_XOR logic op, Model.cpp:249-256), and the read-back walks channels and bits with the
    reference's shifts (Model.cpp:278-441).  Coverage uses the same fixed rules as the oracle."""
    f32 = np.float32
    v = np.asarray(v, f32)
    mn = np.minimum(v.min(0), 0).astype(f32)
    mx = np.maximum(v.max(0), 0).astype(f32)
    ext = (mx - mn).astype(f32)
    W, H, D = (int(np.ceil(f32(ext[a] / f32(res)))) for a in range(3))
    layers = max(1, int(np.ceil(f32(ext[2] / f32(f32(res) * f32(128))))))
    ctr_z = f32(mn[2] + f32(f32(0.5) * f32(mx[2] - mn[2])))
    zo = f32(ext[2] * f32(0.5))
    tex = np.zeros((layers, H, W, 4), np.uint64)

    def proj(p):
        xw = f32(f32(f32(p[0] - mn[0]) / ext[0]) * f32(W))
        yw = f32(f32(f32(p[1] - mn[1]) / ext[1]) * f32(H))
        top = f32(f32(ctr_z - p[2]) + zo)
        return int(np.rint(f32(xw * f32(256)))), int(np.rint(f32(yw * f32(256)))), f32(top / f32(res)), \
            np.floor(f32(top / f32(f32(res) * f32(128))))

    def edge(a, b, px, py):
        return (b[0] - a[0]) * (py - a[1]) - (b[1] - a[1]) * (px - a[0])

    def owns(dx, dy):
        return dy < 0 or (dy == 0 and dx > 0)

    for tri in np.asarray(t).reshape(-1, 3):
        q = [proj(v[i]) for i in tri]
        area = edge(q[0], q[1], q[2][0], q[2][1])
        if area == 0:
            continue
        A, B, C = (q[0], q[1], q[2]) if area > 0 else (q[0], q[2], q[1])
        lay, zc = q[2][3], q[2][2]
        if not (lay >= 0) or lay >= layers:
            continue
        zbits = int(zc) if zc > 0 else 0
        mask = [0, 0, 0, 0]
        for c in range(4):                      # voxel.frag:25-48
            for d in range(32):
                if zbits != 0:
                    mask[c] |= 1 << d
                    zbits -= 1
        for j in range(H):
            for i in range(W):
                px, py = i * 256 + 128, j * 256 + 128
                e0, e1, e2 = edge(B, C, px, py), edge(C, A, px, py), edge(A, B, px, py)
                if not (e0 > 0 or (e0 == 0 and owns(C[0] - B[0], C[1] - B[1]))):
                    continue
                if not (e1 > 0 or (e1 == 0 and owns(A[0] - C[0], A[1] - C[1]))):
                    continue
                if not (e2 > 0 or (e2 == 0 and owns(B[0] - A[0], B[1] - A[1]))):
                    continue
                for c in range(4):
                    tex[int(lay), j, i, c] ^= mask[c]
    inside = np.zeros((D, H, W), np.uint8)
    for l in range(layers):
        for y in range(H):
            for x in range(W):
                for c in range(4):
                    word = int(tex[l, y, x, c])
                    for d in range(32):
                        z = 128 * l + 32 * c + d
                        if word & 1 and z < D:
                            inside[z, y, x] = 1
                        word >>= 1
    return inside


@pytest.mark.parametrize("case", ["box", "sphere", "layered"])
def test_oracle_matches_a_literal_slice_map(case):
    if case == "box":
        v, t = voxel.box_mesh([-0.4, -0.3, -0.5], [0.3, 0.45, 0.2])
        res = 0.07
    elif case == "sphere":
        v, t = voxel.icosphere(2, 0.4, center=(0.05, -0.02, 0.01))
        res = 0.06
    else:  # depth 150: two 128-slice layers
        v, t = voxel.box_mesh([-0.05, -0.05, -0.75], [0.05, 0.05, 0.0])
        res = 0.005
    assert np.array_equal(VO.voxelize(v, t, res, VO.REFERENCE), _literal_slice_map(v, t, res))
