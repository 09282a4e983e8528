"""Mesh voxeliser on the GPU (through the C ABI) against the oracle restatement
of the reference's slice map: bit-identical inside flags in both modes."""
import numpy as np
import pytest

from oracle import voxel_oracle as VO
from parallelspectralfluids3d_b200 import _lib as L
from parallelspectralfluids3d_b200 import voxel

from test_voxel import tessellated_box

pytestmark = pytest.mark.gpu


def lattice_soup(n_tri, seed, step):
    """Random (not closed) triangles with vertices on a lattice that hits pixel centres and edges exactly."""
    rng = np.random.default_rng(seed)
    v = (rng.integers(-16, 17, size=(3 * n_tri, 3)) * step).astype(np.float32)
    t = np.arange(3 * n_tri, dtype=np.uint32).reshape(-1, 3)
    return v, t


MESHES = {
    "box": lambda: voxel.box_mesh([-0.5, -0.4, -0.3], [0.45, 0.5, 0.35]),
    "tess_box": lambda: tessellated_box([-0.4, -0.3, -0.35], [0.3, 0.4, 0.25], 9),
    "sphere": lambda: voxel.icosphere(5, 0.45, center=(0.02, -0.01, 0.03)),
    "torus": lambda: voxel.torus_mesh(0.3, 0.12, 64, 32),
    "soup": lambda: lattice_soup(3000, 5, 1 / 64),
}


@pytest.mark.parametrize("mode", [voxel.REFERENCE, voxel.GEOMETRIC])
@pytest.mark.parametrize("name", sorted(MESHES))
@pytest.mark.parametrize("res", [1 / 32, 1 / 40, 0.0173])
def test_voxelize_matches_oracle(name, mode, res):
    v, t = MESHES[name]()
    want = VO.voxelize(v, t, res, mode)
    got, dims, mn, mx = voxel.voxelize(v, t, res, mode)
    d2, mn2, mx2 = VO.grid(v, res, mode)
    assert dims == d2 and np.array_equal(mn, mn2) and np.array_equal(mx, mx2)
    assert got.shape == want.shape
    assert np.array_equal(got, want), f"{int((got != want).sum())} voxels differ"


def test_layered_reference_mode_and_deep_geometric_columns():
    v, t = voxel.box_mesh([-0.05, -0.05, -1.0], [0.05, 0.05, 0.0])
    sv, st = voxel.icosphere(4, 0.3, center=(0.0, 0.0, -0.5))
    v = np.concatenate([v, sv])
    t = np.concatenate([t, st + 8])
    for mode in (voxel.REFERENCE, voxel.GEOMETRIC):
        want = VO.voxelize(v, t, 1 / 300, mode)
        got, dims, _, _ = voxel.voxelize(v, t, 1 / 300, mode)
        assert dims[2] == 300 and np.array_equal(got, want)


def test_voxelizer_reuse_profile_and_errors():
    vz = voxel.Voxelizer(max_vertices=50000, max_triangles=100000, max_voxels=64 ** 3)
    try:
        for name in ("sphere", "torus", "box"):
            v, t = MESHES[name]()
            got, _, _, _ = vz.run(v, t, 1 / 48, voxel.GEOMETRIC)
            assert np.array_equal(got, VO.voxelize(v, t, 1 / 48, voxel.GEOMETRIC))
        assert vz.profile(3) > 0.0
        v, t = MESHES["box"]()
        with pytest.raises(L.PSFError) as e:
            vz.run(v, np.array([[0, 1, 9]], np.uint32), 1 / 48)
        assert e.value.code == -1
        with pytest.raises(L.PSFError):
            vz.run(v, t, 1 / 200)  # grid larger than the voxeliser's capacity
        # empty triangle list: nothing inside
        got, _, _, _ = vz.run(v, np.zeros((0, 3), np.uint32), 1 / 48)
        assert not got.any()
    finally:
        vz.close()


def test_voxelised_domain_feeds_the_solver_setup():
    v, t = voxel.icosphere(4, 0.45)
    res = 0.9 / 16
    inside, dims, mn, mx = voxel.voxelize(v, t, res, voxel.GEOMETRIC)
    d = voxel.to_domain(inside, dims, res, mn, mx).build()
    assert d.dims == dims and d.inside.sum() == inside.sum() > 0
