"""DEC grid restatement: ids, creators, signs, operators (DEC/decmesh3d.cpp, DEC/dec.cpp)."""
import numpy as np
import pytest

from oracle.dec_literal import LiteralDEC
from parallelspectralfluids3d_b200.domain import (
    box_domain, channel_domain, sphere_obstacle_domain,
)

SMALL = [box_domain(4), box_domain((5, 3, 4)), box_domain((2, 6, 3)), sphere_obstacle_domain(8, 2)]


@pytest.mark.parametrize("dom", SMALL, ids=lambda d: d.name)
def test_vectorised_build_matches_literal_replay(dom):
    dom.build()
    L = LiteralDEC(dom.dims)
    F = dom.n_faces
    assert all(np.array_equal(L.face_normal[f], dom.face_normal[f]) for f in range(F))
    e_idx = np.array([[abs(s) - 1 for s in L.face_e[f]] for f in range(F)])
    e_sgn = np.array([[np.sign(s) for s in L.face_e[f]] for f in range(F)])
    assert np.array_equal(e_idx, dom.face_edges)
    assert np.array_equal(e_sgn, dom.face_edge_sign)
    assert np.array_equal(np.array(L.sign_bits, dtype=np.uint32), dom.sign_bits)
    assert np.array_equal(np.array(L.edge_dual), dom.edge_dual_count)
    vf = np.array([[abs(s) - 1 for s in L.voxel_f[v]] for v in range(dom.n_voxels)])
    vs = np.array([[s > 0 for s in L.voxel_f[v]] for v in range(dom.n_voxels)])
    assert np.array_equal(vf, dom.voxel_faces)
    assert np.array_equal(vs, dom.voxel_face_created)


@pytest.mark.parametrize("dom", SMALL, ids=lambda d: d.name)
def test_boundary_of_boundary_is_zero(dom):
    dom.build()
    assert abs(dom.d2() @ dom.d1().T).max() == 0


@pytest.mark.parametrize("dom", SMALL + [channel_domain((7, 4, 5))], ids=lambda d: d.name)
def test_tracer_sign_rule(dom):
    """x/y faces read +u except on the low grid plane, z faces read -u except on z = 0."""
    s = dom.tracer_face_sign()
    ax = dom.face_axis
    coord = dom.face_xyz[np.arange(dom.n_faces), ax]
    low = coord == 0
    expect = np.where(ax == 2, np.where(low, 1, -1), np.where(low, -1, 1))
    assert np.array_equal(s, expect)
    # Faces on a low grid plane are walls, so every active face reads +u (x, y) or -u (z).
    act = dom.interior_faces
    assert np.array_equal(s[act], np.where(ax[act] == 2, -1, 1))


def test_face_signum_matches_bit_string():
    dom = box_domain((3, 4, 2)).build()
    for vid in range(dom.n_voxels):
        for f in range(6):
            created = dom.voxel_face_created[vid, f]
            assert dom.face_signum(vid, f) == (1 if created else -1)


@pytest.mark.parametrize(
    "dom,F,F_act,E,V",
    [
        (box_domain(16), 13056, 11520, 13872, 4096),
        (sphere_obstacle_domain(32, 8), 101376, 88080, 104544, 30592),
        (box_domain(48), 338688, 324864, 345744, 110592),
        (box_domain(32), 101376, 95232, 104544, 32768),
        (sphere_obstacle_domain(40, 10), 196800, 173580, 201720, 59776),
        (channel_domain((64, 32, 32)), 201728, 191488, 206976, 65536),
    ],
    ids=["C1", "C2", "C3", "C4a", "C4b", "C4c"],
)
def test_config_domain_sizes(dom, F, F_act, E, V):
    dom.build()
    assert (dom.n_faces, len(dom.interior_faces), dom.n_edges, int(dom.inside.sum())) == (F, F_act, E, V)


def test_dual_star_values():
    dom = box_domain(4).build()
    star = dom.dual_hodge_edges() / dom.h
    # 4 faces around an edge -> 2h, 3 -> h, 2 -> h/2 (DEC/dec.cpp:110-121).
    expect = np.select([dom.edge_dual_count == 4, dom.edge_dual_count == 3], [2.0, 1.0], 0.5)
    assert np.allclose(star, expect)
