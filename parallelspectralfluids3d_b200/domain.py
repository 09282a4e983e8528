"""Staggered voxel-grid cell complex (DEC) for a spectral-fluid domain.

This module restates the parts of the reference's ``DECMesh3D`` that the
per-step hot path and its precompute depend on:

* linear ids of voxels, faces and edges
  (``DEC/decmesh3d.cpp:12-45``; z-faces first, then y-faces, then x-faces;
  z-edges first, then y-edges, then x-edges);
* which voxel *creates* each face and which face first creates each edge.
  The reference adds every voxel in ``z, y, x`` order
  (``DEC/decmesh3d.cpp:89-102``), each voxel adds its faces in the order
  front, back, bottom, top, left, right (``:1369-1381``) and each new face
  adds its four edges in the order ``e1..e4`` (``:1202-1366``).  The creator
  fixes a face's stored normal and its ``e1..e4`` list; the first face that
  touches an edge fixes the edge's direction (``addEdge``, ``:1042-1200``);
* the per-voxel 6-bit "created here" sign string (``:1383-1399``) and
  ``getFaceSignum(vid, fidx)`` (``:1848-1853``);
* the signed incidence matrices d1 (edges x faces, ``DEC/dec.cpp:382-456``)
  and d2 (voxels x faces, ``DEC/dec.cpp:351-379``), and the dual Hodge star
  on edges (``DEC/dec.cpp:10-138``).

Inside/outside state follows ``setVoxelInside`` (``DEC/decmesh3d.cpp:1693``):
a face, edge or point is INSIDE when it belongs to at least one INSIDE voxel.

Domains are analytic masks on a grid centred at the origin, so that the
reference tracer's ``(aabb.min + aabb.extent + p) / h`` equals
``(p - aabb.min) / h`` (``Solver/SolverImpl/psfsolver.cpp:80-89``).
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

# Face creator directions, named as in the reference (DEC/decmesh3d.cpp:1202-1366).
FRONT, BACK, BOTTOM, TOP, LEFT, RIGHT = range(6)

# Stored face normal per creator direction (DEC/decmesh3d.cpp:1212,1237,1262,1287,1312,1337).
CREATOR_NORMAL = np.array(
    [
        [0.0, 0.0, -1.0],  # FRONT
        [0.0, 0.0, 1.0],  # BACK
        [0.0, 1.0, 0.0],  # BOTTOM
        [0.0, -1.0, 0.0],  # TOP
        [1.0, 0.0, 0.0],  # LEFT
        [-1.0, 0.0, 0.0],  # RIGHT
    ]
)


@dataclass
class Domain:
    """A voxel grid of ``dims = (nx, ny, nz)`` cells of size ``h`` with a fluid mask.

    ``inside`` is a boolean array of shape ``(nz, ny, nx)``; voxel ``(x, y, z)``
    has linear id ``z*nx*ny + y*nx + x`` (``DEC/decmesh3d.cpp:12-15``).
    """

    dims: tuple
    h: float
    inside: np.ndarray
    name: str = "domain"
    aabb_min: np.ndarray = field(default=None)
    aabb_max: np.ndarray = field(default=None)

    def __post_init__(self):
        nx, ny, nz = (int(d) for d in self.dims)
        self.dims = (nx, ny, nz)
        self.h = float(self.h)
        self.inside = np.asarray(self.inside, dtype=bool).reshape(nz, ny, nx)
        ext = np.array([nx, ny, nz], dtype=np.float64) * self.h
        if self.aabb_min is None:
            self.aabb_min = (-0.5 * ext).astype(np.float32)
        if self.aabb_max is None:
            self.aabb_max = (0.5 * ext).astype(np.float32)
        self.aabb_min = np.asarray(self.aabb_min, dtype=np.float32)
        self.aabb_max = np.asarray(self.aabb_max, dtype=np.float32)
        self._built = False

    # ------------------------------------------------------------------ counts
    @property
    def n_voxels(self) -> int:
        nx, ny, nz = self.dims
        return nx * ny * nz

    @property
    def n_zfaces(self) -> int:
        nx, ny, nz = self.dims
        return (nz + 1) * nx * ny

    @property
    def n_yfaces(self) -> int:
        nx, ny, nz = self.dims
        return (ny + 1) * nx * nz

    @property
    def n_xfaces(self) -> int:
        nx, ny, nz = self.dims
        return (nx + 1) * ny * nz

    @property
    def n_faces(self) -> int:
        return self.n_zfaces + self.n_yfaces + self.n_xfaces

    @property
    def n_zedges(self) -> int:
        nx, ny, nz = self.dims
        return (nx + 1) * (ny + 1) * nz

    @property
    def n_yedges(self) -> int:
        nx, ny, nz = self.dims
        return (nx + 1) * ny * (nz + 1)

    @property
    def n_xedges(self) -> int:
        nx, ny, nz = self.dims
        return nx * (ny + 1) * (nz + 1)

    @property
    def n_edges(self) -> int:
        return self.n_zedges + self.n_yedges + self.n_xedges

    # ----------------------------------------------------------- index maps
    # DEC/decmesh3d.cpp:12-45 (and Resources/Simulation/simulation.cl:6-24).
    def voxel_index(self, x, y, z):
        nx, ny, _ = self.dims
        return z * (nx * ny) + y * nx + x

    def zface_index(self, x, y, z):
        nx, ny, _ = self.dims
        return z * (nx * ny) + y * nx + x

    def yface_index(self, x, y, z):
        nx, ny, _ = self.dims
        return z * ((ny + 1) * nx) + y * nx + x + self.n_zfaces

    def xface_index(self, x, y, z):
        nx, ny, _ = self.dims
        return z * (ny * (nx + 1)) + y * (nx + 1) + x + self.n_zfaces + self.n_yfaces

    def zedge_index(self, x, y, z):
        nx, ny, _ = self.dims
        return z * (nx + 1) * (ny + 1) + y * (nx + 1) + x

    def yedge_index(self, x, y, z):
        nx, ny, _ = self.dims
        return z * (nx + 1) * ny + y * (nx + 1) + x + self.n_zedges

    def xedge_index(self, x, y, z):
        nx, ny, _ = self.dims
        return z * nx * (ny + 1) + y * nx + x + self.n_zedges + self.n_yedges

    # --------------------------------------------------------------- build
    def build(self) -> "Domain":
        """Build the face/edge tables by replaying the reference's creation order."""
        if self._built:
            return self
        nx, ny, nz = self.dims
        F, E = self.n_faces, self.n_edges

        # Grid coordinates of every face, per block.
        zz, yy, xx = np.meshgrid(np.arange(nz + 1), np.arange(ny), np.arange(nx), indexing="ij")
        zf = (xx.ravel(), yy.ravel(), zz.ravel())
        zz, yy, xx = np.meshgrid(np.arange(nz), np.arange(ny + 1), np.arange(nx), indexing="ij")
        yf = (xx.ravel(), yy.ravel(), zz.ravel())
        zz, yy, xx = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx + 1), indexing="ij")
        xf = (xx.ravel(), yy.ravel(), zz.ravel())
        fx = np.concatenate([zf[0], yf[0], xf[0]]).astype(np.int64)
        fy = np.concatenate([zf[1], yf[1], xf[1]]).astype(np.int64)
        fz = np.concatenate([zf[2], yf[2], xf[2]]).astype(np.int64)
        axis = np.concatenate(
            [np.full(self.n_zfaces, 2), np.full(self.n_yfaces, 1), np.full(self.n_xfaces, 0)]
        ).astype(np.int8)
        assert np.array_equal(self.zface_index(zf[0], zf[1], zf[2]), np.arange(self.n_zfaces))

        # Creator direction and creator voxel/slot of every face.  A face on the
        # low grid plane of its axis is created by the voxel above it as its
        # front/bottom/left face; every other face by the voxel below it as its
        # back/top/right face (the only two voxels that touch it, added in id order).
        creator = np.empty(F, dtype=np.int8)
        cvox = np.empty(F, dtype=np.int64)
        cslot = np.empty(F, dtype=np.int64)
        for ax, low_dir, high_dir, low_slot, high_slot in (
            (2, FRONT, BACK, 0, 1),
            (1, BOTTOM, TOP, 2, 3),
            (0, LEFT, RIGHT, 4, 5),
        ):
            m = axis == ax
            c = (fx, fy, fz)[ax][m]
            low = c == 0
            creator[np.where(m)[0]] = np.where(low, low_dir, high_dir)
            vx, vy, vz = fx[m].copy(), fy[m].copy(), fz[m].copy()
            shift = np.where(low, 0, 1)
            if ax == 0:
                vx -= shift
            elif ax == 1:
                vy -= shift
            else:
                vz -= shift
            cvox[m] = self.voxel_index(vx, vy, vz)
            cslot[m] = np.where(low, low_slot, high_slot)
        normal = CREATOR_NORMAL[creator]

        # e1..e4 of every face and the direction in which the face walks each edge
        # (+1 = POS, -1 = NEG), per creator direction (DEC/decmesh3d.cpp:1207-1357).
        fe = np.empty((F, 4), dtype=np.int64)
        fdir = np.empty((F, 4), dtype=np.int8)
        X, Y, Z = self.xedge_index, self.yedge_index, self.zedge_index
        table = {
            FRONT: [(X, 0, 1, 0, +1), (Y, 1, 0, 0, -1), (X, 0, 0, 0, -1), (Y, 0, 0, 0, +1)],
            BACK: [(X, 0, 1, 0, -1), (Y, 0, 0, 0, -1), (X, 0, 0, 0, +1), (Y, 1, 0, 0, +1)],
            TOP: [(X, 0, 0, 1, +1), (Z, 1, 0, 0, -1), (X, 0, 0, 0, -1), (Z, 0, 0, 0, +1)],
            BOTTOM: [(X, 0, 0, 1, -1), (Z, 0, 0, 0, -1), (X, 0, 0, 0, +1), (Z, 1, 0, 0, +1)],
            LEFT: [(Z, 0, 1, 0, -1), (Y, 0, 0, 0, -1), (Z, 0, 0, 0, +1), (Y, 0, 0, 1, +1)],
            RIGHT: [(Z, 0, 1, 0, +1), (Y, 0, 0, 1, -1), (Z, 0, 0, 0, -1), (Y, 0, 0, 0, +1)],
        }
        for d, entries in table.items():
            m = creator == d
            for k, (fn, dx, dy, dz, s) in enumerate(entries):
                fe[m, k] = fn(fx[m] + dx, fy[m] + dy, fz[m] + dz)
                fdir[m, k] = s

        # Edge direction = the walk direction of the first incidence in creation
        # order (voxel id, face slot, edge slot).
        key = ((cvox * 6 + cslot)[:, None] * 4 + np.arange(4)[None, :]).ravel()
        inc_edge = fe.ravel()
        order = np.lexsort((key, inc_edge))
        first = np.ones(order.size, dtype=bool)
        first[1:] = inc_edge[order][1:] != inc_edge[order][:-1]
        edge_dir = np.zeros(E, dtype=np.int8)
        edge_dir[inc_edge[order][first]] = fdir.ravel()[order][first]
        assert np.all(edge_dir != 0), "every edge belongs to at least one face"
        d1sign = np.where(fdir == edge_dir[fe], 1, -1).astype(np.int8)

        # Number of faces around each edge (Edge3D::dualCount).
        dual_count = np.bincount(inc_edge, minlength=E).astype(np.int8)

        # The six faces of every voxel, f1..f6 (DEC/decmesh3d.cpp:1376-1381).
        vz, vy, vx = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
        vx, vy, vz = vx.ravel(), vy.ravel(), vz.ravel()
        vf = np.stack(
            [
                self.zface_index(vx, vy, vz),
                self.zface_index(vx, vy, vz + 1),
                self.yface_index(vx, vy, vz),
                self.yface_index(vx, vy + 1, vz),
                self.xface_index(vx, vy, vz),
                self.xface_index(vx + 1, vy, vz),
            ],
            axis=1,
        )
        vid = np.arange(self.n_voxels)
        created_here = (cvox[vf] == vid[:, None]) & (cslot[vf] == np.arange(6)[None, :])

        # Sign bit string: 5 voxels x 6 bits per uint32 (DEC/decmesh3d.cpp:1390-1399).
        nwords = int(math.ceil(self.n_voxels / 5.0))
        bits = np.zeros(nwords, dtype=np.uint64)
        shifts = (vid % 5)[:, None] * 6 + np.arange(6)[None, :]
        contrib = (created_here.astype(np.uint64) << shifts.astype(np.uint64)).sum(axis=1)
        np.add.at(bits, vid // 5, contrib)
        sign_bits = bits.astype(np.uint32)

        inside_v = self.inside.ravel()
        # Inside voxels adjacent to each face (derivative2 only emits INSIDE voxels).
        n_in = np.zeros(F, dtype=np.int8)
        np.add.at(n_in, vf[inside_v].ravel(), 1)
        face_inside = n_in > 0
        edge_inside = np.zeros(E, dtype=bool)
        edge_inside[fe[face_inside].ravel()] = True

        self.face_xyz = np.stack([fx, fy, fz], axis=1)
        self.face_axis = axis
        self.face_creator = creator
        self.face_normal = normal
        self.face_edges = fe
        self.face_edge_sign = d1sign
        self.edge_dir = edge_dir
        self.edge_dual_count = dual_count
        self.voxel_faces = vf
        self.voxel_face_created = created_here
        self.sign_bits = sign_bits
        self.face_n_inside = n_in
        self.face_inside = face_inside
        self.edge_inside = edge_inside
        self.interior_faces = np.nonzero(n_in == 2)[0].astype(np.int64)
        self._built = True
        return self

    # --------------------------------------------------------------- signs
    def face_signum(self, vid, fidx):
        """``DECMesh3D::getFaceSignum(vid, fidx)`` (DEC/decmesh3d.cpp:1848-1853)."""
        self.build()
        vid = np.asarray(vid, dtype=np.int64)
        word = self.sign_bits[vid // 5].astype(np.int64)
        bit = (word >> ((vid % 5) * 6 + fidx)) & 1
        return np.where(bit == 1, 1, -1)

    def tracer_face_sign(self) -> np.ndarray:
        """Sign with which the reference tracer reads each face's velocity.

        The tracer multiplies every sampled face velocity by a sign taken from
        the voxel whose face it is (``psfsolver.cpp:160-188``,
        ``simulation.cl:129-157``): ``-s(v,4)`` / ``+s(v,5)`` for the x-faces
        at ``x`` / ``x+1`` of voxel ``v``, ``-s(v,2)`` / ``+s(v,3)`` for y, and
        ``+s(v,0)`` / ``-s(v,1)`` for z.  A face can be read from either of its
        two voxels; this returns the per-face sign and raises if the two readings
        disagree, so the sign can be folded into the basis once.
        """
        self.build()
        nx, ny, nz = self.dims
        sign = np.zeros(self.n_faces, dtype=np.int8)
        vz, vy, vx = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
        vx, vy, vz = vx.ravel(), vy.ravel(), vz.ravel()
        vid = self.voxel_index(vx, vy, vz)
        readings = [
            (self.xface_index(vx, vy, vz), -self.face_signum(vid, 4)),
            (self.xface_index(vx + 1, vy, vz), self.face_signum(vid, 5)),
            (self.yface_index(vx, vy, vz), -self.face_signum(vid, 2)),
            (self.yface_index(vx, vy + 1, vz), self.face_signum(vid, 3)),
            (self.zface_index(vx, vy, vz), self.face_signum(vid, 0)),
            (self.zface_index(vx, vy, vz + 1), -self.face_signum(vid, 1)),
        ]
        for f, s in readings:
            prev = sign[f]
            clash = (prev != 0) & (prev != s)
            if np.any(clash):
                raise ValueError("tracer face signs disagree between the two voxels of a face")
            sign[f] = s
        assert np.all(sign != 0)
        return sign

    # ----------------------------------------------------- DEC operators
    def d1(self):
        """Signed edge x face incidence (``derivative1(mesh, true)``, DEC/dec.cpp:382-456)."""
        import scipy.sparse as sp

        self.build()
        F = self.n_faces
        rows = self.face_edges.ravel()
        cols = np.repeat(np.arange(F), 4)
        vals = self.face_edge_sign.ravel().astype(np.float64)
        return sp.csr_matrix((vals, (rows, cols)), shape=(self.n_edges, F))

    def d2(self):
        """Signed voxel x face incidence of INSIDE voxels (``derivative2``, DEC/dec.cpp:351-379)."""
        import scipy.sparse as sp

        self.build()
        inside_v = self.inside.ravel()
        vids = np.nonzero(inside_v)[0]
        faces = self.voxel_faces[vids]
        sgn = np.where(self.voxel_face_created[vids], 1.0, -1.0)
        rows = np.repeat(vids, 6)
        return sp.csr_matrix(
            (sgn.ravel(), (rows, faces.ravel())), shape=(self.n_voxels, self.n_faces)
        )

    def dual_hodge_edges(self) -> np.ndarray:
        """Diagonal of the dual star on edges (``hodge2(mesh, true)``, DEC/dec.cpp:10-138).

        For an INSIDE edge: ``areaPrim / |point - edge centre|`` with
        ``areaPrim = 1/2 * sum_{j != k} (h/2)^2 |dir . (n_j x n_k)|`` over the
        faces around the edge.  Faces around an edge along one axis have normals
        along the two other axes, so the sum counts ordered pairs of faces of
        different orientation.  Non-INSIDE edges get 0.
        """
        self.build()
        E = self.n_edges
        h = self.h
        inc_edge = self.face_edges.ravel()
        inc_axis = np.repeat(self.face_axis, 4)
        n_per_axis = np.zeros((E, 3), dtype=np.int64)
        np.add.at(n_per_axis, (inc_edge, inc_axis), 1)
        tot = n_per_axis.sum(axis=1)
        ordered_pairs = tot * tot - (n_per_axis**2).sum(axis=1)
        area = 0.5 * ordered_pairs * (0.5 * h) ** 2
        star = np.where(self.edge_inside, area / (0.5 * h), 0.0)
        return star

    def primal_hodge_faces(self) -> float:
        """``hodge2(mesh, false)``: ``|voxel - face centre| / area = (h/2)/h^2`` on every face."""
        return (0.5 * self.h) / (self.h * self.h)


# --------------------------------------------------------------------- masks
def box_domain(n, h=None, name=None) -> Domain:
    """Empty box of ``n`` (int or (nx, ny, nz)) voxels, all fluid, solid walls."""
    dims = (n, n, n) if np.isscalar(n) else tuple(n)
    nx, ny, nz = dims
    if h is None:
        h = 1.0 / max(dims)
    inside = np.ones((nz, ny, nx), dtype=bool)
    return Domain(dims, h, inside, name=name or f"box{nx}x{ny}x{nz}")


def sphere_obstacle_domain(n, radius_voxels, h=None, name=None) -> Domain:
    """Box with a solid sphere at its centre; a voxel is solid when its centre is within the radius."""
    dims = (n, n, n) if np.isscalar(n) else tuple(n)
    nx, ny, nz = dims
    if h is None:
        h = 1.0 / max(dims)
    zc, yc, xc = np.meshgrid(
        np.arange(nz) + 0.5 - nz / 2.0,
        np.arange(ny) + 0.5 - ny / 2.0,
        np.arange(nx) + 0.5 - nx / 2.0,
        indexing="ij",
    )
    solid = xc**2 + yc**2 + zc**2 <= float(radius_voxels) ** 2
    return Domain(dims, h, ~solid, name=name or f"sphere{nx}x{ny}x{nz}r{radius_voxels}")


def channel_domain(dims, h=None, name=None) -> Domain:
    """Rectangular channel.  The reference has wall boundaries only, so this is an all-wall box."""
    d = box_domain(tuple(dims), h=h)
    d.name = name or "channel{}x{}x{}".format(*d.dims)
    return d
