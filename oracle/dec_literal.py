"""Test infrastructure (oracle): literal loop restatement of the reference's DEC mesh build.

Only the tests import this module; it is the checker for the vectorised
builder in ``parallelspectralfluids3d_b200/domain.py`` and for the tensor
builder in ``parallelspectralfluids3d_b200/basis.py``.  It replays, one call at
a time and in the same order, the reference's

* ``DECMesh3D::DECMesh3D``  voxel loop          DEC/decmesh3d.cpp:89-102
* ``DECMesh3D::addVoxel``   faces f1..f6, bits  DEC/decmesh3d.cpp:1369-1403
* ``DECMesh3D::addFace``    normals, e1..e4     DEC/decmesh3d.cpp:1202-1366
* ``DECMesh3D::addEdge``    first-creator dir   DEC/decmesh3d.cpp:1042-1200

and the literal dense wedge loop of ``PSFSolver::buildAdvection``
(Solver/SolverImpl/psfsolver.cpp:431-551).  Pure Python: tiny grids only.
"""

from __future__ import annotations

import math

import numpy as np

UNINIT = 0


class LiteralDEC:
    def __init__(self, dims):
        nx, ny, nz = dims
        self.dims = dims
        self.nZF = (nz + 1) * nx * ny
        self.nYF = (ny + 1) * nx * nz
        self.nXF = (nx + 1) * ny * nz
        self.nZE = (nx + 1) * (ny + 1) * nz
        self.nYE = (nx + 1) * ny * (nz + 1)
        self.nXE = nx * (ny + 1) * (nz + 1)
        F = self.nZF + self.nYF + self.nXF
        E = self.nZE + self.nYE + self.nXE
        V = nx * ny * nz
        self.face_made = [False] * F
        self.face_normal = [None] * F
        self.face_e = [None] * F  # signed ids: (index+1) * sign
        self.edge_made = [False] * E
        self.edge_v = [None] * E  # (v1, v2) point indices
        self.edge_dual = [0] * E
        self.voxel_f = [None] * V  # signed face ids
        self.sign_bits = [0] * int(math.ceil(V / 5.0))
        for z in range(nz):
            for y in range(ny):
                for x in range(nx):
                    self.add_voxel(z * nx * ny + y * nx + x, x, y, z)

    # DEC/decmesh3d.cpp:12-50
    def vox(self, x, y, z):
        nx, ny, _ = self.dims
        return z * nx * ny + y * nx + x

    def zf(self, x, y, z):
        nx, ny, _ = self.dims
        return z * nx * ny + y * nx + x

    def yf(self, x, y, z):
        nx, ny, _ = self.dims
        return z * (ny + 1) * nx + y * nx + x + self.nZF

    def xf(self, x, y, z):
        nx, ny, _ = self.dims
        return z * ny * (nx + 1) + y * (nx + 1) + x + self.nZF + self.nYF

    def ze(self, x, y, z):
        nx, ny, _ = self.dims
        return z * (nx + 1) * (ny + 1) + y * (nx + 1) + x

    def ye(self, x, y, z):
        nx, ny, _ = self.dims
        return z * (nx + 1) * ny + y * (nx + 1) + x + self.nZE

    def xe(self, x, y, z):
        nx, ny, _ = self.dims
        return z * nx * (ny + 1) + y * nx + x + self.nZE + self.nYE

    def pt(self, x, y, z):
        nx, ny, _ = self.dims
        return z * (ny + 1) * (nx + 1) + y * (nx + 1) + x

    def add_edge(self, eid, direction, x, y, z):
        """Returns +1 when the edge is new or already walks ``direction``, else -1."""
        step = {"X": (1, 0, 0), "Y": (0, 1, 0), "Z": (0, 0, 1)}[direction[1]]
        a = self.pt(x, y, z)
        b = self.pt(x + step[0], y + step[1], z + step[2])
        v = (a, b) if direction[0] == "+" else (b, a)
        if not self.edge_made[eid]:
            self.edge_made[eid] = True
            self.edge_v[eid] = v
            return 1
        return 1 if self.edge_v[eid] == v else -1

    def add_face(self, fid, direction, x, y, z):
        if self.face_made[fid]:
            return -1
        self.face_made[fid] = True
        X, Y, Z = self.xe, self.ye, self.ze
        spec = {
            "FRONT": ((0, 0, -1), [(X(x, y + 1, z), "+X", (x, y + 1, z)), (Y(x + 1, y, z), "-Y", (x + 1, y, z)),
                                   (X(x, y, z), "-X", (x, y, z)), (Y(x, y, z), "+Y", (x, y, z))]),
            "BACK": ((0, 0, 1), [(X(x, y + 1, z), "-X", (x, y + 1, z)), (Y(x, y, z), "-Y", (x, y, z)),
                                 (X(x, y, z), "+X", (x, y, z)), (Y(x + 1, y, z), "+Y", (x + 1, y, z))]),
            "TOP": ((0, -1, 0), [(X(x, y, z + 1), "+X", (x, y, z + 1)), (Z(x + 1, y, z), "-Z", (x + 1, y, z)),
                                 (X(x, y, z), "-X", (x, y, z)), (Z(x, y, z), "+Z", (x, y, z))]),
            "BOTTOM": ((0, 1, 0), [(X(x, y, z + 1), "-X", (x, y, z + 1)), (Z(x, y, z), "-Z", (x, y, z)),
                                   (X(x, y, z), "+X", (x, y, z)), (Z(x + 1, y, z), "+Z", (x + 1, y, z))]),
            "LEFT": ((1, 0, 0), [(Z(x, y + 1, z), "-Z", (x, y + 1, z)), (Y(x, y, z), "-Y", (x, y, z)),
                                 (Z(x, y, z), "+Z", (x, y, z)), (Y(x, y, z + 1), "+Y", (x, y, z + 1))]),
            "RIGHT": ((-1, 0, 0), [(Z(x, y + 1, z), "+Z", (x, y + 1, z)), (Y(x, y, z + 1), "-Y", (x, y, z + 1)),
                                   (Z(x, y, z), "-Z", (x, y, z)), (Y(x, y, z), "+Y", (x, y, z))]),
        }[direction]
        self.face_normal[fid] = np.array(spec[0], dtype=np.float64)
        for eid, _, _ in spec[1]:
            self.edge_dual[eid] += 1
        signed = []
        for eid, d, (ex, ey, ez) in spec[1]:
            s = self.add_edge(eid, d, ex, ey, ez)
            signed.append((eid + 1) * s)
        self.face_e[fid] = signed
        return 1

    def add_voxel(self, vid, x, y, z):
        ids = [self.zf(x, y, z), self.zf(x, y, z + 1), self.yf(x, y, z), self.yf(x, y + 1, z),
               self.xf(x, y, z), self.xf(x + 1, y, z)]
        where = [("FRONT", (x, y, z)), ("BACK", (x, y, z + 1)), ("BOTTOM", (x, y, z)),
                 ("TOP", (x, y + 1, z)), ("LEFT", (x, y, z)), ("RIGHT", (x + 1, y, z))]
        signed = []
        for fid, (d, c) in zip(ids, where):
            signed.append((fid + 1) * self.add_face(fid, d, *c))
        self.voxel_f[vid] = signed
        idx, off = vid // 5, vid % 5
        word = 0
        for k, s in enumerate(signed):
            word |= (0 if s < 0 else 1) << (off * 6 + k)
        self.sign_bits[idx] |= word


def literal_advection(dec: LiteralDEC, inside, h, phi_full, psi, lam):
    """Dense wedge loop + ``advection[i] = Psi^T (wedges[i] / lambda_i)``.

    Follows Solver/SolverImpl/psfsolver.cpp:431-551 term by term (including
    which edge each wedge lands on).  ``phi_full`` is F x N, ``psi`` is E x N.
    Returns C[k][a][j].
    """
    nx, ny, nz = dec.dims
    N = phi_full.shape[1]
    E = psi.shape[0]
    wedges = np.zeros((N, E, N))
    scale = (h / 2.0) * (h / 2.0)
    ones = np.ones(3)
    insd = np.asarray(inside).reshape(nz, ny, nx)
    for z in range(nz):
        for y in range(ny):
            for x in range(nx):
                if not insd[z, y, x]:
                    continue
                vid = dec.vox(x, y, z)
                fids = [abs(s) - 1 for s in dec.voxel_f[vid]]
                n = [dec.face_normal[f] for f in fids]
                fe = [[abs(s) - 1 for s in dec.face_e[f]] for f in fids]
                ie = [fe[0][0], fe[0][1], fe[0][2], fe[0][3], fe[1][0], fe[1][1], fe[1][2], fe[1][3],
                      fe[4][0], fe[4][2], fe[5][0], fe[5][2]]
                pairs = [(0, 3), (5, 0), (2, 0), (0, 4), (3, 1), (4, 1), (1, 2), (1, 5), (4, 3), (2, 4),
                         (3, 5), (5, 2)]
                for i in range(N):
                    va = [phi_full[f, i] for f in fids]
                    for j in range(N):
                        vb = [phi_full[f, j] for f in fids]
                        for t, (p, q) in enumerate(pairs):
                            wedges[i, ie[t], j] += scale * (va[p] * vb[q] - vb[p] * va[q]) * float(
                                np.dot(np.cross(n[p], n[q]), ones))
    C = np.empty((N, N, N))
    for i in range(N):
        C[i] = psi.T @ (wedges[i] / lam[i])
    return C
