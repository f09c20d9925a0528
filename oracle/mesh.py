"""Oracle restatement of the reference's grid generator and HEXA8 element kernels.

Test infrastructure only (see ``oracle/__init__.py``).

* node numbering: global lexicographic grid index, x fastest
  (src/input/meshgenerator/composition/gridgenerator.cpp:74-90,
  src/input/meshgenerator/primitives/block.cpp:84-102);
* element numbering: clusters (x fastest), then domains of the cluster
  (x fastest), then elements of the domain (x fastest)
  (gridgenerator.cpp:42-71, block.cpp:148-168);
* HEXA8 node order and 2x2x2 Gauss rule with +-0.577350269189626, unit
  weights (src/mesh/elements/volume/hexahedron8.cpp:8-79);
* isotropic elasticity matrix with engineering shear strains
  (src/assembler/physics/structuralmechanics3d.cpp:191-240) and
  K_e = sum_gp B^T C B detJ, f_e = sum_gp rho a N detJ (:353-509);
* heat: K_e = sum_gp dN^T k dN detJ, f_e = sum_gp q N detJ
  (src/assembler/physics/heattransfer3d.cpp:248-539, isotropic case).
"""
from __future__ import annotations

import numpy as np

GP = 0.577350269189626
# HEXA8 reference coordinates of the 8 nodes (hexahedron8.cpp:33-42)
HEX_NODES = np.array([[-1, -1, -1], [1, -1, -1], [1, 1, -1], [-1, 1, -1],
                      [-1, -1, 1], [1, -1, 1], [1, 1, 1], [-1, 1, 1]], dtype=np.float64)
# faces with outward orientation (hexahedron8.cpp:12-19)
HEX_FACES = np.array([[0, 1, 5, 4], [3, 2, 1, 0], [4, 5, 6, 7],
                      [7, 6, 2, 3], [1, 2, 6, 5], [3, 0, 4, 7]], dtype=np.int64)


def _gauss_points():
    pts = []
    for i in range(8):
        r = GP if (i & 4) else -GP
        s = GP if (i & 2) else -GP
        t = GP if (i & 1) else -GP
        pts.append((r, s, t))
    return np.array(pts)


def shape(rst):
    """N (8,) and dN/d(r,s,t) (3,8) at one reference point."""
    r, s, t = rst
    xi = HEX_NODES
    N = 0.125 * (1 + xi[:, 0] * r) * (1 + xi[:, 1] * s) * (1 + xi[:, 2] * t)
    dN = np.empty((3, 8))
    dN[0] = 0.125 * xi[:, 0] * (1 + xi[:, 1] * s) * (1 + xi[:, 2] * t)
    dN[1] = 0.125 * xi[:, 1] * (1 + xi[:, 0] * r) * (1 + xi[:, 2] * t)
    dN[2] = 0.125 * xi[:, 2] * (1 + xi[:, 0] * r) * (1 + xi[:, 1] * s)
    return N, dN


_GPS = _gauss_points()
_SHAPES = [shape(p) for p in _GPS]


class Grid:
    """Box of HEXA8 elements decomposed into clusters x domains x elements."""

    def __init__(self, clusters=(1, 1, 1), domains=(1, 1, 1), elements=(1, 1, 1),
                 start=(0.0, 0.0, 0.0), length=(1.0, 1.0, 1.0)):
        self.clusters = tuple(int(v) for v in clusters)
        self.domains = tuple(int(v) for v in domains)
        self.elements = tuple(int(v) for v in elements)
        ne = [c * d * e for c, d, e in zip(self.clusters, self.domains, self.elements)]
        self.ne = tuple(ne)
        self.nn = tuple(v + 1 for v in ne)
        nx, ny, nz = self.nn
        step = [l / e for l, e in zip(length, ne)]
        x = start[0] + np.arange(nx) * step[0]
        y = start[1] + np.arange(ny) * step[1]
        z = start[2] + np.arange(nz) * step[2]
        Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
        self.coords = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)
        self.length = tuple(length)
        self.start = tuple(start)
        self._build_elements()

    def node_id(self, i, j, k):
        nx, ny, _ = self.nn
        return i + nx * (j + ny * k)

    def _build_elements(self):
        cx, cy, cz = self.clusters
        dx, dy, dz = self.domains
        ex, ey, ez = self.elements
        elems, edom, eclu = [], [], []
        ndom_c = dx * dy * dz
        ci = 0
        for kc in range(cz):
            for jc in range(cy):
                for ic in range(cx):
                    di = 0
                    for kd in range(dz):
                        for jd in range(dy):
                            for id_ in range(dx):
                                i0 = (ic * dx + id_) * ex
                                j0 = (jc * dy + jd) * ey
                                k0 = (kc * dz + kd) * ez
                                kk, jj, ii = np.meshgrid(np.arange(k0, k0 + ez), np.arange(j0, j0 + ey),
                                                         np.arange(i0, i0 + ex), indexing="ij")
                                ii, jj, kk = ii.ravel(), jj.ravel(), kk.ravel()
                                corners = []
                                for (a, b, c) in ((0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0),
                                                  (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1)):
                                    corners.append(self.node_id(ii + a, jj + b, kk + c))
                                elems.append(np.stack(corners, axis=1))
                                edom.append(np.full(ii.size, ci * ndom_c + di, dtype=np.int64))
                                eclu.append(np.full(ii.size, ci, dtype=np.int64))
                                di += 1
                    ci += 1
        self.elem_nodes = np.concatenate(elems).astype(np.int64)
        self.elem_domain = np.concatenate(edom)
        self.elem_cluster = np.concatenate(eclu)
        self.ndomains = int(self.elem_domain.max()) + 1

    def nodes_where(self, axis, value, tol=1e-9):
        return np.nonzero(np.abs(self.coords[:, axis] - value) < tol)[0]


def isotropic_C(E, nu):
    """6x6 elasticity matrix (structuralmechanics3d.cpp:199-235)."""
    EE = E / ((1 + nu) * (1 - 2 * nu))
    C = np.zeros((6, 6))
    C[:3, :3] = EE * nu
    for i in range(3):
        C[i, i] = EE * (1 - nu)
        C[3 + i, 3 + i] = EE * (0.5 - nu)
    return C


def _jac(X):
    """Per-gauss-point (detJ, dN/dx) for element coordinates X (E,8,3)."""
    out = []
    for N, dN in _SHAPES:
        J = np.einsum("an,enk->eak", dN, X)          # (E,3,3): J[a][k] = d x_k / d r_a
        det = np.linalg.det(J)
        invJ = np.linalg.inv(J)
        dNx = np.einsum("eka,an->ekn", invJ, dN)      # (E,3,8) d N / d x_k
        out.append((N, det, dNx))
    return out


def elasticity(X, E, nu, body=None):
    """Element stiffness (E,24,24) with node-major DOFs 3*a+c, and body-force rhs (E,24).

    ``E`` may be a scalar or a per-element array; ``body`` is a force density
    (3,) or (E,3) in N/m^3 (rho*acceleration).
    """
    X = np.asarray(X, dtype=np.float64)
    ne = X.shape[0]
    Earr = np.broadcast_to(np.asarray(E, dtype=np.float64), (ne,))
    C1 = isotropic_C(1.0, nu)
    K = np.zeros((ne, 24, 24))
    f = np.zeros((ne, 24))
    b = None if body is None else np.broadcast_to(np.asarray(body, dtype=np.float64), (ne, 3))
    for N, det, dNx in _jac(X):
        B = np.zeros((ne, 6, 24))
        for a in range(8):
            B[:, 0, 3 * a + 0] = dNx[:, 0, a]
            B[:, 1, 3 * a + 1] = dNx[:, 1, a]
            B[:, 2, 3 * a + 2] = dNx[:, 2, a]
            B[:, 3, 3 * a + 0] = dNx[:, 1, a]
            B[:, 3, 3 * a + 1] = dNx[:, 0, a]
            B[:, 4, 3 * a + 1] = dNx[:, 2, a]
            B[:, 4, 3 * a + 2] = dNx[:, 1, a]
            B[:, 5, 3 * a + 0] = dNx[:, 2, a]
            B[:, 5, 3 * a + 2] = dNx[:, 0, a]
        K += np.einsum("eia,ij,ejb->eab", B, C1, B) * (Earr * det)[:, None, None]
        if b is not None:
            for a in range(8):
                f[:, 3 * a:3 * a + 3] += (N[a] * det)[:, None] * b
    return K, f


def heat(X, k, source=0.0):
    """Element conductivity matrix (E,8,8) and heat-source rhs (E,8)."""
    X = np.asarray(X, dtype=np.float64)
    ne = X.shape[0]
    karr = np.broadcast_to(np.asarray(k, dtype=np.float64), (ne,))
    qarr = np.broadcast_to(np.asarray(source, dtype=np.float64), (ne,))
    K = np.zeros((ne, 8, 8))
    f = np.zeros((ne, 8))
    for N, det, dNx in _jac(X):
        K += np.einsum("ekn,ekm->enm", dNx, dNx) * (karr * det)[:, None, None]
        f += (qarr * det)[:, None] * N[None, :]
    return K, f


def face_pressure(Xf, p):
    """Nodal forces (F,4,3) of a normal pressure ``p`` acting on quad faces Xf (F,4,3).

    The face node order follows HEX_FACES (outward normal by the right-hand
    rule of the node order); a positive pressure pushes against the outward
    normal.
    """
    Xf = np.asarray(Xf, dtype=np.float64)
    out = np.zeros(Xf.shape)
    q = np.array([[-1, -1], [1, -1], [1, 1], [-1, 1]], dtype=np.float64)
    for (r, s) in ((-GP, -GP), (GP, -GP), (GP, GP), (-GP, GP)):
        N = 0.25 * (1 + q[:, 0] * r) * (1 + q[:, 1] * s)
        dNr = 0.25 * q[:, 0] * (1 + q[:, 1] * s)
        dNs = 0.25 * q[:, 1] * (1 + q[:, 0] * r)
        tr = np.einsum("a,fak->fk", dNr, Xf)
        ts = np.einsum("a,fak->fk", dNs, Xf)
        nvec = np.cross(tr, ts)                        # outward normal * dA
        out += -p * N[None, :, None] * nvec[:, None, :]
    return out


def boundary_faces(elem_nodes):
    """Faces of the element set that belong to exactly one element: (F,4) node lists."""
    faces = elem_nodes[:, HEX_FACES].reshape(-1, 4)
    key = np.sort(faces, axis=1)
    _, inv, cnt = np.unique(key, axis=0, return_inverse=True, return_counts=True)
    return faces[cnt[inv.ravel()] == 1]
