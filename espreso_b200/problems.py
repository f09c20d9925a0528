"""Synthetic FETI4I callers: HEXA8 cube meshes decomposed into box subdomains.

This module plays the role of the finite-element code that calls FETI4I
(the reference's src/app/apitest.cpp provider): it builds a structured HEXA8
mesh, element stiffness matrices and loads, the Dirichlet DOFs and the
element -> subdomain partition.  Node IDs are grid indices (x fastest) and
DOF = dofs_per_node * node + component, as in the reference's grid generator
(src/input/meshgenerator/composition/gridgenerator.cpp:74-90).  Subdomains
are numbered cluster by cluster, x fastest (gridgenerator.cpp:42-71).

Workloads (seeded, synthetic; no dataset is involved):
  elasticity_cube   -- 3D linear elasticity, x=0 face clamped, body force
  heat_cube         -- 3D heat, log-uniform per-element conductivity, T=0 on z=0
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

_GP = 0.577350269189626
_XI = np.array([[-1, -1, -1], [1, -1, -1], [1, 1, -1], [-1, 1, -1],
                [-1, -1, 1], [1, -1, 1], [1, 1, 1], [-1, 1, 1]], dtype=np.float64)


@dataclass
class Problem:
    name: str
    dpn: int
    coords: np.ndarray        # (N,3)
    elem_nodes: np.ndarray    # (E,8)
    elem_domain: np.ndarray   # (E,)
    Ke: np.ndarray            # (E,nd,nd)
    fe: np.ndarray            # (E,nd)
    dirichlet: dict           # component -> (nodes, values)
    grid: tuple

    @property
    def n_nodes(self):
        return self.coords.shape[0]

    @property
    def ndofs(self):
        return self.n_nodes * self.dpn

    def elem_dofs(self):
        d = self.dpn
        return (d * self.elem_nodes[:, :, None] + np.arange(d)[None, None, :]).reshape(self.elem_nodes.shape[0], -1)

    def rhs(self):
        f = np.zeros(self.ndofs)
        np.add.at(f, self.elem_dofs().ravel(), self.fe.ravel())
        return f

    def dirichlet_dofs(self):
        dofs, vals = [], []
        for c, (nodes, v) in sorted(self.dirichlet.items()):
            nodes = np.asarray(nodes)
            dofs.append(self.dpn * nodes + c)
            vals.append(np.broadcast_to(np.asarray(v, dtype=np.float64), nodes.shape))
        return np.concatenate(dofs).astype(np.int32), np.concatenate(vals)


def _grid(clusters, domains, elements, length):
    ne = [c * d * e for c, d, e in zip(clusters, domains, elements)]
    nn = [v + 1 for v in ne]
    x = np.linspace(0.0, length[0], nn[0])
    y = np.linspace(0.0, length[1], nn[1])
    z = np.linspace(0.0, length[2], nn[2])
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    coords = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)
    # elements in (cluster, domain, element) order
    ex, ey, ez = ne
    K, J, I = np.meshgrid(np.arange(ez), np.arange(ey), np.arange(ex), indexing="ij")
    I, J, K = I.ravel(), J.ravel(), K.ravel()
    nid = lambda i, j, k: i + nn[0] * (j + nn[1] * k)
    nodes = np.stack([nid(I + a, J + b, K + c) for (a, b, c) in
                      ((0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1))], axis=1)
    el = np.array(elements)
    dd = np.array(domains)
    cl = (np.stack([I, J, K], 1) // (el * dd))
    dl = (np.stack([I, J, K], 1) // el) % dd
    cid = cl[:, 0] + clusters[0] * (cl[:, 1] + clusters[1] * cl[:, 2])
    did = dl[:, 0] + dd[0] * (dl[:, 1] + dd[1] * dl[:, 2])
    dom = cid * int(np.prod(dd)) + did
    order = np.lexsort((I, J, K, dom))
    return coords, nodes[order].astype(np.int64), dom[order].astype(np.int64), ne


def _ref_element(h, dpn, physics):
    """Element matrix of one box element with edges h (x,y,z), unit material, 2x2x2 Gauss."""
    X = _XI * 0.5 * np.asarray(h)[None, :] + 0.5 * np.asarray(h)[None, :]
    nd = 8 * dpn
    K = np.zeros((nd, nd))
    fN = np.zeros(8)
    if physics == "elasticity":
        nu = _NU
        EE = 1.0 / ((1 + nu) * (1 - 2 * nu))
        C = np.zeros((6, 6))
        C[:3, :3] = EE * nu
        for i in range(3):
            C[i, i] = EE * (1 - nu)
            C[3 + i, 3 + i] = EE * (0.5 - nu)
    for g in range(8):
        r = _GP if g & 4 else -_GP
        s = _GP if g & 2 else -_GP
        t = _GP if g & 1 else -_GP
        N = 0.125 * (1 + _XI[:, 0] * r) * (1 + _XI[:, 1] * s) * (1 + _XI[:, 2] * t)
        dN = np.stack([0.125 * _XI[:, 0] * (1 + _XI[:, 1] * s) * (1 + _XI[:, 2] * t),
                       0.125 * _XI[:, 1] * (1 + _XI[:, 0] * r) * (1 + _XI[:, 2] * t),
                       0.125 * _XI[:, 2] * (1 + _XI[:, 0] * r) * (1 + _XI[:, 1] * s)])
        J = dN @ X
        det = np.linalg.det(J)
        dNx = np.linalg.solve(J, dN)
        fN += N * det
        if physics == "heat":
            K += dNx.T @ dNx * det
        else:
            B = np.zeros((6, nd))
            for a in range(8):
                B[0, 3 * a], B[1, 3 * a + 1], B[2, 3 * a + 2] = dNx[0, a], dNx[1, a], dNx[2, a]
                B[3, 3 * a], B[3, 3 * a + 1] = dNx[1, a], dNx[0, a]
                B[4, 3 * a + 1], B[4, 3 * a + 2] = dNx[2, a], dNx[1, a]
                B[5, 3 * a], B[5, 3 * a + 2] = dNx[2, a], dNx[0, a]
            K += B.T @ C @ B * det
    return K, fN


_NU = 0.3


def elasticity_cube(clusters=(1, 1, 1), domains=(4, 4, 4), elements=(8, 8, 8), length=(1.0, 1.0, 1.0),
                    E=2.1e11, nu=0.3, body=(0.0, 0.0, -7850 * 9.81), clamp_axis=0, E_elem=None, name="elasticity"):
    """Linear elasticity on a box, the face ``clamp_axis``=0 fully fixed, uniform body force (N/m^3)."""
    global _NU
    _NU = nu
    coords, nodes, dom, ne = _grid(clusters, domains, elements, length)
    h = [l / n for l, n in zip(length, ne)]
    K1, fN = _ref_element(h, 3, "elasticity")
    nel = nodes.shape[0]
    Evec = np.full(nel, E) if E_elem is None else np.asarray(E_elem, dtype=np.float64)
    Ke = K1[None, :, :] * Evec[:, None, None]
    fe = np.zeros((nel, 24))
    for c in range(3):
        fe[:, c::3] = fN[None, :] * body[c]
    fixed = np.nonzero(np.abs(coords[:, clamp_axis]) < 1e-12)[0]
    dirichlet = {c: (fixed, 0.0) for c in range(3)}
    return Problem(name, 3, coords, nodes, dom, Ke, fe, dirichlet, (clusters, domains, elements))


def adjoint_cube(clusters=(1, 1, 1), domains=(8, 8, 8), elements=(12, 12, 12), length=(1.0, 1.0, 1.0),
                 nu=0.3, seed=0, name="adjoint"):
    """Adjoint workload: x=0 face clamped, unit point load at the centre node of the x=1 face (-z),
    rho_e ~ U[0.3, 1] seeded.  Returns (problem with unit-modulus element matrices, rho, load vector)."""
    P = elasticity_cube(clusters, domains, elements, length, E=1.0, nu=nu, body=(0.0, 0.0, 0.0), name=name)
    rng = np.random.default_rng(seed)
    gid = _grid_element_index(P.elem_nodes, P.coords, [c * d * e for c, d, e in zip(clusters, domains, elements)],
                              [l / (c * d * e) for l, c, d, e in zip(length, clusters, domains, elements)])
    rho = rng.uniform(0.3, 1.0, size=P.elem_nodes.shape[0])[gid]
    face = np.nonzero(np.abs(P.coords[:, 0] - length[0]) < 1e-12)[0]
    c = np.array([length[0], 0.5 * length[1], 0.5 * length[2]])
    node = face[np.argmin(np.sum((P.coords[face] - c) ** 2, axis=1))]
    f = np.zeros(P.ndofs)
    f[3 * node + 2] = -1.0
    return P, rho, f


def heat_cube(clusters=(1, 1, 1), domains=(8, 8, 8), elements=(10, 10, 10), length=(1.0, 1.0, 1.0),
              k_range=(1.0, 100.0), source=1.0, seed=0, name="heat"):
    """Heat conduction, per-element conductivity log-uniform on k_range, T=0 on z=0, uniform source."""
    coords, nodes, dom, ne = _grid(clusters, domains, elements, length)
    h = [l / n for l, n in zip(length, ne)]
    K1, fN = _ref_element(h, 1, "heat")
    nel = nodes.shape[0]
    rng = np.random.default_rng(seed)
    lo, hi = np.log10(k_range[0]), np.log10(k_range[1])
    # draw per element in grid order, independent of the subdomain ordering of the element list
    gid = _grid_element_index(nodes, coords, ne, h)
    kk = 10.0 ** rng.uniform(lo, hi, size=nel)[gid]
    Ke = K1[None, :, :] * kk[:, None, None]
    fe = np.broadcast_to(fN[None, :] * source, (nel, 8)).copy()
    fixed = np.nonzero(np.abs(coords[:, 2]) < 1e-12)[0]
    return Problem(name, 1, coords, nodes, dom, Ke, fe, {0: (fixed, 0.0)}, (clusters, domains, elements))


def _grid_element_index(nodes, coords, ne, h):
    lo = coords[nodes[:, 0]]
    ijk = np.rint(lo / np.asarray(h)[None, :]).astype(np.int64)
    return ijk[:, 0] + ne[0] * (ijk[:, 1] + ne[1] * ijk[:, 2])


def make_instance(problem: Problem, iopts=None, ropts=None, ext=None, batched=True):
    """Push a problem through the FETI4I API exactly as a caller would."""
    from . import feti4i as F
    if ext:
        for k, v in ext.items():
            F.set_extended(k, v)
    M = F.Matrix(index_base=0)
    dofs = problem.elem_dofs()
    if batched:
        M.add_elements(problem.elem_nodes, dofs, problem.Ke)
    else:
        for e in range(problem.elem_nodes.shape[0]):
            M.add_element(problem.elem_nodes[e], dofs[e], problem.Ke[e])
    M.set_partition(problem.elem_domain)
    dd, dv = problem.dirichlet_dofs()
    try:
        inst = F.Instance(M, problem.rhs(), dd, dv, iopts=iopts, ropts=ropts)
    finally:
        M.destroy()
        if ext:
            # restore the process-wide defaults
            F.set_extended(F.EXT_SCHUR_PRECISION, 0)
            F.set_extended(F.EXT_HOST_ONLY, 0)
            F.set_extended(F.EXT_SCALING, 1)
            F.set_extended(F.EXT_TILE_KERNEL, 0)
            F.set_extended(F.EXT_AUTOTUNE, 1)
            F.set_extended(F.EXT_RELIABLE_DELTA, 0.1)
    return inst


CONFIGS = {
    # configs of the benchmark definition; sizes as stated there
    "c1_elasticity_64": dict(kind="elasticity", domains=(4, 4, 4), elements=(8, 8, 8)),
    "c2_heat_512": dict(kind="heat", domains=(8, 8, 8), elements=(10, 10, 10)),
    # smaller variant of the heat workload (profiling captures; a few GB on the device)
    "c2_heat_216": dict(kind="heat", domains=(6, 6, 6), elements=(10, 10, 10)),
}


def build_config(name, **over):
    cfg = dict(CONFIGS[name])
    cfg.update(over)
    kind = cfg.pop("kind")
    if kind == "elasticity":
        return elasticity_cube(**cfg, name=name)
    return heat_cube(**cfg, name=name)
