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

    def sub_cluster(self):
        """Cluster of every subdomain: the grid's clusters, subdomains numbered cluster by cluster."""
        per = int(np.prod(self.grid[1]))
        return np.arange(int(self.elem_domain.max()) + 1) // per

    def elem_dofs(self):
        d = self.dpn
        return (d * self.elem_nodes[:, :, None] + np.arange(d)[None, None, :]).reshape(self.elem_nodes.shape[0], -1)

    def rhs(self):
        f = np.zeros(self.ndofs)
        np.add.at(f, self.elem_dofs().ravel(), self.fe.ravel())
        return f

    def relative_residual(self, u, f=None):
        """||(K u - f)_free|| / ||f_free|| over the DOFs that are not Dirichlet-fixed, with the
        assembled global stiffness K (the primal residual check of the reference's
        src/solver/specific/itersolver.cpp:171-370, on the caller's assembled system)."""
        import scipy.sparse as sp
        if getattr(self, "_K", None) is None:
            dofs = self.elem_dofs()
            nd = dofs.shape[1]
            rows = np.repeat(dofs, nd, axis=1).ravel()
            cols = np.tile(dofs, (1, nd)).ravel()
            self._K = sp.csr_matrix((self.Ke.reshape(-1), (rows, cols)), shape=(self.ndofs, self.ndofs))
            free = np.ones(self.ndofs, dtype=bool)
            free[self.dirichlet_dofs()[0]] = False
            self._free = free
        f = self.rhs() if f is None else np.asarray(f)
        r = (self._K @ np.asarray(u).ravel() - f)[self._free]
        return float(np.linalg.norm(r) / np.linalg.norm(f[self._free]))

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


def bisection_boxes(side, levels, lo, hi, seed=0):
    """Seeded recursive bisection of an element box into 2**levels boxes.

    Level l splits every box along axis l % 3 at a position drawn uniformly from the
    positions that still let both halves be split by the remaining levels on that axis
    into pieces of lo..hi elements.  Returns a list of (origin, size) boxes."""
    rng = np.random.default_rng(seed)
    per_axis = [len([l for l in range(levels) if l % 3 == a]) for a in range(3)]
    for a in range(3):
        n = 2 ** per_axis[a]
        if not (lo * n <= side[a] <= hi * n):
            raise ValueError(f"side {side[a]} cannot be split into {n} pieces of {lo}..{hi} elements")
    boxes = [((0, 0, 0), tuple(int(v) for v in side))]
    done = [0, 0, 0]
    for level in range(levels):
        ax = level % 3
        done[ax] += 1
        pieces = 2 ** (per_axis[ax] - done[ax])          # pieces each half still becomes
        out = []
        for org, size in boxes:
            n = size[ax]
            amin = max(lo * pieces, n - hi * pieces)
            amax = min(hi * pieces, n - lo * pieces)
            a = int(rng.integers(amin, amax + 1))
            s1, s2 = list(size), list(size)
            s1[ax], s2[ax] = a, n - a
            o2 = list(org)
            o2[ax] += a
            out += [(org, tuple(s1)), (tuple(o2), tuple(s2))]
        boxes = out
    return boxes


def uneven_cube(physics="elasticity", side=(94, 94, 94), levels=9, lo=6, hi=14, seed=0, name=None, **kw):
    """Unit cube whose subdomains come from seeded recursive bisection (2**levels subdomains of
    lo..hi elements per side).  Elasticity: x=0 clamped, gravity; heat: the heat_cube setup."""
    gen = elasticity_cube if physics == "elasticity" else heat_cube
    P = gen(domains=(1, 1, 1), elements=tuple(side), name=name or f"{physics}_uneven", **kw)
    boxes = bisection_boxes(side, levels, lo, hi, seed)
    h = [1.0 / n for n in side]
    ijk = np.rint(P.coords[P.elem_nodes[:, 0]] / np.asarray(h)[None, :]).astype(np.int64)
    dom = np.full(P.elem_nodes.shape[0], -1, dtype=np.int64)
    for d, (org, size) in enumerate(boxes):
        m = np.all((ijk >= np.asarray(org)) & (ijk < np.asarray(org) + np.asarray(size)), axis=1)
        dom[m] = d
    assert (dom >= 0).all()
    order = np.argsort(dom, kind="stable")
    return Problem(P.name, P.dpn, P.coords, P.elem_nodes[order], dom[order], P.Ke[order], P.fe[order], P.dirichlet,
                   ((1, 1, 1), (len(boxes), 1, 1), tuple(side)))


def traction_loads(P: Problem, nrhs, seed=0, sigma=1e6, face_axis=0):
    """Load cases of seeded random nodal tractions on the face x = 1: every DOF of every
    node of the face draws N(0, sigma) (Pa per node; the cube is the unit cube)."""
    rng = np.random.default_rng(seed)
    face = np.nonzero(np.abs(P.coords[:, face_axis] - P.coords[:, face_axis].max()) < 1e-12)[0]
    R = np.zeros((nrhs, P.ndofs))
    dofs = (P.dpn * face[:, None] + np.arange(P.dpn)[None, :]).ravel()
    R[:, dofs] = rng.normal(0.0, sigma, size=(nrhs, dofs.size))
    return R


def _grid_element_index(nodes, coords, ne, h):
    lo = coords[nodes[:, 0]]
    ijk = np.rint(lo / np.asarray(h)[None, :]).astype(np.int64)
    return ijk[:, 0] + ne[0] * (ijk[:, 1] + ne[1] * ijk[:, 2])


def make_instance(problem: Problem, iopts=None, ropts=None, ext=None, batched=True, clusters=None):
    """Push a problem through the FETI4I API exactly as a caller would.

    ``clusters``: subdomain -> cluster map passed with FETI4ISetClusterPartition (HYBRID_FETI)."""
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
    if clusters is not None:
        M.set_clusters(clusters)
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
            F.set_extended(F.EXT_SYMM_TENSOR, 1)
            F.set_extended(F.EXT_DEVICE_PREP, 1)
            F.set_extended(F.EXT_RELIABLE_DELTA, 0.003)
            F.set_extended(F.EXT_SCHUR_EXPLICIT, 1)
            F.set_extended(F.EXT_OWNED_FIRST, 0)
            F.set_extended(F.EXT_OWNED_COUNT, 0)
            F.set_extended(F.EXT_TRUNCATE, 0)
    return inst


CONFIGS = {
    # configs of the benchmark definition; sizes as stated there
    "c1_elasticity_64": dict(kind="elasticity", domains=(4, 4, 4), elements=(8, 8, 8)),
    "c2_heat_512": dict(kind="heat", domains=(8, 8, 8), elements=(10, 10, 10)),
    # smaller variant of the heat workload (profiling captures; a few GB on the device)
    "c2_heat_216": dict(kind="heat", domains=(6, 6, 6), elements=(10, 10, 10)),
    # four subdomains of the c4/c5 subdomain size (device preprocessing captures; about 3 GB)
    "prep_elasticity_4x12": dict(kind="elasticity", domains=(2, 2, 1), elements=(12, 12, 12)),
    # 512 subdomains of 6..14 elements per side by seeded recursive bisection of a 94^3 grid
    "c3_elasticity_uneven": dict(kind="uneven", physics="elasticity", side=(94, 94, 94), levels=9, lo=6, hi=14),
    # the same construction at 64 subdomains
    "c3_elasticity_uneven_64": dict(kind="uneven", physics="elasticity", side=(40, 40, 40), levels=6, lo=6, hi=14),
    # Hybrid Total FETI: 4x4x4 clusters of 2x2x2 subdomains of 12^3 elements (run with --method 1)
    "c4_htfeti": dict(kind="elasticity", clusters=(4, 4, 4), domains=(2, 2, 2), elements=(12, 12, 12)),
    # the same cluster structure at 2x2x2 clusters of 2x2x2 subdomains of 6^3 elements
    "c4_htfeti_small": dict(kind="elasticity", clusters=(2, 2, 2), domains=(2, 2, 2), elements=(6, 6, 6)),
}


def build_config(name, **over):
    cfg = dict(CONFIGS[name])
    cfg.update(over)
    kind = cfg.pop("kind")
    if kind == "elasticity":
        return elasticity_cube(**cfg, name=name)
    if kind == "uneven":
        return uneven_cube(**cfg, name=name)
    return heat_cube(**cfg, name=name)
