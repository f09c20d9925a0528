"""Oracle restatement of ESPRESO's Total-FETI solve with explicit Schur complements.

Test infrastructure only (see ``oracle/__init__.py``).  Every function cites
the reference code it restates (paths relative to the reference project).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np
import scipy.linalg as sla
import scipy.sparse as sp

from .numbering import Numbering

PREC_NONE, PREC_LUMPED, PREC_WEIGHT, PREC_DIRICHLET = 0, 1, 2, 3
# src/config/ecf/solver/feti.h:45-47
PREC_SUPER_DIRICHLET, PREC_MAGIC = 4, 5


@dataclass
class Subdomain:
    K: sp.csr_matrix            # unregularised stiffness, local DOF order
    f: np.ndarray
    R: np.ndarray               # kernel basis (n x nk)
    regmat: sp.csr_matrix
    chol: tuple                 # scipy cho_factor of K + RegMat
    lam: np.ndarray             # global multiplier index per local row
    dof: np.ndarray             # local DOF per local row
    sign: np.ndarray
    c: np.ndarray
    w: np.ndarray               # B1 scale (duplicity) per local row
    S: np.ndarray = None        # B K+ B^T (n_i x n_i)
    Sdir: np.ndarray = None     # Dirichlet preconditioner on sorted touched DOFs
    Ssd: sp.csr_matrix = None   # SUPER_DIRICHLET preconditioner on the same DOFs
    tdofs: np.ndarray = None    # sorted touched DOFs
    trow: np.ndarray = None     # local row -> index into tdofs
    extra: dict = field(default_factory=dict)

    def kplus(self, v):
        return sla.cho_solve(self.chol, v)


def assemble_subdomain(num: Numbering, d, elem_nodes, elem_domain, Ke, fe):
    """Domain stiffness/rhs in local DOF numbering (equivalent of the assembler's per-domain K)."""
    dpn = num.dpn
    sel = np.nonzero(elem_domain == d)[0]
    ln = num.g2l[d][elem_nodes[sel]]                        # (e,8) local nodes
    ldof = (dpn * ln[:, :, None] + np.arange(dpn)[None, None, :]).reshape(sel.size, -1)
    n = num.ndofs(d)
    rows = np.repeat(ldof, ldof.shape[1], axis=1).ravel()
    cols = np.tile(ldof, (1, ldof.shape[1])).ravel()
    K = sp.coo_matrix((Ke[sel].reshape(sel.size, -1).ravel(), (rows, cols)), shape=(n, n)).tocsr()
    f = np.zeros(n)
    np.add.at(f, ldof.ravel(), fe[sel].ravel())
    return K, f


def analytic_kernel(num: Numbering, d, coords):
    """Rigid-body kernel of a floating domain, orthonormalised.

    Heat: constant 1/sqrt(n) (src/assembler/physics/heattransfer.cpp:137-176).
    Elasticity: three translations and three rotations about the domain
    centre (src/assembler/physics/structuralmechanics3d.cpp:34-100); the
    reference's explicit Gram-Schmidt is replaced by a QR factorisation, which
    spans the same space.
    """
    nodes = num.dom_nodes[d]
    if num.dpn == 1:
        return np.full((nodes.size, 1), 1.0 / np.sqrt(nodes.size))
    p = coords[nodes] - coords[nodes].mean(axis=0)
    n = nodes.size
    R = np.zeros((3 * n, 6))
    for c in range(3):
        R[c::3, c] = 1.0
    R[0::3, 3], R[1::3, 3] = -p[:, 1], p[:, 0]
    R[0::3, 4], R[2::3, 4] = -p[:, 2], p[:, 0]
    R[1::3, 5], R[2::3, 5] = -p[:, 2], p[:, 1]
    q, _ = np.linalg.qr(R)
    return q


def fixpoint_regmat(num: Numbering, d, K, R, coords):
    """RegMat = max(diag K) * N (N^T N)^-1 N^T on fix-point DOFs.

    Restates structuralmechanics3d.cpp:102-183 (elasticity) and
    heattransfer.cpp:164-175 (heat: max diagonal on the first DOF).  The fix
    points themselves are chosen by this oracle (the reference uses METIS and
    a power iteration, src/mesh/preprocessing/fetidata.cpp:190-335): the
    nodes nearest to the 8 corners of the domain's bounding box.
    """
    n = K.shape[0]
    rho = K.diagonal().max()
    if num.dpn == 1:
        return sp.csr_matrix(([rho], ([0], [0])), shape=(n, n))
    nodes = num.dom_nodes[d]
    X = coords[nodes]
    lo, hi = X.min(0), X.max(0)
    fix = []
    for cx in (lo[0], hi[0]):
        for cy in (lo[1], hi[1]):
            for cz in (lo[2], hi[2]):
                fix.append(int(np.argmin(np.sum((X - np.array([cx, cy, cz])) ** 2, axis=1))))
    fix = sorted(set(fix))
    fd = np.array([3 * a + c for a in fix for c in range(3)])
    N = R[fd]
    blk = rho * N @ np.linalg.solve(N.T @ N, N.T)
    rr, cc = np.meshgrid(fd, fd, indexing="ij")
    return sp.csr_matrix((blk.ravel(), (rr.ravel(), cc.ravel())), shape=(n, n))


def dirichlet_schur(K, tdofs):
    """Schur complement of the unregularised K onto the touched DOFs
    (src/solver/specific/cpu/clustercpu.cpp:167-334)."""
    n = K.shape[0]
    inner = np.setdiff1d(np.arange(n), tdofs)
    Kd = K.toarray()
    Kbb = Kd[np.ix_(tdofs, tdofs)]
    if inner.size == 0:
        return Kbb
    Kii = Kd[np.ix_(inner, inner)]
    Kib = Kd[np.ix_(inner, tdofs)]
    return Kbb - Kib.T @ sla.cho_solve(sla.cho_factor(Kii), Kib)


def super_dirichlet_schur(K, tdofs):
    """SUPER_DIRICHLET preconditioner: S_sd = K_ss - K_sr diag(K_rr)^-1 K_rs on the touched DOFs s,
    with r the remaining DOFs (src/solver/specific/cpu/clustercpu.cpp:254-311, branch
    diagonalized_K_rr: K_rs scaled by 1/diag(K_rr) in place of K_rr^-1).  K is the unregularised
    stiffness (K_modif = K_reg - RegMat, :191-192).  Symmetric, sparse."""
    n = K.shape[0]
    inner = np.setdiff1d(np.arange(n), tdofs)
    K = sp.csr_matrix(K)
    Kss = K[tdofs][:, tdofs]
    if inner.size == 0:
        return sp.csr_matrix(Kss)
    Krs = K[inner][:, tdofs]
    dinv = 1.0 / K.diagonal()[inner]
    return sp.csr_matrix(Kss - Krs.T @ sp.diags(dinv) @ Krs)


class FETIProblem:
    """Total-FETI problem built the reference's way on a single cluster."""

    def __init__(self, num: Numbering, elem_nodes, elem_domain, Ke, fe, coords,
                 scaling=True, build_dirichlet=False, subdomains=None):
        self.num = num
        self.coords = coords
        self.sub = []
        for d in range(num.ndomains):
            K, f = assemble_subdomain(num, d, elem_nodes, elem_domain, Ke, fe)
            R = analytic_kernel(num, d, coords)
            RM = fixpoint_regmat(num, d, K, R, coords)
            Kreg = (K + RM).toarray()
            chol = sla.cho_factor(Kreg, lower=True)
            B = num.B[d]
            self.sub.append(Subdomain(K=K, f=f, R=R, regmat=RM, chol=chol, lam=B["lam"], dof=B["dof"],
                                      sign=B["sign"], c=B["c"], w=None))
        diags = [s.K.diagonal() for s in self.sub] if scaling else None
        for s, w in zip(self.sub, num.weights(diags)):
            s.w = w
        for s in self.sub:
            self._schur(s)
            if build_dirichlet:
                s.tdofs = np.unique(s.dof)
                s.trow = np.searchsorted(s.tdofs, s.dof)
                s.Sdir = dirichlet_schur(s.K, s.tdofs)
                s.Ssd = super_dirichlet_schur(s.K, s.tdofs)
        self.n_lambda = num.n_lambda
        self._coarse()

    def set_rhs(self, f_global):
        """Subdomain loads from a global DOF vector, split over the subdomains that share a node
        (value / multiplicity, src/assembler/physics/precomputed.cpp:61-65)."""
        num, dpn = self.num, self.num.dpn
        mult = np.zeros(int(max(n.max() for n in num.dom_nodes)) + 1)
        for nodes in num.dom_nodes:
            mult[nodes] += 1
        f_global = np.asarray(f_global, dtype=np.float64).reshape(-1, dpn)
        for d, s in enumerate(self.sub):
            nodes = num.dom_nodes[d]
            s.f = (f_global[nodes] / mult[nodes, None]).ravel()

    # -- explicit Schur complement (SparseSolverMKL.cpp:1207-1428: S = B K_reg^-1 B^T)
    def _schur(self, s: Subdomain):
        u, inv = np.unique(s.dof, return_inverse=True)
        E = np.zeros((s.K.shape[0], u.size))
        E[u, np.arange(u.size)] = 1.0
        X = s.kplus(E)[u]
        s.S = X[np.ix_(inv, inv)] * np.outer(s.sign, s.sign)

    # -- G = -(B R)^T stacked per domain (cluster.cpp:2018-2159), GG^T, e = -R^T f
    def _coarse(self):
        rows, cols, vals = [], [], []
        self.kofs = [0]
        for s in self.sub:
            nk = s.R.shape[1]
            Gi = -(s.sign[:, None] * s.R[s.dof]).T          # nk x n_i
            s.G = Gi
            for k in range(nk):
                rows.append(np.full(s.lam.size, self.kofs[-1] + k))
                cols.append(s.lam)
                vals.append(Gi[k])
            self.kofs.append(self.kofs[-1] + nk)
        self.n_kern = self.kofs[-1]
        self.G = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                               shape=(self.n_kern, self.n_lambda))
        GGt = (self.G @ self.G.T).toarray()
        self.GGt = GGt
        self.GGt_chol = sla.cho_factor(GGt, lower=True)

    # -- dual operators -----------------------------------------------------
    def apply_F(self, x, precision="f64"):
        """F x = sum_i B_i S_i B_i^T x (itersolvercpu.cpp:49-70); 'f32' restates the
        single-precision DenseMatVec path (SparseMatrix.cpp:1093-1104)."""
        y = np.zeros(self.n_lambda)
        for s in self.sub:
            xi = x[s.lam]
            if precision == "f32":
                yi = (s.S.astype(np.float32) @ xi.astype(np.float32)).astype(np.float64)
            else:
                yi = s.S @ xi
            np.add.at(y, s.lam, yi)
        return y

    def coarse_solve(self, d):
        return sla.cho_solve(self.GGt_chol, d)

    def projector(self, x, mode=0):
        """Projector_Inv (itersolver.cpp:5541-5623): mode 0 -> x - G^T (GG^T)^-1 G x,
        mode 1 -> G^T (GG^T)^-1 x (x in kernel space), mode 2 -> (GG^T)^-1 G x."""
        if mode == 1:
            return self.G.T @ self.coarse_solve(x)
        a = self.coarse_solve(self.G @ x)
        if mode == 2:
            return a
        return x - self.G.T @ a

    def precondition(self, x, kind):
        """Apply_Prec (itersolvercpu.cpp:520-602): scaled B (K | S_dir) B^T.  MAGIC applies the
        stored K - RegMat (cluster.cpp:413-433), the same operator as LUMPED's K x - RegMat x;
        SUPER_DIRICHLET applies the sparse S_sd of ``super_dirichlet_schur`` on the touched DOFs."""
        y = np.zeros(self.n_lambda)
        if kind == PREC_NONE:
            return x.copy()
        for s in self.sub:
            xi = x[s.lam] * s.w
            if kind in (PREC_LUMPED, PREC_MAGIC):
                u = np.zeros(s.K.shape[0])
                np.add.at(u, s.dof, s.sign * xi)
                v = s.K @ u
                yi = s.sign * v[s.dof]
            elif kind == PREC_WEIGHT:
                yi = xi.copy()
            elif kind in (PREC_DIRICHLET, PREC_SUPER_DIRICHLET):
                u = np.zeros(s.tdofs.size)
                np.add.at(u, s.trow, s.sign * xi)
                v = (s.Sdir if kind == PREC_DIRICHLET else s.Ssd) @ u
                yi = s.sign * v[s.trow]
            else:
                raise ValueError(kind)
            np.add.at(y, s.lam, yi * s.w)
        return y

    def vec_b(self):
        """b = sum_i B_i K_i^+ f_i - c (cluster.cpp:2732-2769)."""
        b = np.zeros(self.n_lambda)
        for s in self.sub:
            kf = s.kplus(s.f)
            np.add.at(b, s.lam, s.sign * kf[s.dof] - s.c)
        return b

    def vec_e(self):
        """e = -R^T f stacked (cluster.cpp:2660-2729)."""
        return np.concatenate([-(s.R.T @ s.f) for s in self.sub])

    # -- PCG (itersolver.cpp:1406-1724) ---------------------------------------
    def solve(self, precision=1e-8, max_it=1000, prec=PREC_LUMPED, f_precision="f64", history=None):
        b = self.vec_b()
        e = self.vec_e()
        x = self.projector(e, mode=1)
        Ax = self.apply_F(x, f_precision)
        r = b - Ax
        u = self.projector(r)
        tol = precision * min(np.linalg.norm(u), np.linalg.norm(b))
        n = self.n_lambda
        w = np.zeros(n); y = np.zeros(n); p = np.zeros(n)
        it = 0
        for it in range(max_it):
            wp, yp = w, y
            w = self.projector(r)
            if prec == PREC_NONE:
                y = w.copy()
            else:
                z = self.precondition(w, prec)
                y = self.projector(z)
            if it == 0:
                p = y.copy()
            else:
                beta = np.dot(y, w) / np.dot(yp, wp)
                p = y + beta * p
            Ap = self.apply_F(p, f_precision)
            alpha = np.dot(y, w) / np.dot(p, Ap)
            x = x + alpha * p
            r = r - alpha * Ap
            norm = np.linalg.norm(w)
            if history is not None:
                history.append(norm)
            if norm < tol:
                break
        self.iterations = it + 1
        self.lam = x
        self.residual = r
        self.alpha = self.projector(r, mode=2)
        return x

    def primal(self, lam=None, alpha=None):
        """u_i = K_i^+ (f_i - B_i^T lambda) + R_i alpha_i (itersolver.cpp:372-431)."""
        lam = self.lam if lam is None else lam
        alpha = self.alpha if alpha is None else alpha
        out = []
        for k, s in enumerate(self.sub):
            g = s.f.copy()
            np.add.at(g, s.dof, -s.sign * lam[s.lam])
            out.append(s.kplus(g) + s.R @ alpha[self.kofs[k]:self.kofs[k + 1]])
        return out

    def merge(self, us, n_nodes):
        """Average subdomain values per node -> global (n_nodes, dpn)."""
        dpn = self.num.dpn
        acc = np.zeros((n_nodes, dpn))
        cnt = np.zeros(n_nodes)
        for d, u in enumerate(us):
            nodes = self.num.dom_nodes[d]
            acc[nodes] += u.reshape(-1, dpn)
            cnt[nodes] += 1
        return acc / cnt[:, None]


def global_system(elem_nodes, Ke, fe, n_nodes, dpn):
    """Assembled global K, f (node-major DOFs) for direct-solve cross-checks."""
    ldof = (dpn * elem_nodes[:, :, None] + np.arange(dpn)[None, None, :]).reshape(elem_nodes.shape[0], -1)
    rows = np.repeat(ldof, ldof.shape[1], axis=1).ravel()
    cols = np.tile(ldof, (1, ldof.shape[1])).ravel()
    n = n_nodes * dpn
    K = sp.coo_matrix((Ke.reshape(Ke.shape[0], -1).ravel(), (rows, cols)), shape=(n, n)).tocsr()
    f = np.zeros(n)
    np.add.at(f, ldof.ravel(), fe.ravel())
    return K, f


def direct_solve(K, f, fixed_dofs, fixed_vals):
    """Global solve with Dirichlet DOFs eliminated (independent cross-check)."""
    import scipy.sparse.linalg as spla
    n = K.shape[0]
    u = np.zeros(n)
    u[fixed_dofs] = fixed_vals
    free = np.setdiff1d(np.arange(n), fixed_dofs)
    rhs = f[free] - K[free][:, fixed_dofs] @ u[fixed_dofs]
    u[free] = spla.spsolve(K[free][:, free].tocsc(), rhs)
    return u


def espreso_truncate(u, precision):
    """The reference's output formatting (src/solver/generic/FETISolver.cpp:130-147): every value
    truncated to dplaces = 1 / precision / max(1, 10^ceil(log10 max|u|)) places."""
    u = np.asarray(u, dtype=np.float64)
    gmax = np.abs(u).max()
    if gmax == 0.0:
        return u.copy()
    dplaces = 1.0 / precision / max(1.0, 10.0 ** np.ceil(np.log10(gmax)))
    return np.trunc(dplaces * u) / dplaces
