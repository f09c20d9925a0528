"""Oracle restatement of ESPRESO's Hybrid Total FETI (HTFETI) with corner gluing.

Test infrastructure only (see ``oracle/__init__.py``).

Subdomains are grouped into clusters.  Inside a cluster the subdomains are
glued at corner nodes by a second constraint matrix B0; the dual iteration then
runs with the cluster's generalised inverse K_c^+ and the cluster kernels R_c,
so the coarse problem has one kernel block per cluster instead of one per
subdomain.  Restated (paths relative to the reference project):

* corner nodes: src/mesh/preprocessing/fetidata.cpp:146-188 -- for every node
  interval shared by at least two domains, the middle node; on intervals of
  the external-surface group every len/3-th node.  The surface check walks the
  list of surface intervals with one cursor that advances only on intervals
  shared by two or more domains, so after the first single-domain surface
  interval the middle-node rule applies to all remaining intervals; the
  restatement keeps that;
* B0 rows: src/assembler/constraints/equalityconstraints.cpp:504-555 -- per
  corner, per pair of consecutive domains of the corner's domain list, per
  DOF: +1 in the first domain, -1 in the second.  The reference runs one
  cluster per process and keeps the process's domains; with several clusters
  in one process each cluster keeps its own domains and numbers its own rows;
* B0 compression (cluster.cpp:1186-1224), G0 = -(B0 R)^T (:1226-1291),
  F0 = B0 K^+ B0^T (:1293-1478), S_alpha = G0 F0^-1 G0^T regularised with
  its own kernel H scaled by the mean of its diagonal (:1480-1700);
* the cluster solve multKplusGlobal (cluster.cpp:796-916):
    g0 = B0 K^+ x, e0 = -R^T x,
    alpha = S_alpha^-1 (G0 F0^-1 g0 - e0), lambda0 = F0^-1 (g0 - G0^T alpha),
    K_c^+ x = K^+ (x - B0^T lambda0) + R alpha;
* cluster kernels R_c = R H (Kplus_Rb, cluster.cpp:1776-1800), the dual
  G = -(B1 R_c)^T (:2040-2080), e = -R_c^T f (:2675-2700) and the primal
  u = K_c^+ (f - B1^T lambda) + R_c alpha (itersolver.cpp:372-431).
"""
from __future__ import annotations

import numpy as np
import scipy.linalg as sla
import scipy.sparse as sp

from .feti import FETIProblem
from .numbering import Numbering


def corner_nodes(num: Numbering):
    """Corner nodes with their domain lists, in the reference's order (fetidata.cpp:146-188)."""
    ext = [i for i, e in enumerate(num.interval_ext) if e]
    out = []
    ei = 0
    for i, (doms, nodes) in enumerate(num.intervals):
        if len(doms) == 1:
            continue
        if ei < len(ext) and ext[ei] == i:
            ei += 1
            inc = max(nodes.size // 3, 1)
            for n in nodes[::inc].tolist():
                out.append((n, doms))
        else:
            out.append((int(nodes[nodes.size // 2]), doms))
    return out


def b0_rows(num: Numbering, clusters):
    """B0 per domain as (cluster row, local DOF, sign) arrays, and rows per cluster
    (equalityconstraints.cpp:504-555)."""
    clusters = np.asarray(clusters, dtype=np.int64)
    ncl = int(clusters.max()) + 1
    dpn = num.dpn
    rows = [[] for _ in range(num.ndomains)]
    n0 = [0] * ncl
    for n, doms in corner_nodes(num):
        for c in sorted(set(int(clusters[d]) for d in doms)):
            cd = [d for d in doms if clusters[d] == c]
            for d1, d2 in zip(cd[:-1], cd[1:]):
                for comp in range(dpn):
                    r = n0[c]
                    n0[c] += 1
                    rows[d1].append((r, dpn * int(num.g2l[d1][n]) + comp, 1.0))
                    rows[d2].append((r, dpn * int(num.g2l[d2][n]) + comp, -1.0))
    out = []
    for d in range(num.ndomains):
        a = np.array(rows[d], dtype=np.float64).reshape(-1, 3)
        out.append(dict(row=a[:, 0].astype(np.int64), dof=a[:, 1].astype(np.int64), sign=a[:, 2].copy()))
    return out, n0


class HTFETIProblem(FETIProblem):
    """Hybrid Total FETI on clusters of subdomains (``clusters``: subdomain -> cluster)."""

    def __init__(self, num, elem_nodes, elem_domain, Ke, fe, coords, clusters, **kw):
        self.clusters = np.asarray(clusters, dtype=np.int64)
        super().__init__(num, elem_nodes, elem_domain, Ke, fe, coords, **kw)

    # -- cluster preprocessing and the coarse problem of the dual iteration
    def _coarse(self):
        nd = len(self.sub)
        ncl = int(self.clusters.max()) + 1
        self.B0, self.n0 = b0_rows(self.num, self.clusters)
        self.members = [[d for d in range(nd) if self.clusters[d] == c] for c in range(ncl)]
        self.cl = []
        for c in range(ncl):
            mem = self.members[c]
            n0 = self.n0[c]
            F0 = np.zeros((n0, n0))
            G0 = []
            for d in mem:
                s, b0 = self.sub[d], self.B0[d]
                n = s.K.shape[0]
                E = np.zeros((n, n0))
                np.add.at(E, (b0["dof"], b0["row"]), b0["sign"])       # B0_d^T
                F0 += E.T @ s.kplus(E)                                 # B0_d K_d^+ B0_d^T
                G0.append(-(E.T @ s.R).T)                              # -(B0_d R_d)^T
            G0 = np.vstack(G0) if G0 else np.zeros((0, n0))
            ka = G0.shape[0]
            if n0:
                F0inv = np.linalg.inv(F0)
                Sa = G0 @ F0inv @ G0.T
                _, sv, vt = np.linalg.svd(G0.T, full_matrices=True)   # ker S_alpha = ker G0^T
                tol = 1e-9 * (sv.max() if sv.size else 1.0)
                rank = int(np.sum(sv > tol))
                H = vt[rank:].T
            else:
                F0inv = np.zeros((0, 0))
                Sa = np.zeros((ka, ka))
                H = np.eye(ka)
            rho = float(np.mean(np.diag(Sa))) if ka and np.mean(np.diag(Sa)) > 0 else 1.0
            Sinv = np.linalg.inv(Sa + rho * H @ H.T)
            akofs = np.cumsum([0] + [self.sub[d].R.shape[1] for d in mem])
            self.cl.append(dict(members=mem, n0=n0, F0=F0, F0inv=F0inv, G0=G0, Sa=Sa, H=H, rho=rho,
                                Sinv=Sinv, akofs=akofs))
        # cluster kernels R_c restricted to each subdomain, G = -(B1 R_c)^T, GG^T
        self.kofs = [0]
        self.Rc = [None] * nd
        for C in self.cl:
            for i, d in enumerate(C["members"]):
                self.Rc[d] = self.sub[d].R @ C["H"][C["akofs"][i]:C["akofs"][i + 1]]
            self.kofs.append(self.kofs[-1] + C["H"].shape[1])
        self.n_kern = self.kofs[-1]
        rows, cols, vals = [], [], []
        for d, s in enumerate(self.sub):
            c = int(self.clusters[d])
            Gi = -(s.sign[:, None] * self.Rc[d][s.dof]).T
            s.G = Gi
            for k in range(Gi.shape[0]):
                rows.append(np.full(s.lam.size, self.kofs[c] + k))
                cols.append(s.lam)
                vals.append(Gi[k])
        self.G = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                               shape=(self.n_kern, self.n_lambda))
        self.GGt = (self.G @ self.G.T).toarray()
        self.GGt_chol = sla.cho_factor(self.GGt, lower=True)

    # -- cluster generalised inverse (cluster.cpp:796-916)
    def kplus_cluster(self, c, xs):
        """K_c^+ applied to the primal vectors xs[d] of the cluster's subdomains."""
        C = self.cl[c]
        mem = C["members"]
        g0 = np.zeros(C["n0"])
        e0 = []
        for d in mem:
            s, b0 = self.sub[d], self.B0[d]
            kx = s.kplus(xs[d])
            np.add.at(g0, b0["row"], b0["sign"] * kx[b0["dof"]])
            e0.append(-(s.R.T @ xs[d]))
        e0 = np.concatenate(e0) if e0 else np.zeros(0)
        t = (C["G0"] @ (C["F0inv"] @ g0) - e0) if C["n0"] else -e0
        alpha = C["Sinv"] @ t
        lam0 = C["F0inv"] @ (g0 - C["G0"].T @ alpha) if C["n0"] else np.zeros(0)
        out = {}
        for i, d in enumerate(mem):
            s, b0 = self.sub[d], self.B0[d]
            v = xs[d].copy()
            np.add.at(v, b0["dof"], -b0["sign"] * lam0[b0["row"]])
            out[d] = s.kplus(v) + s.R @ alpha[C["akofs"][i]:C["akofs"][i + 1]]
        return out

    def kplus_all(self, xs):
        out = {}
        for c in range(len(self.cl)):
            out.update(self.kplus_cluster(c, xs))
        return out

    # -- dual operators -----------------------------------------------------
    def apply_F(self, x, precision="f64"):
        """F x = B1 K_c^+ B1^T x (itersolvercpu.cpp:12-41 with multKplusGlobal_Kinv)."""
        if precision != "f64":
            raise NotImplementedError("the HTFETI oracle restates the FP64 operator")
        xs = {}
        for d, s in enumerate(self.sub):
            v = np.zeros(s.K.shape[0])
            np.add.at(v, s.dof, s.sign * x[s.lam])
            xs[d] = v
        ks = self.kplus_all(xs)
        y = np.zeros(self.n_lambda)
        for d, s in enumerate(self.sub):
            np.add.at(y, s.lam, s.sign * ks[d][s.dof])
        return y

    def vec_b(self):
        """b = B1 K_c^+ f - c (cluster.cpp:2732-2769 with the cluster solve)."""
        ks = self.kplus_all({d: s.f for d, s in enumerate(self.sub)})
        b = np.zeros(self.n_lambda)
        for d, s in enumerate(self.sub):
            np.add.at(b, s.lam, s.sign * ks[d][s.dof] - s.c)
        return b

    def vec_e(self):
        """e = -R_c^T f per cluster (cluster.cpp:2675-2700)."""
        e = np.zeros(self.n_kern)
        for d, s in enumerate(self.sub):
            c = int(self.clusters[d])
            e[self.kofs[c]:self.kofs[c + 1]] -= self.Rc[d].T @ s.f
        return e

    def primal(self, lam=None, alpha=None):
        """u = K_c^+ (f - B1^T lambda) + R_c alpha (itersolver.cpp:372-431)."""
        lam = self.lam if lam is None else lam
        alpha = self.alpha if alpha is None else alpha
        gs = {}
        for d, s in enumerate(self.sub):
            g = s.f.copy()
            np.add.at(g, s.dof, -s.sign * lam[s.lam])
            gs[d] = g
        ks = self.kplus_all(gs)
        out = []
        for d in range(len(self.sub)):
            c = int(self.clusters[d])
            out.append(ks[d] + self.Rc[d] @ alpha[self.kofs[c]:self.kofs[c + 1]])
        return out
