"""Oracle restatement of ESPRESO's node/DOF/multiplier numbering (single process).

Test infrastructure only (see ``oracle/__init__.py``).

Rules restated (one MPI rank, so no neighbour exchange):

* nodes are grouped into intervals of equal sorted domain lists, separately
  for nodes on the external surface of the body and the rest
  (src/mesh/preprocessing/arrangement.cpp:32-170); intervals are ordered by
  their domain lists (element-wise; on a common prefix the longer list
  first; ties by original order, surface group first) (:187-202); nodes of
  an interval are ordered by node ID (:181-185);
* a domain numbers its nodes interval by interval (:229-241); local DOF =
  dofs_per_node * local_node + component;
* Dirichlet multipliers come first: per interval, per component, per domain
  of the interval (redundant multipliers), per Dirichlet node
  (src/assembler/constraints/equalityconstraints.cpp:25-86,
  src/assembler/constraints/constraints.cpp:198-232);
* gluing multipliers follow: per interval, component-major, per
  non-Dirichlet node, one multiplier per pair of domains (a,b), a<b, with
  +1 in domain a and -1 in domain b (equalityconstraints.cpp:148-214,
  constraints.cpp:234-260);
* duplicity weights: 1 for Dirichlet rows, 1/ndomains for gluing rows, or
  with scaling diag_other / sum(diag) of the subdomain stiffness diagonals
  (equalityconstraints.cpp:287-423).
"""
from __future__ import annotations

import functools

import numpy as np

from .mesh import HEX_FACES


def _cmp_domains(a, b):
    """Interval order of arrangement.cpp:189-202 applied to (domains, group, idx)."""
    da, db = a[0], b[0]
    m = min(len(da), len(db))
    for i in range(m):
        if da[i] != db[i]:
            return -1 if da[i] < db[i] else 1
    if len(da) == len(db):
        ka, kb = (a[1], a[2]), (b[1], b[2])
        return -1 if ka < kb else (1 if ka > kb else 0)
    return -1 if len(da) > len(db) else 1


class Numbering:
    """Intervals, local DOF numbering and B1 rows for a single-cluster problem.

    Parameters
    ----------
    elem_nodes : (E,8) int node IDs of HEXA8 elements
    elem_domain : (E,) int domain of each element
    dpn : DOFs per node
    dirichlet : dict component -> (node array, value array)
    """

    def __init__(self, elem_nodes, elem_domain, n_nodes, dpn, dirichlet, redundant=True):
        if not redundant:
            raise NotImplementedError("the oracle restates redundant multipliers only")
        self.dpn = dpn
        self.n_nodes = n_nodes
        elem_nodes = np.asarray(elem_nodes, dtype=np.int64)
        elem_domain = np.asarray(elem_domain, dtype=np.int64)
        self.ndomains = int(elem_domain.max()) + 1

        # node -> sorted domain list
        pairs = np.unique(np.stack([elem_nodes.ravel(), np.repeat(elem_domain, elem_nodes.shape[1])], 1), axis=0)
        starts = np.searchsorted(pairs[:, 0], np.arange(n_nodes + 1))
        node_doms = [tuple(pairs[starts[n]:starts[n + 1], 1].tolist()) for n in range(n_nodes)]

        # external surface nodes: faces owned by exactly one element
        faces = elem_nodes[:, HEX_FACES].reshape(-1, 4)
        key = np.sort(faces, axis=1)
        _, inv, cnt = np.unique(key, axis=0, return_inverse=True, return_counts=True)
        ext = np.zeros(n_nodes, dtype=bool)
        ext[faces[cnt[inv.ravel()] == 1].ravel()] = True

        groups = {}
        for n in range(n_nodes):
            groups.setdefault((node_doms[n], 0 if ext[n] else 1), []).append(n)
        keys = list(groups.keys())
        # original interval index: surface intervals first, each group in its comp order
        ordered0 = sorted(keys, key=functools.cmp_to_key(
            lambda a, b: (a[1] > b[1]) - (a[1] < b[1]) or _cmp_initial(a[0], b[0])))
        idx_of = {k: i for i, k in enumerate(ordered0)}
        ivals = sorted(((k[0], k[1], idx_of[k]) for k in keys), key=functools.cmp_to_key(_cmp_domains))
        self.intervals = []            # list of (domains tuple, node array sorted by ID)
        self.interval_ext = []         # True for intervals of the external-surface group
        perm = []
        for doms, grp, _ in ivals:
            nodes = np.array(sorted(groups[(doms, grp)]), dtype=np.int64)
            self.intervals.append((doms, nodes))
            self.interval_ext.append(grp == 0)
            perm.append(nodes)
        self.perm = np.concatenate(perm)                 # new index -> node ID

        # domain local node numbering
        self.dom_nodes = [[] for _ in range(self.ndomains)]
        for doms, nodes in self.intervals:
            for d in doms:
                self.dom_nodes[d].append(nodes)
        self.dom_nodes = [np.concatenate(v) if v else np.zeros(0, np.int64) for v in self.dom_nodes]
        self.g2l = []
        for d in range(self.ndomains):
            m = np.full(n_nodes, -1, dtype=np.int64)
            m[self.dom_nodes[d]] = np.arange(self.dom_nodes[d].size)
            self.g2l.append(m)

        # Dirichlet nodes per (component, interval)
        dvals = {}
        dmask = np.zeros((dpn, n_nodes), dtype=bool)
        for comp, (nodes, vals) in dirichlet.items():
            nodes = np.asarray(nodes, dtype=np.int64)
            vals = np.broadcast_to(np.asarray(vals, dtype=np.float64), nodes.shape)
            dmask[comp, nodes] = True
            for n, v in zip(nodes.tolist(), vals.tolist()):
                dvals[(comp, n)] = v
        self.dirichlet_mask = dmask

        nint = len(self.intervals)
        idir = [[nodes[dmask[c, nodes]] for (_, nodes) in self.intervals] for c in range(dpn)]

        # offsets (constraints.cpp:198-260, computeIntervalsOffsets for one rank)
        dsize = [sum(idir[c][p].size for c in range(dpn)) for p in range(nint)]
        doff, off = [], 0
        for p in range(nint):
            doff.append(off)
            off += len(self.intervals[p][0]) * dsize[p]
        self.n_dirichlet = off
        goff = []
        for p in range(nint):
            goff.append(off)
            m = len(self.intervals[p][0])
            if m > 1:
                off += (dpn * self.intervals[p][1].size - dsize[p]) * (m * (m - 1) // 2)
        self.n_lambda = off

        rows = [[] for _ in range(self.ndomains)]     # (lambda, local dof, sign, c, partner domain or -1)
        for p, (doms, nodes) in enumerate(self.intervals):
            m = len(doms)
            for k, d in enumerate(doms):
                lm = 0
                for c in range(dpn):
                    dn = idir[c][p]
                    base = doff[p] + k * dn.size + lm
                    for t, n in enumerate(dn.tolist()):
                        rows[d].append((base + t, dpn * self.g2l[d][n] + c, 1.0, dvals[(c, n)], -1, n, c))
                    lm += m * dn.size
            if m > 1:
                npairs = m * (m - 1) // 2
                for k, d in enumerate(doms):
                    cnt_ = 0
                    for c in range(dpn):
                        glued = nodes[~dmask[c, nodes]]
                        for n in glued.tolist():
                            base = goff[p] + cnt_ * npairs
                            for a in range(k):            # pairs (a,k): -1
                                rows[d].append((base + _pair(a, k, m), dpn * self.g2l[d][n] + c, -1.0, 0.0, doms[a], n, c))
                            for b in range(k + 1, m):     # pairs (k,b): +1
                                rows[d].append((base + _pair(k, b, m), dpn * self.g2l[d][n] + c, 1.0, 0.0, doms[b], n, c))
                            cnt_ += 1
        self.B = []
        for d in range(self.ndomains):
            r = np.array(rows[d], dtype=np.float64).reshape(-1, 7)
            order = np.argsort(r[:, 0], kind="stable")
            r = r[order]
            self.B.append(dict(
                lam=r[:, 0].astype(np.int64), dof=r[:, 1].astype(np.int64), sign=r[:, 2].copy(),
                c=r[:, 3].copy(), other=r[:, 4].astype(np.int64), node=r[:, 5].astype(np.int64),
                comp=r[:, 6].astype(np.int64)))
            assert np.all(np.diff(self.B[d]["lam"]) > 0)
        self.node_doms = node_doms

    def ndofs(self, d):
        return self.dpn * self.dom_nodes[d].size

    def weights(self, diags=None):
        """Duplicity weights per domain row (equalityconstraints.cpp:148-214, 287-423).

        ``diags``: per-domain stiffness diagonals (local DOF order) for K-diagonal
        scaling, or None for 1/ndomains.
        """
        out = []
        for d in range(self.ndomains):
            B = self.B[d]
            w = np.ones(B["lam"].size)
            glue = B["other"] >= 0
            if diags is None:
                for i in np.nonzero(glue)[0]:
                    w[i] = 1.0 / len(self.node_doms[B["node"][i]])
            else:
                for i in np.nonzero(glue)[0]:
                    n, c, o = B["node"][i], B["comp"][i], B["other"][i]
                    tot = sum(diags[q][self.dpn * self.g2l[q][n] + c] for q in self.node_doms[n])
                    w[i] = diags[o][self.dpn * self.g2l[o][n] + c] / tot
            out.append(w)
        return out


def _pair(a, b, m):
    """Index of pair (a,b), a<b, in the order (0,1),(0,2)..(0,m-1),(1,2).. ."""
    return a * m - a * (a + 1) // 2 + (b - a - 1)


def _cmp_initial(da, db):
    """Order of the initial interval split (arrangement.cpp:99-112): larger lists first."""
    if len(da) == len(db):
        for x, y in zip(da, db):
            if x != y:
                return -1 if x < y else 1
        return 0
    return -1 if len(da) > len(db) else 1
