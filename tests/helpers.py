"""Shared test helpers: build the oracle for a synthetic problem, and an
oracle-driven PCG that uses the library's own host operators (S_i, R_i, K^+)."""
import numpy as np

from oracle import feti as OF
from oracle import numbering as ON


def oracle_problem(P, scaling=True, dirichlet_prec=False):
    num = ON.Numbering(P.elem_nodes, P.elem_domain, P.n_nodes, P.dpn, P.dirichlet)
    return OF.FETIProblem(num, P.elem_nodes, P.elem_domain, P.Ke, P.fe, P.coords, scaling=scaling,
                          build_dirichlet=dirichlet_prec)


def with_library_operators(OP, inst):
    """Replace the oracle's S_i, R_i and K^+ by the ones the library computed."""
    for d, s in enumerate(OP.sub):
        s.S = inst.schur(d)
        s.R = np.asarray(inst.kernel(d))
        s.kplus = (lambda v, d=d: _kplus_cols(inst, d, v))
    OP._coarse()
    return OP


def _kplus_cols(inst, d, v):
    v = np.asarray(v, dtype=np.float64)
    if v.ndim == 1:
        return inst.kplus(d, v)
    return np.stack([inst.kplus(d, v[:, j]) for j in range(v.shape[1])], axis=1)


def global_u(P, sol):
    return np.asarray(sol).reshape(-1, P.dpn)


def direct_u(P):
    K, f = OF.global_system(P.elem_nodes, P.Ke, P.fe, P.n_nodes, P.dpn)
    dd, dv = P.dirichlet_dofs()
    return OF.direct_solve(K, f, dd, dv).reshape(-1, P.dpn)
