"""Hybrid Total FETI host preprocessing against the oracle (no GPU).

* corner rows B0 (cluster row, local DOF, sign) are bit-exact with the oracle's
  restatement of fetidata.cpp:146-188 and equalityconstraints.cpp:504-555;
* the dual right-hand side b = B1 K_c^+ f - c built with the library's cluster solve
  equals the oracle's with the same subdomain K^+ and kernels (1e-10);
* the dual kernel space has one block per cluster.
"""
import numpy as np
import pytest

from espreso_b200 import feti4i as F
from espreso_b200 import problems
from oracle import htfeti as OH
from oracle import numbering as ON

from helpers import with_library_operators

CASES = {
    "heat_3x2x1": problems.heat_cube(clusters=(3, 2, 1), domains=(1, 2, 3), elements=(4, 3, 4), seed=0),
    "elast_2x2x1": problems.elasticity_cube(clusters=(2, 2, 1), domains=(1, 2, 2), elements=(3, 3, 3)),
}


def host_instance(P, clusters, prec=F.PREC_LUMPED):
    return problems.make_instance(P, iopts={F.FETI_METHOD: 1, F.VERBOSE_LEVEL: 0, F.PRECONDITIONER: prec},
                                  ext={F.EXT_HOST_ONLY: 1}, clusters=clusters)


def oracle(P, clusters):
    num = ON.Numbering(P.elem_nodes, P.elem_domain, P.n_nodes, P.dpn, P.dirichlet)
    return OH.HTFETIProblem(num, P.elem_nodes, P.elem_domain, P.Ke, P.fe, P.coords, clusters)


@pytest.mark.parametrize("name", list(CASES))
def test_corners_bit_exact(name):
    P = CASES[name]
    cl = P.sub_cluster()
    inst = host_instance(P, cl)
    OP = oracle(P, cl)
    for d in range(len(OP.sub)):
        got = inst.corners(d)
        for key in ("row", "dof", "sign"):
            np.testing.assert_array_equal(got[key], OP.B0[d][key])
    info = inst.cluster_info()
    assert info["method"] == 1 and info["clusters"] == int(cl.max()) + 1
    assert info["corner_rows"] == sum(OP.n0)
    assert info["kernel_size"] == OP.n_kern
    inst.destroy()


@pytest.mark.parametrize("name", list(CASES))
def test_dual_rhs_matches_oracle(name):
    P = CASES[name]
    cl = P.sub_cluster()
    inst = host_instance(P, cl)
    OP = with_library_operators(oracle(P, cl), inst)
    b, e = inst.dual_rhs()
    bo = OP.vec_b()
    assert np.linalg.norm(b - bo) <= 1e-10 * np.linalg.norm(bo)
    # e depends on the basis chosen for each cluster kernel; its norm per cluster does not
    eo = OP.vec_e()
    for c in range(len(OP.cl)):
        sl = slice(OP.kofs[c], OP.kofs[c + 1])
        assert abs(np.linalg.norm(e[sl]) - np.linalg.norm(eo[sl])) <= 1e-10 * max(1.0, np.linalg.norm(eo[sl]))
    inst.destroy()


def test_single_cluster_default():
    """HYBRID_FETI without a cluster partition: one cluster, as one reference process."""
    P = CASES["heat_3x2x1"]
    inst = problems.make_instance(P, iopts={F.FETI_METHOD: 1, F.VERBOSE_LEVEL: 0}, ext={F.EXT_HOST_ONLY: 1})
    info = inst.cluster_info()
    assert info["clusters"] == 1 and info["kernel_size"] == 1
    OP = oracle(P, np.zeros(int(P.elem_domain.max()) + 1, dtype=np.int64))
    for d in range(len(OP.sub)):
        np.testing.assert_array_equal(inst.corners(d)["row"], OP.B0[d]["row"])
    inst.destroy()


def test_cluster_partition_errors():
    P = CASES["heat_3x2x1"]
    with pytest.raises(F.FETI4IError, match="cluster partition"):
        host_instance(P, np.zeros(3, dtype=np.int32))
    # TOTAL_FETI ignores a cluster partition
    inst = problems.make_instance(P, iopts={F.FETI_METHOD: 0, F.VERBOSE_LEVEL: 0}, ext={F.EXT_HOST_ONLY: 1},
                                  clusters=P.sub_cluster())
    assert inst.cluster_info()["method"] == 0
    inst.destroy()


def test_uneven_subdomains_prepare():
    """Recursive-bisection subdomains of uneven shape (thin slabs included) get fix nodes
    that remove every rigid-body mode."""
    for seed in range(6):
        for phys in ("elasticity", "heat"):
            P = problems.uneven_cube(phys, side=(16, 12, 12), levels=4, lo=3, hi=9, seed=seed)
            inst = problems.make_instance(P, iopts={F.VERBOSE_LEVEL: 0}, ext={F.EXT_HOST_ONLY: 1})
            st = inst.stats()
            assert st["subdomains"] == 16
            assert st["kernel_size"] == 16 * (6 if phys == "elasticity" else 1)
            inst.destroy()
