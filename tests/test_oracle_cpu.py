"""The OpenMP C++ restatement of Solve_RegCG (oracle/cpu_pcg.cpp) against the numpy oracle, and the
oracle's SUPER_DIRICHLET / MAGIC preconditioners and global-load split against a direct solve (CPU)."""
import numpy as np
import pytest

from espreso_b200 import problems
from oracle import cpu as OC
from oracle import feti as OF
from oracle import numbering as ON
from tests.helpers import direct_u

CASES = {
    "elast": lambda: problems.elasticity_cube(domains=(2, 2, 2), elements=(3, 3, 3)),
    "heat": lambda: problems.heat_cube(domains=(3, 2, 2), elements=(3, 3, 3)),
}


def _oracle(P):
    num = ON.Numbering(P.elem_nodes, P.elem_domain, P.n_nodes, P.dpn, P.dirichlet)
    return OF.FETIProblem(num, P.elem_nodes, P.elem_domain, P.Ke, P.fe, P.coords, build_dirichlet=True)


@pytest.fixture(scope="module", params=sorted(CASES))
def case(request):
    P = CASES[request.param]()
    return P, _oracle(P)


@pytest.mark.parametrize("prec", [OF.PREC_NONE, OF.PREC_LUMPED, OF.PREC_WEIGHT, OF.PREC_DIRICHLET,
                                  OF.PREC_SUPER_DIRICHLET, OF.PREC_MAGIC])
def test_cpp_pcg_matches_numpy_oracle(case, prec):
    P, OP = case
    lam = OP.solve(precision=1e-10, prec=prec).copy()
    it, alpha = OP.iterations, OP.alpha.copy()
    C = OC.CpuPCG(OP, prec, threads=2)
    lam2, alpha2 = C.solve(precision=1e-10, max_it=1000)
    assert abs(C.iterations - it) <= 1
    assert np.linalg.norm(lam2 - lam) <= 1e-9 * np.linalg.norm(lam)
    assert np.linalg.norm(alpha2 - alpha) <= 1e-8 * max(np.linalg.norm(alpha), 1e-300)
    u = OP.merge(OP.primal(lam2, alpha2), P.n_nodes)
    ud = direct_u(P)
    assert np.linalg.norm(u - ud) <= 1e-8 * np.linalg.norm(ud)


@pytest.mark.parametrize("prec", [OF.PREC_SUPER_DIRICHLET, OF.PREC_MAGIC])
def test_new_preconditioners_converge_faster_than_none(case, prec):
    """SUPER_DIRICHLET (diagonal K_rr) lies between LUMPED and DIRICHLET; MAGIC is LUMPED's operator."""
    P, OP = case
    OP.solve(precision=1e-8, prec=OF.PREC_NONE)
    it_none = OP.iterations
    lam = OP.solve(precision=1e-8, prec=prec).copy()
    it = OP.iterations
    assert it < it_none
    if prec == OF.PREC_MAGIC:
        lam_l = OP.solve(precision=1e-8, prec=OF.PREC_LUMPED)
        assert OP.iterations == it
        assert np.linalg.norm(lam_l - lam) <= 1e-12 * np.linalg.norm(lam)


def test_super_dirichlet_operator_definition(case):
    """S_sd = K_ss - K_sr diag(K_rr)^-1 K_rs, symmetric, built densely here."""
    P, OP = case
    s = OP.sub[0]
    K = s.K.toarray()
    t = s.tdofs
    r = np.setdiff1d(np.arange(K.shape[0]), t)
    ref = K[np.ix_(t, t)] - K[np.ix_(t, r)] @ np.diag(1.0 / np.diag(K)[r]) @ K[np.ix_(r, t)]
    Ssd = s.Ssd.toarray()
    assert np.allclose(Ssd, Ssd.T, atol=1e-12 * np.abs(ref).max())
    assert np.abs(Ssd - ref).max() <= 1e-12 * np.abs(ref).max()


def test_global_load_split(case):
    """A global load vector split by node multiplicity gives the same displacements."""
    P, OP = case
    OP.set_rhs(P.rhs())
    C = OC.CpuPCG(OP, OF.PREC_LUMPED)
    lam, alpha = C.solve(precision=1e-11)
    u = OP.merge(OP.primal(lam, alpha), P.n_nodes)
    ud = direct_u(P)
    assert np.linalg.norm(u - ud) <= 1e-8 * np.linalg.norm(ud)


def test_espreso_truncate():
    """FETISolver.cpp:130-147: 1 / precision places relative to 10^ceil(log10 max|u|)."""
    dp = 1.0 / 1e-5          # the reference divides by the precision in double, as here
    u = np.array([0.123456789, -0.0004567, 0.0])
    np.testing.assert_array_equal(OF.espreso_truncate(u, 1e-5), np.trunc(dp * u) / dp)
    v = np.array([123.456789, -0.5])
    dv = dp / 1000.0         # max|v| = 123.5: 10^ceil(log10) = 1000
    np.testing.assert_array_equal(OF.espreso_truncate(v, 1e-5), np.trunc(dv * v) / dv)
    assert abs(OF.espreso_truncate(v, 1e-5)[0] - 123.45) < 1e-12
