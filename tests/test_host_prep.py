"""Host preprocessing of the library (C++, no GPU) against the oracle.

* integer maps (multiplier index, local DOF, sign, local node order) are
  bit-exact against the oracle's restatement of ESPRESO's numbering;
* B1 scaling weights and Dirichlet values match;
* the algebraic kernels span ker K; P F P is independent of the generalised
  inverse, so the library's explicit S_i give the oracle's projected operator;
* the oracle's PCG driven by the library's S_i, R_i and K^+ reproduces the
  oracle's own displacements and a direct solve.
"""
import numpy as np
import pytest

from espreso_b200 import feti4i as F
from espreso_b200 import problems
from oracle import feti as OF

from helpers import direct_u, oracle_problem, with_library_operators

CASES = {
    "elast_2x2x2": lambda: problems.elasticity_cube(domains=(2, 2, 2), elements=(3, 3, 3)),
    "elast_3x2x1": lambda: problems.elasticity_cube(domains=(3, 2, 1), elements=(2, 3, 4)),
    "heat_3x3x2": lambda: problems.heat_cube(domains=(3, 3, 2), elements=(3, 2, 3), seed=3),
    "elast_clusters": lambda: problems.elasticity_cube(clusters=(2, 1, 1), domains=(1, 2, 2), elements=(2, 2, 2)),
}


def host_instance(P, prec=F.PREC_LUMPED, scaling=1):
    return problems.make_instance(P, iopts={F.PRECONDITIONER: prec, F.VERBOSE_LEVEL: 0},
                                  ext={F.EXT_HOST_ONLY: 1, F.EXT_SCALING: scaling})


@pytest.mark.parametrize("case", sorted(CASES))
def test_maps_bit_exact(case):
    P = CASES[case]()
    inst = host_instance(P)
    OP = oracle_problem(P)
    num = OP.num
    st = inst.stats()
    assert int(st["dual_size"]) == num.n_lambda
    assert int(st["subdomains"]) == num.ndomains
    for d in range(num.ndomains):
        m = inst.multipliers(d)
        B = num.B[d]
        assert np.array_equal(m["lam"], B["lam"])
        assert np.array_equal(m["dof"], B["dof"])
        assert np.array_equal(m["sign"], B["sign"])
        assert np.array_equal(m["c"], B["c"])
        np.testing.assert_allclose(m["w"], OP.sub[d].w, rtol=1e-14, atol=0)
        nodes = inst.nodes(d)[: num.dom_nodes[d].size]
        assert np.array_equal(nodes, num.dom_nodes[d])
    inst.destroy()


def test_unscaled_weights():
    P = CASES["elast_3x2x1"]()
    inst = host_instance(P, scaling=0)
    OP = oracle_problem(P, scaling=False)
    for d in range(OP.num.ndomains):
        np.testing.assert_allclose(inst.multipliers(d)["w"], OP.sub[d].w, rtol=1e-15)
    inst.destroy()


@pytest.mark.parametrize("case", ["elast_2x2x2", "heat_3x3x2"])
def test_kernel_and_projected_operator(case):
    P = CASES[case]()
    inst = host_instance(P)
    OP = oracle_problem(P)
    for d, s in enumerate(OP.sub):
        R = inst.kernel(d)
        assert R.shape[1] == s.R.shape[1]
        KR = s.K @ R
        assert np.linalg.norm(KR) <= 1e-9 * abs(s.K).max() * np.sqrt(R.shape[0])
        # same column space as the analytic kernel
        Q, _ = np.linalg.qr(s.R)
        assert np.linalg.norm(R - Q @ (Q.T @ R)) < 1e-8
    rng = np.random.default_rng(0)
    x = rng.standard_normal(OP.n_lambda)
    ref = OP.projector(OP.apply_F(OP.projector(x)))
    LP = with_library_operators(oracle_problem(P), inst)
    got = LP.projector(LP.apply_F(LP.projector(x)))
    assert np.linalg.norm(got - ref) <= 1e-10 * np.linalg.norm(ref)
    inst.destroy()


@pytest.mark.parametrize("case,prec", [("elast_2x2x2", OF.PREC_LUMPED), ("heat_3x3x2", OF.PREC_DIRICHLET),
                                       ("elast_3x2x1", OF.PREC_NONE), ("heat_3x3x2", OF.PREC_SUPER_DIRICHLET),
                                       ("elast_2x2x2", OF.PREC_MAGIC)])
def test_host_operators_reproduce_solution(case, prec):
    P = CASES[case]()
    inst = host_instance(P, prec=prec)
    OP = oracle_problem(P, dirichlet_prec=True)
    OP.solve(precision=1e-11, prec=prec)
    u_or = OP.merge(OP.primal(), P.n_nodes)
    LP = with_library_operators(oracle_problem(P, dirichlet_prec=True), inst)
    LP.solve(precision=1e-11, prec=prec)
    u_lib = LP.merge(LP.primal(), P.n_nodes)
    ud = direct_u(P)
    assert np.linalg.norm(u_lib - u_or) <= 1e-8 * np.linalg.norm(u_or)
    assert np.linalg.norm(u_lib - ud) <= 1e-8 * np.linalg.norm(ud)
    # dual right-hand sides computed by the library equal B K^+ f - c with its own K^+
    b, e = inst.dual_rhs()
    np.testing.assert_allclose(b, LP.vec_b(), rtol=1e-10, atol=1e-12 * np.abs(b).max())
    np.testing.assert_allclose(e, LP.vec_e(), rtol=1e-10, atol=1e-12 * np.abs(e).max())
    inst.destroy()


def test_error_paths():
    P = CASES["elast_2x2x2"]()
    with pytest.raises(F.FETI4IError, match="HYBRID"):
        problems.make_instance(P, iopts={F.FETI_METHOD: 2, F.VERBOSE_LEVEL: 0}, ext={F.EXT_HOST_ONLY: 1})
    with pytest.raises(F.FETI4IError, match="PCG"):
        problems.make_instance(P, iopts={F.CGSOLVER: 3, F.VERBOSE_LEVEL: 0}, ext={F.EXT_HOST_ONLY: 1})
    with pytest.raises(F.FETI4IError, match="PRECONDITIONER"):
        problems.make_instance(P, iopts={F.PRECONDITIONER: 6, F.VERBOSE_LEVEL: 0}, ext={F.EXT_HOST_ONLY: 1})
    inst = host_instance(P)
    with pytest.raises(F.FETI4IError, match="HOST_ONLY"):
        inst.solve()
    inst.destroy()
    lib = F.load()
    lib.FETI4IDestroy(None)          # unknown handles are ignored, like the reference
    with pytest.raises(F.FETI4IError, match="invalid instance"):
        inst.stats()


def test_default_options():
    io, ro = F.default_options()
    assert io.tolist() == [4, 200, 0, 3, 0, 2, 1, 0, 0, 200]
    assert ro.tolist() == [1e-5]


def test_single_element_calls_equal_batched():
    P = problems.elasticity_cube(domains=(2, 1, 1), elements=(2, 2, 2))
    a = problems.make_instance(P, iopts={F.VERBOSE_LEVEL: 0}, ext={F.EXT_HOST_ONLY: 1}, batched=True)
    b = problems.make_instance(P, iopts={F.VERBOSE_LEVEL: 0}, ext={F.EXT_HOST_ONLY: 1}, batched=False)
    for d in range(2):
        np.testing.assert_array_equal(a.schur(d), b.schur(d))
    a.destroy()
    b.destroy()


def test_update_rhs_and_dirichlet():
    P = CASES["elast_2x2x2"]()
    inst = host_instance(P)
    b0, e0 = inst.dual_rhs()
    inst.update_rhs(2.0 * P.rhs())
    b1, e1 = inst.dual_rhs()
    np.testing.assert_allclose(b1, 2.0 * b0, rtol=1e-12, atol=1e-30)
    np.testing.assert_allclose(e1, 2.0 * e0, rtol=1e-12, atol=1e-30)
    dd, dv = P.dirichlet_dofs()
    inst.update_dirichlet(dd, np.full(dd.size, 1e-3))
    for d in range(int(inst.stats()["subdomains"])):
        m = inst.multipliers(d)
        dir_rows = m["c"] != 0
        assert np.all(m["c"][dir_rows] == 1e-3)
    inst.destroy()


def test_update_matrix_scaled():
    """FETI4IUpdateStiffnessMatrixScaled: K_e := s_e K_e of a matrix object, decomposition kept;
    the result equals an instance built from the scaled element matrices."""
    P = CASES["elast_2x2x2"]()
    rng = np.random.default_rng(4)
    scale = rng.uniform(0.5, 2.0, P.elem_nodes.shape[0])
    unit = F.Matrix(0)
    unit.add_elements(P.elem_nodes, P.elem_dofs(), P.Ke)
    unit.set_partition(P.elem_domain)
    inst = host_instance(P)
    inst.update_matrix_scaled(unit, scale)
    scaled = problems.elasticity_cube(domains=(2, 2, 2), elements=(3, 3, 3))
    scaled.Ke = P.Ke * scale[:, None, None]
    ref = host_instance(scaled)
    for d in range(int(ref.stats()["subdomains"])):
        np.testing.assert_allclose(inst.schur(d), ref.schur(d), rtol=1e-12, atol=1e-12 * np.abs(ref.schur(d)).max())
        np.testing.assert_array_equal(inst.multipliers(d)["lam"], ref.multipliers(d)["lam"])
    with pytest.raises(F.FETI4IError, match="one scale per stored element"):
        inst.update_matrix_scaled(unit, scale[:-1])
    unit.destroy()
    inst.destroy()
    ref.destroy()


def test_per_instance_extended_options():
    """FETI4ISetExtendedOptions changes one instance only; the process-wide defaults stay."""
    P = CASES["elast_3x2x1"]()
    a = host_instance(P)
    b = host_instance(P)
    b.set_extended(F.EXT_SCALING, 0)      # preparation-dependent: redone with the decomposition kept
    OP = oracle_problem(P, scaling=False)
    OS = oracle_problem(P, scaling=True)
    for d in range(OP.num.ndomains):
        np.testing.assert_allclose(b.multipliers(d)["w"], OP.sub[d].w, rtol=1e-15)
        np.testing.assert_allclose(a.multipliers(d)["w"], OS.sub[d].w, rtol=1e-14)
    b.set_extended(F.EXT_RELIABLE_DELTA, 0.05)   # solve-only option (no device solver on a host-only instance)
    with pytest.raises(F.FETI4IError, match="unknown extended option"):
        b.set_extended(99, 1)
    c = host_instance(P)                  # new instances still take the defaults
    for d in range(OP.num.ndomains):
        np.testing.assert_allclose(c.multipliers(d)["w"], OS.sub[d].w, rtol=1e-14)
    for i in (a, b, c):
        i.destroy()
