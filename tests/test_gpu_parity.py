"""GPU parity: the sm_100a dual iteration (through the FETI4I C ABI) against the oracle.

Tolerances:
  * F apply, FP64 tiles: 1e-13 relative to the oracle's F with the same S_i
    (re-association of the FP64 sums only);
  * F apply, FP32 tiles: 1e-6; BF16 tiles with per-tile scale: 1e-2 (storage precision);
  * solves: displacements within 1e-8 relative of the oracle's FP64 solve and of
    a direct solve, for FP64 and for FP32 storage inside
    FP64 residual replacement.
"""
import numpy as np
import pytest

from espreso_b200 import feti4i as F
from espreso_b200 import problems
from oracle import feti as OF

from helpers import direct_u, oracle_problem, with_library_operators

pytestmark = pytest.mark.gpu


def gpu_instance(P, prec=F.PREC_LUMPED, precision=1e-10, schur=F.FP64, max_it=1000, tile_kernel=None):
    """tile_kernel None: autotuned; 0/1: that SYMV variant, autotuner off."""
    ext = {F.EXT_SCHUR_PRECISION: schur}
    if tile_kernel is not None:
        ext.update({F.EXT_TILE_KERNEL: tile_kernel, F.EXT_AUTOTUNE: 0})
    return problems.make_instance(P, iopts={F.PRECONDITIONER: prec, F.VERBOSE_LEVEL: 0, F.MAX_ITERATIONS: max_it},
                                  ropts={F.PRECISION: precision}, ext=ext)


@pytest.fixture(scope="module")
def elast():
    return problems.elasticity_cube(domains=(3, 3, 2), elements=(4, 4, 4))


@pytest.fixture(scope="module")
def heat():
    return problems.heat_cube(domains=(4, 3, 3), elements=(5, 5, 5), seed=1)


@pytest.mark.parametrize("tile_kernel", [0, 1])
@pytest.mark.parametrize("schur,tol", [(F.FP64, 1e-13), (F.FP32, 1e-6), (F.BF16, 2e-2)])
def test_fapply_parity(elast, schur, tol, tile_kernel):
    inst = gpu_instance(elast, schur=schur, tile_kernel=tile_kernel)
    OP = with_library_operators(oracle_problem(elast), inst)
    rng = np.random.default_rng(1)
    for _ in range(3):
        x = rng.standard_normal(OP.n_lambda)
        ref = OP.apply_F(x)
        got = inst.apply_F(x, schur)
        assert np.linalg.norm(got - ref) <= tol * np.linalg.norm(ref)
    if schur == F.FP32:
        ref32 = OP.apply_F(x, "f32")
        assert np.linalg.norm(inst.apply_F(x, schur) - ref32) <= 1e-6 * np.linalg.norm(ref32)
    inst.destroy()


def test_fapply_edge_sizes():
    """Subdomains whose interface sizes are not multiples of the 32-row tile,
    single-tile subdomains and a large multi-item subdomain."""
    P = problems.elasticity_cube(domains=(2, 1, 1), elements=(1, 1, 1))
    inst = gpu_instance(P)
    OP = with_library_operators(oracle_problem(P), inst)
    x = np.random.default_rng(2).standard_normal(OP.n_lambda)
    np.testing.assert_allclose(inst.apply_F(x), OP.apply_F(x), rtol=1e-12, atol=1e-12 * np.abs(OP.apply_F(x)).max())
    inst.destroy()
    P = problems.elasticity_cube(domains=(2, 2, 1), elements=(9, 9, 9))
    from espreso_b200.feti4i import EXT_TILES_PER_ITEM, set_extended
    set_extended(EXT_TILES_PER_ITEM, 7)
    try:
        inst = gpu_instance(P, tile_kernel=1)
    finally:
        set_extended(EXT_TILES_PER_ITEM, 48)
    OP = with_library_operators(oracle_problem(P), inst)
    x = np.random.default_rng(3).standard_normal(OP.n_lambda)
    ref = OP.apply_F(x)
    assert np.linalg.norm(inst.apply_F(x) - ref) <= 1e-13 * np.linalg.norm(ref)
    inst.destroy()


@pytest.mark.parametrize("prec,tile_kernel", [(OF.PREC_NONE, 1), (OF.PREC_LUMPED, 1), (OF.PREC_WEIGHT, 1),
                                               (OF.PREC_DIRICHLET, 1), (OF.PREC_LUMPED, 0), (OF.PREC_DIRICHLET, 0),
                                               (OF.PREC_SUPER_DIRICHLET, 0), (OF.PREC_MAGIC, 0)])
def test_solve_elasticity(elast, prec, tile_kernel):
    inst = gpu_instance(elast, prec=prec, tile_kernel=tile_kernel)
    sol = inst.solve()
    st = inst.stats()
    assert st["converged"] == 1.0
    OP = oracle_problem(elast, dirichlet_prec=True)
    OP.solve(precision=1e-10, prec=prec)
    u_or = OP.merge(OP.primal(), elast.n_nodes)
    u = sol.reshape(-1, 3)
    assert np.linalg.norm(u - u_or) <= 1e-8 * np.linalg.norm(u_or)
    ud = direct_u(elast)
    assert np.linalg.norm(u - ud) <= 1e-8 * np.linalg.norm(ud)
    # same operator -> same PCG trajectory as the oracle driven by the library's S_i
    LP = with_library_operators(oracle_problem(elast, dirichlet_prec=True), inst)
    lam_ref = LP.solve(precision=1e-10, prec=prec)
    lam, _ = inst.dual_solution()
    assert abs(LP.iterations - st["iterations"]) <= 1
    assert np.linalg.norm(lam - lam_ref) <= 1e-7 * np.linalg.norm(lam_ref)
    inst.destroy()


@pytest.mark.parametrize("prec", [F.PREC_DIRICHLET, F.PREC_SUPER_DIRICHLET])
def test_solve_heat_dirichlet(heat, prec):
    inst = gpu_instance(heat, prec=prec)
    u = inst.solve().reshape(-1, 1)
    ud = direct_u(heat)
    assert np.linalg.norm(u - ud) <= 1e-8 * np.linalg.norm(ud)
    inst.destroy()


@pytest.mark.parametrize("schur,tile_kernel", [(F.FP32, 1), (F.FP32, 0)])
def test_mixed_precision_reaches_fp64_accuracy(heat, schur, tile_kernel):
    """FP32 Schur storage inside FP64 residual replacement reaches the FP64 answer.
    (BF16 storage is a measured F-apply variant: its 8-bit mantissa makes the
    projected operator lose definiteness and the PCG diverges.)"""
    inst = gpu_instance(heat, prec=F.PREC_LUMPED, schur=schur, precision=1e-10, max_it=3000, tile_kernel=tile_kernel)
    u = inst.solve().reshape(-1, 1)
    st = inst.stats()
    assert st["converged"] == 1.0
    assert st["replacements"] >= 1
    ud = direct_u(heat)
    assert np.linalg.norm(u - ud) <= 1e-8 * np.linalg.norm(ud)
    inst.destroy()


def test_resolve_after_rhs_update(elast):
    inst = gpu_instance(elast, prec=F.PREC_DIRICHLET)
    u1 = inst.solve()
    inst.update_rhs(-3.0 * elast.rhs())
    u2 = inst.solve()
    assert np.linalg.norm(u2 + 3.0 * u1) <= 1e-8 * np.linalg.norm(u2)
    ms = inst.solve_resident()
    assert ms > 0
    inst.destroy()


def test_device_kplus_matches_host(elast):
    """FETI4ISolve runs K^+ f, b, e and the primal recovery on the device; the
    dual quantities it produces equal the host restatement with the same factors."""
    inst = gpu_instance(elast, prec=F.PREC_LUMPED)
    sol = inst.solve()
    lam, alpha = inst.dual_solution()
    LP = with_library_operators(oracle_problem(elast), inst)
    u_host = LP.merge(LP.primal(lam, alpha), elast.n_nodes)
    assert np.linalg.norm(sol.reshape(-1, 3) - u_host) <= 1e-12 * np.linalg.norm(u_host)
    inst.destroy()


def test_max_iterations_stop(elast):
    inst = gpu_instance(elast, prec=F.PREC_NONE, max_it=5)
    inst.solve()
    st = inst.stats()
    assert st["converged"] == 0.0 and st["iterations"] == 5
    inst.destroy()


def test_per_instance_schur_precision(elast):
    """Two instances in one process with different Schur storage (FETI4ISetExtendedOptions)."""
    a = gpu_instance(elast)
    b = gpu_instance(elast)
    b.set_extended(F.EXT_SCHUR_PRECISION, F.FP32)
    assert b.stats()["fapply_bytes"] < 0.6 * a.stats()["fapply_bytes"]
    ua, ub = a.solve(), b.solve()
    assert b.stats()["converged"] == 1.0 and b.stats()["replacements"] > 0
    assert np.linalg.norm(ua - ub) <= 1e-8 * np.linalg.norm(ua)
    a.destroy()
    b.destroy()


def test_reference_truncated_output(heat):
    """FETI4I_EXT_TRUNCATE: the solution formatted as the reference's FETISolver returns it (the
    oracle's espreso_truncate of the full solution, up to one truncation unit where two solves of the
    same instance differ in their last bits)."""
    inst = gpu_instance(heat, precision=1e-6)
    u = inst.solve()
    assert np.abs(u).max() > 1e-4          # several significant places survive the truncation
    inst.set_extended(F.EXT_TRUNCATE, 1)
    ut = inst.solve()
    ref = OF.espreso_truncate(u, 1e-6)
    unit = 1.0 / (1e6 / max(1.0, 10.0 ** np.ceil(np.log10(np.abs(u).max()))))
    assert np.all(np.abs(ut - ref) <= unit * (1 + 1e-9))
    assert np.mean(ut == ref) > 0.99
    assert np.all(np.abs(ut - u) <= unit)
    inst.set_extended(F.EXT_TRUNCATE, 0)
    assert np.linalg.norm(inst.solve() - u) <= 1e-9 * np.linalg.norm(u)
    inst.destroy()
