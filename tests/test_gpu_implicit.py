"""Implicit F apply (FETI4I_EXT_SCHUR_EXPLICIT 0): F = sum_i B_i K_i^+ B_i^T applied through the device
Cholesky factors, no S_i stored -- the reference's default dual operator
(src/solver/specific/cpu/itersolvercpu.cpp:73-106).  Against the explicit path of the same instance
data: F x to 1e-12 relative (same operator, different rounding), solves to 1e-10 against each other
and 1e-8 against a direct solve, with the iteration counts within one."""
import numpy as np
import pytest

from espreso_b200 import feti4i as F
from espreso_b200 import problems

from helpers import direct_u

pytestmark = pytest.mark.gpu


def _inst(P, explicit, prec=F.PREC_LUMPED, device_prep=1, schur=F.FP64):
    return problems.make_instance(P, iopts={F.PRECONDITIONER: prec, F.VERBOSE_LEVEL: 0, F.MAX_ITERATIONS: 1000},
                                  ropts={F.PRECISION: 1e-10},
                                  ext={F.EXT_SCHUR_EXPLICIT: explicit, F.EXT_DEVICE_PREP: device_prep,
                                       F.EXT_SCHUR_PRECISION: schur})


CASES = {
    "elast": lambda: problems.elasticity_cube(domains=(3, 3, 2), elements=(4, 4, 4)),
    "heat": lambda: problems.heat_cube(domains=(4, 3, 3), elements=(5, 5, 5), seed=1),
    "uneven": lambda: problems.uneven_cube(physics="elasticity", side=(16, 16, 16), levels=3, lo=6, hi=10, seed=2),
}


@pytest.mark.parametrize("case,prec,device_prep", [("elast", F.PREC_LUMPED, 1), ("heat", F.PREC_DIRICHLET, 1),
                                                   ("elast", F.PREC_DIRICHLET, 0), ("uneven", F.PREC_LUMPED, 1)])
def test_implicit_matches_explicit(case, prec, device_prep):
    P = CASES[case]()
    ex = _inst(P, 1, prec, device_prep)
    im = _inst(P, 0, prec, device_prep)
    n_lambda = int(ex.stats()["dual_size"])
    rng = np.random.default_rng(5)
    for _ in range(2):
        x = rng.standard_normal(n_lambda)
        ref = ex.apply_F(x, F.FP64)
        got = im.apply_F(x, F.FP64)
        assert np.linalg.norm(got - ref) <= 1e-12 * np.linalg.norm(ref)
    ue, ui = ex.solve(), im.solve()
    se, si = ex.stats(), im.stats()
    assert si["converged"] == 1.0 and abs(si["iterations"] - se["iterations"]) <= 1
    assert np.linalg.norm(ui - ue) <= 1e-10 * np.linalg.norm(ue)
    ud = direct_u(P).ravel()
    assert np.linalg.norm(ui - ud) <= 1e-8 * np.linalg.norm(ud)
    # no S_i on the device: the implicit instance holds less memory
    assert si["device_bytes"] < se["device_bytes"]
    assert si["fapply_bytes"] > 0
    assert im.time_F(F.FP64, 3) > 0
    ex.destroy()
    im.destroy()


def test_implicit_rejects_unsupported_combinations():
    P = CASES["elast"]()
    with pytest.raises(F.FETI4IError, match="FP64"):
        _inst(P, 0, schur=F.FP32)
    im = _inst(P, 0)
    with pytest.raises(F.FETI4IError, match="explicit"):
        im.solve_multi(np.stack([P.rhs(), P.rhs()]))
    im.destroy()
    Q = problems.elasticity_cube(clusters=(2, 1, 1), domains=(2, 1, 1), elements=(3, 3, 3))
    with pytest.raises(F.FETI4IError, match="Total FETI"):
        problems.make_instance(Q, iopts={F.FETI_METHOD: 1, F.VERBOSE_LEVEL: 0}, ext={F.EXT_SCHUR_EXPLICIT: 0},
                               clusters=Q.sub_cluster())
