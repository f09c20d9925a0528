"""Several load cases solved together (FETI4ISolveMulti): block PCG + tile SYMM.

Every column must equal the single right-hand-side solve and a direct solve to 1e-8,
for FP64 Schur storage and for FP32 storage with FP64 residual replacement, and for
right-hand-side counts that are padded to the SYMM width (5 -> 8) or fill it (32).
"""
import numpy as np
import pytest

from espreso_b200 import feti4i as F
from espreso_b200 import problems
from oracle import feti as OF

pytestmark = pytest.mark.gpu


def load_cases(P, nrhs, seed):
    rng = np.random.default_rng(seed)
    base = P.rhs()
    out = []
    for j in range(nrhs):
        f = base * rng.uniform(0.5, 2.0) + rng.normal(0.0, np.abs(base).max(), size=base.size) * (j % 3 == 0)
        out.append(f)
    return np.array(out)


def direct(P, f):
    K, _ = OF.global_system(P.elem_nodes, P.Ke, np.zeros((P.Ke.shape[0], P.Ke.shape[1])), P.n_nodes, P.dpn)
    dd, dv = P.dirichlet_dofs()
    return OF.direct_solve(K, f, dd, dv)


@pytest.mark.parametrize("kind,schur,nrhs,prec,tensor", [("elast", F.FP64, 5, F.PREC_LUMPED, 0),
                                                         ("elast", F.FP32, 8, F.PREC_LUMPED, 0),
                                                         ("elast", F.FP32, 8, F.PREC_LUMPED, 1),
                                                         ("heat", F.FP32, 32, F.PREC_LUMPED, 0),
                                                         ("heat", F.FP32, 32, F.PREC_LUMPED, 1),
                                                         # Schur complements of 12-16 tiles: every block
                                                         # kind of the 32-column tensor-core SYMM
                                                         ("heat_big", F.FP32, 32, F.PREC_LUMPED, 1),
                                                         # subdomains of 3,993 DOFs: the multi-column K+
                                                         # keeps its vectors in global memory
                                                         ("elast_big", F.FP32, 16, F.PREC_LUMPED, 0),
                                                         ("heat", F.FP32, 13, F.PREC_WEIGHT, 1),
                                                         ("heat", F.FP64, 3, F.PREC_NONE, 0),
                                                         ("elast", F.FP32, 8, F.PREC_DIRICHLET, 1),
                                                         ("heat", F.FP64, 6, F.PREC_DIRICHLET, 0)])
def test_multi_rhs_matches_single_and_direct(kind, schur, nrhs, prec, tensor):
    """tensor=1: FP32 SYMM on the tensor cores (tcgen05, 3xTF32) inside FP64 residual replacement."""
    if kind == "elast":
        P = problems.elasticity_cube(domains=(3, 2, 2), elements=(3, 3, 3))
    elif kind == "elast_big":
        P = problems.elasticity_cube(domains=(2, 1, 1), elements=(10, 10, 10))
    elif kind == "heat_big":
        P = problems.heat_cube(domains=(2, 2, 2), elements=(10, 10, 10), seed=3)
    else:
        P = problems.heat_cube(domains=(3, 3, 2), elements=(4, 4, 4), seed=2)
    inst = problems.make_instance(P, iopts={F.PRECONDITIONER: prec, F.VERBOSE_LEVEL: 0, F.MAX_ITERATIONS: 3000},
                                  ropts={F.PRECISION: 1e-10},
                                  ext={F.EXT_SCHUR_PRECISION: schur, F.EXT_SYMM_TENSOR: tensor})
    R = load_cases(P, nrhs, seed=nrhs)
    U = inst.solve_multi(R)
    st = inst.stats()
    assert st["converged"] == 1.0
    for j in range(nrhs):
        ud = direct(P, R[j])
        assert np.linalg.norm(U[j] - ud) <= 1e-8 * np.linalg.norm(ud), j
    # the single right-hand-side path gives the same columns
    for j in (0, nrhs - 1):
        inst.update_rhs(R[j])
        u1 = inst.solve()
        assert np.linalg.norm(U[j] - u1) <= 1e-8 * np.linalg.norm(u1)
    assert inst.solve_multi_resident(nrhs) > 0
    inst.destroy()


def test_multi_rhs_dirichlet_hybrid():
    """Dirichlet preconditioner in the block PCG (S_dir SYMM) with Hybrid Total FETI."""
    P = problems.elasticity_cube(clusters=(2, 2, 1), domains=(1, 2, 2), elements=(3, 3, 3))
    inst = problems.make_instance(P, iopts={F.PRECONDITIONER: F.PREC_DIRICHLET, F.VERBOSE_LEVEL: 0,
                                            F.FETI_METHOD: 1, F.MAX_ITERATIONS: 3000},
                                  ropts={F.PRECISION: 1e-10}, clusters=P.sub_cluster())
    R = load_cases(P, 4, 3)
    U = inst.solve_multi(R)
    for j in range(R.shape[0]):
        ud = direct(P, R[j])
        assert np.linalg.norm(U[j] - ud) <= 1e-8 * np.linalg.norm(ud)
    inst.destroy()
