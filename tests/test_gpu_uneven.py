"""Subdomains of uneven size from seeded recursive bisection (the uneven-decomposition
workload at a small scale): several Schur size classes in one persistent launch.

Tolerances: displacements within 1e-8 of a direct solve, FP64 tiles and FP32 tiles inside
FP64 residual replacement; F apply with FP64 tiles within 1e-13 of the oracle's F built
from the library's S_i."""
import numpy as np
import pytest

from espreso_b200 import feti4i as F
from espreso_b200 import problems
from oracle import feti as OF

from helpers import direct_u, oracle_problem, with_library_operators

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def uneven():
    return problems.uneven_cube("elasticity", side=(16, 12, 12), levels=4, lo=3, hi=9, seed=2)


def test_sizes_are_uneven(uneven):
    counts = np.bincount(uneven.elem_domain)
    assert counts.size == 16 and counts.max() >= 2 * counts.min()


@pytest.mark.parametrize("schur", [F.FP64, F.FP32])
def test_solve_uneven(uneven, schur):
    inst = problems.make_instance(uneven, iopts={F.PRECONDITIONER: F.PREC_LUMPED, F.VERBOSE_LEVEL: 0,
                                                 F.MAX_ITERATIONS: 3000},
                                  ropts={F.PRECISION: 1e-10}, ext={F.EXT_SCHUR_PRECISION: schur})
    u = inst.solve().reshape(-1, 3)
    assert inst.stats()["converged"] == 1.0
    ud = direct_u(uneven)
    assert np.linalg.norm(u - ud) <= 1e-8 * np.linalg.norm(ud)
    if schur == F.FP64:
        OP = with_library_operators(oracle_problem(uneven), inst)
        x = np.random.default_rng(0).standard_normal(OP.n_lambda)
        ref = OP.apply_F(x)
        assert np.linalg.norm(inst.apply_F(x, F.FP64) - ref) <= 1e-13 * np.linalg.norm(ref)
    inst.destroy()


def test_multi_rhs_uneven(uneven):
    """32 load cases on subdomains of different Schur sizes through the 32-column tensor-core SYMM
    (FP32 tiles, 3xTF32), where the last 32-row block of each subdomain is partial and the subdomains
    have different numbers of tile rows: the multi right-hand-side F apply agrees with the FP64
    single-vector apply to 2e-5 (FP32 storage), and every column of FETI4ISolveMulti with FP64
    residual replacement with a direct solve to 1e-8."""
    inst = problems.make_instance(uneven, iopts={F.PRECONDITIONER: F.PREC_LUMPED, F.VERBOSE_LEVEL: 0,
                                                 F.MAX_ITERATIONS: 3000},
                                  ropts={F.PRECISION: 1e-10},
                                  ext={F.EXT_SCHUR_PRECISION: F.FP32, F.EXT_SYMM_TENSOR: 1})
    nl = int(inst.stats()["dual_size"])
    X = np.random.default_rng(4).standard_normal((32, nl))
    Y = inst.apply_F_multi(X, F.FP32)
    for j in range(32):
        ref = inst.apply_F(X[j], F.FP64)
        assert np.linalg.norm(Y[j] - ref) <= 2e-5 * np.linalg.norm(ref), j
    R = problems.traction_loads(uneven, 32, seed=5) + uneven.rhs()[None, :]
    U = inst.solve_multi(R)
    assert inst.stats()["converged"] == 1.0
    K, _ = OF.global_system(uneven.elem_nodes, uneven.Ke, np.zeros((uneven.Ke.shape[0], uneven.Ke.shape[1])),
                            uneven.n_nodes, uneven.dpn)
    dd, dv = uneven.dirichlet_dofs()
    for j in range(32):
        ud = OF.direct_solve(K, R[j], dd, dv)
        assert np.linalg.norm(U[j] - ud) <= 1e-8 * np.linalg.norm(ud), j
    inst.destroy()
