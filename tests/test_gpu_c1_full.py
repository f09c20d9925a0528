"""Parity at a full benchmark size: the c1 elasticity workload (unit cube, 4x4x4 subdomains of 8^3
HEXA8, 107,811 DOFs, x=0 clamped, gravity), solved through FETI4ISolve and FETI4ISolveMulti with FP64
Schur tiles and with FP32 tiles inside FP64 residual replacement, against the oracle's FP64 solve of the
same mesh and loads (its own factorisations and S_i; OpenMP C++ PCG to 1e-11) at 1e-8 relative, with
the primal residual ||(Ku - f)_free|| / ||f_free|| on the assembled system as an independent check.  A
global sparse direct solve of this size takes minutes on the host, so the residual stands in for it
here; the smaller meshes of the other tests are checked against the direct solve."""
import numpy as np
import pytest

from espreso_b200 import feti4i as F
from espreso_b200 import problems
from oracle import cpu as OC
from oracle import feti as OF
from oracle import numbering as ON

pytestmark = pytest.mark.gpu

TOL = 1e-8


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def c1():
    P = problems.build_config("c1_elasticity_64")
    num = ON.Numbering(P.elem_nodes, P.elem_domain, P.n_nodes, P.dpn, P.dirichlet)
    OP = OF.FETIProblem(num, P.elem_nodes, P.elem_domain, P.Ke, P.fe, P.coords)
    C = OC.CpuPCG(OP, OF.PREC_LUMPED)
    loads = np.concatenate([P.rhs()[None, :], problems.traction_loads(P, 3, seed=11)])
    refs = []
    for f in loads:
        OP.set_rhs(f)
        lam, alpha = C.solve(precision=1e-11, max_it=2000)
        assert C.final_norm < C.tol
        refs.append(OP.merge(OP.primal(lam, alpha), P.n_nodes).ravel())
    inst = problems.make_instance(P, iopts={F.PRECONDITIONER: F.PREC_LUMPED, F.VERBOSE_LEVEL: 0,
                                            F.MAX_ITERATIONS: 2000},
                                  ropts={F.PRECISION: TOL}, ext={F.EXT_SCHUR_PRECISION: F.FP32})
    yield P, loads, refs, inst
    inst.destroy()


@pytest.mark.parametrize("precision", [F.FP64, F.FP32])
def test_c1_single_rhs(c1, precision):
    P, loads, refs, inst = c1
    inst.set_solve_precision(precision)
    inst.update_rhs(loads[0])
    u = inst.solve()
    st = inst.stats()
    assert st["converged"] == 1.0
    assert st["dual_size"] > 40000 and st["subdomains"] == 64
    assert _rel(u, refs[0]) <= TOL
    assert P.relative_residual(u, loads[0]) <= 1e-6


@pytest.mark.parametrize("precision", [F.FP64, F.FP32])
def test_c1_multi_rhs(c1, precision):
    P, loads, refs, inst = c1
    inst.set_solve_precision(precision)
    U = inst.solve_multi(loads)
    assert inst.stats()["converged"] == 1.0
    for j in range(len(loads)):
        assert _rel(U[j], refs[j]) <= TOL, j
        assert P.relative_residual(U[j], loads[j]) <= 1e-6, j
