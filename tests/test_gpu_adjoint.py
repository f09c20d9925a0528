"""Adjoint sensitivities through torch.autograd.Function over the FETI4I C ABI.

Loss L = f^T u + 1/2 u^T Q u (Q seeded diagonal); E_e = 1e-9 + rho_e^3 (2.1e11 - 1e-9).
Checked against (1) an FP64 CPU adjoint with direct sparse solves (oracle) to
1e-7 relative, and (2) central finite differences (h = 1e-6) of the library's
own forward solves on 64 seeded elements to 1e-5 relative.
"""
import numpy as np
import pytest
import torch

from espreso_b200 import adjoint, problems
from oracle import feti as OF

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup():
    P, rho, f = problems.adjoint_cube(domains=(2, 2, 2), elements=(3, 3, 3), seed=5)
    model = adjoint.SIMPModel(P, P.Ke, rhs=f, precision=1e-13, max_it=5000)
    q = np.random.default_rng(9).uniform(0.0, 1e10, size=P.ndofs)
    return P, rho, f, model, q


def loss_np(u, f, q):
    return float(f @ u + 0.5 * np.sum(q * u * u))


def test_adjoint_vs_cpu_adjoint_and_fd(setup):
    P, rho, f, model, q = setup
    r = torch.tensor(rho, dtype=torch.float64, requires_grad=True)
    u = adjoint.solve(r, model)
    L = torch.dot(torch.from_numpy(f), u) + 0.5 * torch.sum(torch.from_numpy(q) * u * u)
    L.backward()
    g = r.grad.numpy()
    # FP64 CPU adjoint (oracle): direct solves of K u = f, K v = dL/du with zero Dirichlet values
    E = model.modulus(rho)
    Ke = P.Ke * E[:, None, None]
    K, _ = OF.global_system(P.elem_nodes, Ke, np.zeros((Ke.shape[0], Ke.shape[1])), P.n_nodes, 3)
    dd, dv = P.dirichlet_dofs()
    u_ref = OF.direct_solve(K, f, dd, dv)
    assert np.linalg.norm(u.detach().numpy() - u_ref) <= 1e-9 * np.linalg.norm(u_ref)
    v_ref = OF.direct_solve(K, f + q * u_ref, dd, np.zeros(dd.size))
    edofs = P.elem_dofs()
    en = np.einsum("ea,eab,eb->e", v_ref[edofs], Ke, u_ref[edofs])
    g_ref = -(model.dmodulus(rho) / E) * en
    assert np.linalg.norm(g - g_ref) <= 1e-7 * np.linalg.norm(g_ref)
    # central finite differences of the library's forward solves
    h = 1e-6
    idx = np.random.default_rng(11).choice(rho.size, size=64, replace=False)
    for i in idx:
        rp, rm = rho.copy(), rho.copy()
        rp[i] += h
        rm[i] -= h
        fd = (loss_np(model.solve(rp), f, q) - loss_np(model.solve(rm), f, q)) / (2 * h)
        assert abs(fd - g[i]) <= 1e-5 * np.abs(g).max(), (i, fd, g[i])
