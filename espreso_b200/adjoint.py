"""Differentiable FETI solve: per-element material parameter rho -> displacements u.

``FetiSolve`` is a ``torch.autograd.Function`` over the FETI4I C ABI:

* forward: element matrices K_e = E(rho_e) * K_e^unit, one FETI4I instance
  (host factorisation + explicit Schur complements), one GPU dual solve -> u;
* backward: the SAME instance solves the adjoint problem K v = dL/du with zero
  Dirichlet values (FETI4IUpdateRhs / FETI4IUpdateDirichlet reuse the factors
  and the Schur complements), then the GPU element kernel
  (FETI4IElementEnergies) gives v_e^T K_e u_e and
  dL/drho_e = -(E'(rho_e) / E(rho_e)) * v_e^T K_e u_e.

u is kept from the forward solve (no per-iteration PCG state is stored).
"""
from __future__ import annotations

import numpy as np
import torch

from . import feti4i as F
from . import problems


class SIMPModel:
    """E(rho) = E_min + rho^p (E0 - E_min) on a fixed mesh with unit-modulus element matrices."""

    def __init__(self, problem: problems.Problem, K_unit, E0=2.1e11, E_min=1e-9, p=3.0, rhs=None,
                 precond=F.PREC_LUMPED, precision=1e-10, max_it=2000, device_prep=True):
        self.P = problem
        self.device_prep = device_prep   # subdomain factorisations and S_i on the GPU (FETI4I_EXT_DEVICE_PREP)
        self.K_unit = np.ascontiguousarray(K_unit, dtype=np.float64)   # (E, nd, nd)
        self.E0, self.E_min, self.p = E0, E_min, p
        self.f = problem.rhs() if rhs is None else np.asarray(rhs, dtype=np.float64)
        self.dd, self.dv = problem.dirichlet_dofs()
        self.iopts = {F.PRECONDITIONER: precond, F.VERBOSE_LEVEL: 0, F.MAX_ITERATIONS: max_it}
        self.ropts = {F.PRECISION: precision}

    def modulus(self, rho):
        return self.E_min + rho ** self.p * (self.E0 - self.E_min)

    def dmodulus(self, rho):
        return self.p * rho ** (self.p - 1) * (self.E0 - self.E_min)

    def instance(self, rho):
        E = self.modulus(rho)
        M = F.Matrix(0)
        M.add_elements(self.P.elem_nodes, self.P.elem_dofs(), self.K_unit * E[:, None, None])
        M.set_partition(self.P.elem_domain)
        F.set_extended(F.EXT_DEVICE_PREP, 1 if self.device_prep else 0)
        try:
            inst = F.Instance(M, self.f, self.dd, self.dv, iopts=self.iopts, ropts=self.ropts)
        finally:
            F.set_extended(F.EXT_DEVICE_PREP, 1)
            M.destroy()
        return inst

    def solve(self, rho):
        inst = self.instance(np.asarray(rho, dtype=np.float64))
        try:
            return inst.solve()
        finally:
            inst.destroy()


class FetiSolve(torch.autograd.Function):
    @staticmethod
    def forward(ctx, rho, model: SIMPModel):
        r = rho.detach().cpu().numpy().astype(np.float64)
        inst = model.instance(r)
        u = inst.solve()
        ctx.model = model
        ctx.inst = inst
        ctx.rho = r
        ctx.u = u
        return torch.from_numpy(u.copy())

    @staticmethod
    def backward(ctx, grad_u):
        model, inst = ctx.model, ctx.inst
        g = grad_u.detach().cpu().numpy().astype(np.float64)
        try:
            # adjoint solve with the forward factors and Schur complements
            inst.update_rhs(g)
            inst.update_dirichlet(model.dd, np.zeros(model.dd.size))
            v = inst.solve()
            energies = inst.element_energies(ctx.u, v)
        finally:
            inst.destroy()
        E = model.modulus(ctx.rho)
        grad = -(model.dmodulus(ctx.rho) / E) * energies
        return torch.from_numpy(grad), None


def solve(rho: torch.Tensor, model: SIMPModel) -> torch.Tensor:
    return FetiSolve.apply(rho, model)
