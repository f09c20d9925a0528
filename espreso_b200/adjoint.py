"""Differentiable FETI solve: per-element material parameter rho -> displacements u.

``FetiSolve`` is a ``torch.autograd.Function`` over the FETI4I C ABI:

* forward: element matrices K_e = E(rho_e) * K_e^unit in one FETI4I instance (kept between calls:
  the library rescales the unit matrices, repeats the subdomain factorisations and explicit Schur
  complements on the GPU), one GPU dual solve -> u;
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
                 precond=F.PREC_LUMPED, precision=1e-10, max_it=2000, device_prep=True, reuse=True):
        self.P = problem
        self.reuse = reuse
        self._inst = None   # persistent instance (reuse)
        self._unit = None   # unit-modulus element matrices in the library (reuse)
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
        """A FETI4I instance of K(rho).  With ``reuse`` (default) one instance serves every call: the
        unit-modulus element matrices are passed once and each call rescales them in the library
        (FETI4IUpdateStiffnessMatrixScaled keeps the decomposition and repeats the factorisations
        and Schur complements); otherwise every call builds a new matrix and instance."""
        E = self.modulus(rho)
        if self.reuse and self._inst is not None:
            inst = self._inst
            inst.update_dirichlet(self.dd, self.dv)
            inst.update_rhs(self.f)
            inst.update_matrix_scaled(self._unit, E)
            return inst
        F.set_extended(F.EXT_DEVICE_PREP, 1 if self.device_prep else 0)
        try:
            if self.reuse:
                self._unit = F.Matrix(0)
                self._unit.add_elements(self.P.elem_nodes, self.P.elem_dofs(), self.K_unit)
                self._unit.set_partition(self.P.elem_domain)
                M = F.Matrix(0)
                M.add_elements(self.P.elem_nodes, self.P.elem_dofs(), self.K_unit * E[:, None, None])
                M.set_partition(self.P.elem_domain)
                try:
                    self._inst = F.Instance(M, self.f, self.dd, self.dv, iopts=self.iopts, ropts=self.ropts)
                finally:
                    M.destroy()
                return self._inst
            M = F.Matrix(0)
            M.add_elements(self.P.elem_nodes, self.P.elem_dofs(), self.K_unit * E[:, None, None])
            M.set_partition(self.P.elem_domain)
            try:
                return F.Instance(M, self.f, self.dd, self.dv, iopts=self.iopts, ropts=self.ropts)
            finally:
                M.destroy()
        finally:
            F.set_extended(F.EXT_DEVICE_PREP, 1)

    def release(self, inst):
        """End of one forward/backward: instances of the model persist, others are destroyed."""
        if inst is not self._inst:
            inst.destroy()

    def close(self):
        if self._inst is not None:
            self._inst.destroy()
            self._inst = None
        if self._unit is not None:
            self._unit.destroy()
            self._unit = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def solve(self, rho):
        inst = self.instance(np.asarray(rho, dtype=np.float64))
        try:
            return inst.solve()
        finally:
            self.release(inst)


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
            model.release(inst)
        E = model.modulus(ctx.rho)
        grad = -(model.dmodulus(ctx.rho) / E) * energies
        return torch.from_numpy(grad), None


def solve(rho: torch.Tensor, model: SIMPModel) -> torch.Tensor:
    return FetiSolve.apply(rho, model)
