"""Total-FETI dual problem partitioned over processes (one GPU each).

The reference runs one cluster of subdomains per MPI process and exchanges the multipliers the
processes share after every F apply and preconditioner apply (All_Reduce_lambdas_compB,
src/solver/specific/itersolver.cpp:6373-6406), reduces its dot products over the processes
(parallel_ddot_compressed, :6427-6467) and gathers G x for the projector (Projector_Inv, :5541-5623).

Here every process holds one contiguous block of the subdomains on its GPU: a FETI4I instance with
FETI4I_EXT_OWNED_FIRST / OWNED_COUNT numbers the whole problem but prepares and uploads only its block
(Schur complements, factors, preconditioner).  The dual vectors are replicated on every process in the
whole problem's multiplier numbering, so the multipliers two processes share are summed by ONE
allreduce of the dual vector after each local F apply and each local preconditioner apply; the dot
products and the projector then need no collective (the coarse matrix G, a few entries per multiplier,
and the explicit (GG^T)^-1 are replicated: the allgather of G happens once, at set-up, not per
iteration).  The recurrences are Solve_RegCG's (itersolver.cpp:1406-1724).

A block is any object with the operators below (``LibraryBlock`` is the product's, on the GPU through
the FETI4I C ABI); the collectives are torch.distributed's (NCCL between GPUs, gloo between CPU
processes).  With one process the driver runs the same steps with no collective.
"""
from __future__ import annotations

import warnings

import numpy as np
import torch

from . import feti4i as F
from . import problems


def owned_range(nsub, rank, world):
    """Contiguous, balanced block of subdomains of ``rank``: [first, first + count)."""
    first = rank * nsub // world
    return first, (rank + 1) * nsub // world - first


class LibraryBlock:
    """One process's block of subdomains: a FETI4I instance over the whole mesh that prepares only
    subdomains [first, first + count) on the current CUDA device."""

    def __init__(self, problem, first, count, iopts=None, ropts=None, ext=None, precision=F.FP64):
        ext = dict(ext or {})
        ext.update({F.EXT_OWNED_FIRST: first, F.EXT_OWNED_COUNT: count})
        self.inst = problems.make_instance(problem, iopts=iopts, ropts=ropts, ext=ext)
        st = self.inst.stats()
        self.n_lambda = int(st["dual_size"])
        self.first, self.count = first, count
        self.precision = precision
        self.ndofs = problem.ndofs
        self.nk = [int(self.inst.subdomain_info(k)["nk"]) for k in range(count)]
        self.device = torch.device("cuda", torch.cuda.current_device())

    def coarse_blocks(self):
        """(global subdomain, multipliers, G_i = -(B_i R_i)^T) of the owned subdomains (cluster.cpp:2018-2159)."""
        out = []
        for k in range(self.count):
            R = self.inst.kernel(k)
            m = self.inst.multipliers(k)
            out.append((self.first + k, m["lam"].astype(np.int64), -(m["sign"][:, None] * R[m["dof"]]).T))
        return out

    def dual_rhs(self):
        """This block's part of b = sum B_i K_i^+ f_i - c, and e_i = -R_i^T f_i per owned subdomain."""
        b, e = self.inst.dual_rhs()
        ofs = np.concatenate([[0], np.cumsum(self.nk)])
        return b, {self.first + k: e[ofs[k]:ofs[k + 1]] for k in range(self.count)}

    def apply_F(self, x, y):
        """y += the block's part of F x (device tensors in the whole multiplier numbering)."""
        self.inst.apply_F_device(x.data_ptr(), y.data_ptr(), self.precision, torch.cuda.current_stream().cuda_stream)

    def precondition(self, x, y):
        self.inst.apply_prec_device(x.data_ptr(), y.data_ptr(), torch.cuda.current_stream().cuda_stream)

    def primal(self, lam, alpha_blocks):
        """The block's part of the primal solution (averaged with the whole problem's multiplicities)."""
        alpha = np.concatenate([alpha_blocks[self.first + k] for k in range(self.count)]) if self.count else np.zeros(0)
        return self.inst.primal_from_dual(lam, alpha)

    def destroy(self):
        self.inst.destroy()


class PartitionedSolver:
    """Projected PCG (Solve_RegCG) over the blocks of all processes.  ``group``: a torch.distributed
    process group, or None for one process."""

    def __init__(self, block, group=None, device=None):
        self.block = block
        self.group = group
        self.device = device if device is not None else getattr(block, "device", torch.device("cpu"))
        self.n_lambda = block.n_lambda
        self.collectives = 0
        # coarse problem: every process gathers the G blocks once and inverts G G^T itself
        blocks = block.coarse_blocks()
        if group is not None:
            import torch.distributed as dist
            gathered = [None] * dist.get_world_size(group)
            dist.all_gather_object(gathered, blocks, group=group)
            blocks = [b for part in gathered for b in part]
        blocks.sort(key=lambda t: t[0])
        self.kofs = {}
        rows, cols, vals = [], [], []
        k0 = 0
        for d, lam, G in blocks:
            self.kofs[d] = (k0, G.shape[0])
            for k in range(G.shape[0]):
                rows.append(np.full(lam.size, k0 + k))
                cols.append(lam)
                vals.append(G[k])
            k0 += G.shape[0]
        self.n_kern = k0
        r = torch.from_numpy(np.concatenate(rows))
        c = torch.from_numpy(np.concatenate(cols))
        v = torch.from_numpy(np.concatenate(vals))
        with warnings.catch_warnings():
            warnings.simplefilter("ignore", UserWarning)   # torch marks its sparse tensors as beta
            Gd = torch.sparse_coo_tensor(torch.stack([r, c]), v, (self.n_kern, self.n_lambda),
                                         check_invariants=True).coalesce()
            self.G = Gd.to_sparse_csr().to(self.device)
            self.Gt = Gd.t().coalesce().to_sparse_csr().to(self.device)
        GGt = (Gd.to_dense() @ Gd.to_dense().t()).to(self.device)
        self.GGtinv = torch.cholesky_inverse(torch.linalg.cholesky(GGt))
        # right-hand sides: b summed over the processes, e assembled from the owners' blocks
        b, eb = block.dual_rhs()
        self.b = self._sum(torch.from_numpy(np.asarray(b, dtype=np.float64)).to(self.device))
        e = np.zeros(self.n_kern)
        if group is not None:
            import torch.distributed as dist
            parts = [None] * dist.get_world_size(group)
            dist.all_gather_object(parts, eb, group=group)
            for part in parts:
                eb_all = part
                for d, v in eb_all.items():
                    o, n = self.kofs[d]
                    e[o:o + n] = v
        else:
            for d, v in eb.items():
                o, n = self.kofs[d]
                e[o:o + n] = v
        self.e = torch.from_numpy(e).to(self.device)

    # -- collectives ------------------------------------------------------------------------------
    def _sum(self, t):
        if self.group is not None:
            import torch.distributed as dist
            dist.all_reduce(t, op=dist.ReduceOp.SUM, group=self.group)
            self.collectives += 1
        return t

    def apply_F(self, x):
        y = torch.zeros_like(x)
        self.block.apply_F(x, y)
        return self._sum(y)

    def precondition(self, x):
        y = torch.zeros_like(x)
        self.block.precondition(x, y)
        return self._sum(y)

    # -- projector (Projector_Inv, itersolver.cpp:5541-5623), replicated ---------------------------
    def projector(self, x, mode=0):
        if mode == 1:
            return self.Gt @ (self.GGtinv @ x)
        a = self.GGtinv @ (self.G @ x)
        if mode == 2:
            return a
        return x - self.Gt @ a

    def solve(self, precision=1e-8, max_it=1000, prec=F.PREC_LUMPED):
        """lambda, alpha (whole numbering); sets ``iterations`` and ``converged``."""
        dot = lambda a, b: float(torch.dot(a, b))
        x = self.projector(self.e, 1)
        r = self.b - self.apply_F(x)
        u = self.projector(r)
        tol = precision * min(dot(u, u) ** 0.5, dot(self.b, self.b) ** 0.5)
        w = y = p = None
        it, norm = 0, float("inf")
        for it in range(max_it):
            wp, yp = w, y
            w = self.projector(r)
            y = w if prec == F.PREC_NONE else self.projector(self.precondition(w))
            yw = dot(y, w)
            p = y.clone() if it == 0 else y + (yw / dot(yp, wp)) * p
            Ap = self.apply_F(p)
            a = yw / dot(p, Ap)
            x = x + a * p
            r = r - a * Ap
            norm = dot(w, w) ** 0.5
            if norm < tol:
                break
        self.iterations = it + 1
        self.converged = norm < tol
        self.final_norm, self.tol = norm, tol
        self.lam = x
        self.alpha = self.projector(r, 2)
        return x, self.alpha

    def primal(self):
        """Displacements of the whole problem on every process (the blocks' parts summed)."""
        lam = self.lam.cpu().numpy()
        alpha = self.alpha.cpu().numpy()
        blocks = {d: alpha[o:o + n] for d, (o, n) in self.kofs.items()}
        u = torch.from_numpy(np.asarray(self.block.primal(lam, blocks), dtype=np.float64)).to(self.device)
        return self._sum(u).cpu().numpy()
