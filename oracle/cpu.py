"""OpenMP C++ restatement of the dual PCG (``oracle/cpu_pcg.cpp``) driven from the numpy oracle.

Test infrastructure only (see ``oracle/__init__.py``): the tests use it as a checker at sizes the
numpy loops take too long for, and ``bench.py`` times it as the CPU baseline and as the reference
arm.  The numpy ``FETIProblem`` builds every operator (S_i, G, (GG^T)^-1, K, S_dir); the C++ code
runs Solve_RegCG (src/solver/specific/itersolver.cpp:1406-1724) over all host cores with the
packed-upper S_i SPMV of the reference's CPU path (src/solver/specific/cpu/itersolvercpu.cpp:49-70,
src/solver/generic/SparseMatrix.cpp:1057-1172).

    python -m oracle.cpu          # compile oracle/_build/liboracle_pcg.so
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np
import scipy.linalg as sla
import scipy.sparse as sp

from . import feti as OF

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "cpu_pcg.cpp")
LIB = os.path.join(HERE, "_build", "liboracle_pcg.so")


def build(force=False):
    """Compile the restatement with g++ (OpenMP, generic x86-64-v3 code so it runs on any host)."""
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= os.path.getmtime(SRC):
        return LIB
    cmd = ["g++", "-O3", "-march=x86-64-v3", "-fopenmp", "-fPIC", "-shared", "-std=c++17", SRC, "-o", LIB]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"oracle PCG build failed:\n{r.stderr}")
    return LIB


_lib = None


def _load():
    global _lib
    if _lib is None:
        _lib = ctypes.CDLL(build())
        _lib.oracle_pcg_solve.restype = ctypes.c_int
    return _lib


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None and a.size else None


def _packed_upper(A):
    """Column-major packed upper triangle (cblas_dspmv uplo 'U'): column j holds rows 0..j."""
    n = A.shape[0]
    # row i of the lower triangle of A^T is column i of the upper triangle of A, rows 0..i
    return np.ascontiguousarray(np.asarray(A, dtype=np.float64).T[np.tril_indices(n)])


class CpuPCG:
    """The dual problem of a numpy ``FETIProblem`` packed for the C++ iteration."""

    def __init__(self, OP: OF.FETIProblem, prec: int, threads: int = 0):
        self.OP = OP
        self.prec = int(prec)
        self.threads = int(threads)
        sub = OP.sub
        ni = np.array([s.lam.size for s in sub])
        self.loff = np.concatenate([[0], np.cumsum(ni)]).astype(np.int32)
        self.lam = np.concatenate([s.lam for s in sub]).astype(np.int32)
        packs = [_packed_upper(s.S) for s in sub]
        self.soff = np.concatenate([[0], np.cumsum([p.size for p in packs])]).astype(np.int64)
        self.Sp = np.concatenate(packs)
        NL = int(self.loff[-1])
        order = np.argsort(self.lam, kind="stable")
        self.l2r_row = order.astype(np.int32)
        self.l2r_ptr = np.concatenate([[0], np.cumsum(np.bincount(self.lam, minlength=OP.n_lambda))]).astype(np.int32)
        G = sp.csr_matrix(OP.G)
        Gt = sp.csr_matrix(OP.G.T)
        self.g = (G.indptr.astype(np.int32), G.indices.astype(np.int32), G.data.astype(np.float64))
        self.gt = (Gt.indptr.astype(np.int32), Gt.indices.astype(np.int32), Gt.data.astype(np.float64))
        nk = OP.n_kern
        self.GGtinv = np.ascontiguousarray(sla.cho_solve(OP.GGt_chol, np.eye(nk)))
        self.w = np.concatenate([s.w for s in sub]).astype(np.float64)
        self.sign = np.concatenate([s.sign for s in sub]).astype(np.float64)
        self.tofs = self.trow = self.m = self.doff = self.Dp = None
        if self.prec in (OF.PREC_LUMPED, OF.PREC_MAGIC, OF.PREC_DIRICHLET, OF.PREC_SUPER_DIRICHLET):
            tsets = [np.unique(s.dof) for s in sub]
            self.tofs = np.concatenate([[0], np.cumsum([t.size for t in tsets])]).astype(np.int32)
            self.trow = np.concatenate([np.searchsorted(t, s.dof) for t, s in zip(tsets, sub)]).astype(np.int32)
            if self.prec == OF.PREC_DIRICHLET:
                packs = [_packed_upper(s.Sdir) for s in sub]
                self.doff = np.concatenate([[0], np.cumsum([p.size for p in packs])]).astype(np.int64)
                self.Dp = np.concatenate(packs)
            else:
                blocks = []
                for t, s in zip(tsets, sub):
                    if self.prec == OF.PREC_SUPER_DIRICHLET:
                        blocks.append(sp.csr_matrix(s.Ssd))
                    else:   # LUMPED / MAGIC: K - RegMat = K restricted to the touched DOFs
                        blocks.append(sp.csr_matrix(s.K)[t][:, t])
                M = sp.block_diag(blocks, format="csr")
                M.sort_indices()
                self.m = (M.indptr.astype(np.int32), M.indices.astype(np.int32), M.data.astype(np.float64))
        assert NL == self.lam.size

    def solve(self, b=None, e=None, precision=1e-8, max_it=1000):
        """Solve_RegCG from b, e (default: the oracle's own vec_b / vec_e); returns lambda, alpha and
        sets ``iterations``, ``final_norm`` and ``tol``."""
        OP = self.OP
        b = np.ascontiguousarray(OP.vec_b() if b is None else b, dtype=np.float64)
        e = np.ascontiguousarray(OP.vec_e() if e is None else e, dtype=np.float64)
        lam = np.zeros(OP.n_lambda)
        alpha = np.zeros(OP.n_kern)
        stats = np.zeros(2)
        m = self.m if self.m is not None else (None, None, None)
        lib = _load()
        vp = ctypes.c_void_p
        it = lib.oracle_pcg_solve(
            ctypes.c_int(len(OP.sub)), ctypes.c_int(OP.n_lambda), ctypes.c_int(OP.n_kern), ctypes.c_int(self.prec),
            ctypes.c_int(self.threads), _ptr(self.loff), _ptr(self.lam), _ptr(self.soff), _ptr(self.Sp),
            _ptr(self.l2r_ptr), _ptr(self.l2r_row), _ptr(self.g[0]), _ptr(self.g[1]), _ptr(self.g[2]),
            _ptr(self.gt[0]), _ptr(self.gt[1]), _ptr(self.gt[2]), _ptr(self.GGtinv), _ptr(self.w), _ptr(self.sign),
            _ptr(self.tofs), _ptr(self.trow), _ptr(m[0]), _ptr(m[1]), _ptr(m[2]), _ptr(self.doff), _ptr(self.Dp),
            _ptr(b), _ptr(e), ctypes.c_double(precision), ctypes.c_int(max_it), _ptr(lam), _ptr(alpha),
            _ptr(stats))
        del vp
        self.iterations = int(it)
        self.final_norm, self.tol = float(stats[0]), float(stats[1])
        OP.lam, OP.alpha, OP.iterations = lam, alpha, self.iterations
        return lam, alpha


if __name__ == "__main__":
    print(build(force=True))
