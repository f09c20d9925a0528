"""ctypes binding of libfeti4i_b200.so (the FETI4I C ABI of include/feti4i.h).

The binding mirrors the reference's call sequence (src/app/apitest.cpp:6-86):
create the stiffness matrix, add elements, set options, create an instance,
solve, destroy.  Errors raised by the library surface as ``FETI4IError``
carrying FETI4IGetLastError().
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfeti4i_b200.so")

# integer options (include/feti4i.h)
SUBDOMAINS, MAX_ITERATIONS, FETI_METHOD, PRECONDITIONER, CGSOLVER, N_MICS, VERBOSE_LEVEL, MEASURE_LEVEL, \
    PRINT_MATRICES, SC_SIZE, INTEGER_OPTIONS_SIZE = range(11)
PRECISION, REAL_OPTIONS_SIZE = 0, 1
PREC_NONE, PREC_LUMPED, PREC_WEIGHT, PREC_DIRICHLET, PREC_SUPER_DIRICHLET, PREC_MAGIC = 0, 1, 2, 3, 4, 5
# extended options (include/feti4i_ext.h)
EXT_SCHUR_PRECISION, EXT_SCALING, EXT_HOST_ONLY, EXT_TILES_PER_ITEM, EXT_GRAPH_CHUNK, EXT_RELIABLE_DELTA, \
    EXT_HOST_THREADS, EXT_TILE_KERNEL, EXT_AUTOTUNE, EXT_SYMM_TENSOR, EXT_DEVICE_PREP, EXT_SCHUR_EXPLICIT, \
    EXT_OWNED_FIRST, EXT_OWNED_COUNT, EXT_TRUNCATE = range(15)
FP64, FP32, BF16 = 0, 1, 2
STAT_NAMES = ["iterations", "converged", "dual_size", "kernel_size", "subdomains", "prep_seconds",
              "upload_seconds", "solve_ms", "solve_wall_ms", "fapply_bytes", "replacements",
              "kernel_launches", "device_bytes", "final_norm", "tolerance", "elements", "prep_device_ms",
              "prep_device_flops", "kplus_tiles"]

EXPORTED = [
    "FETI4ISetDefaultIntegerOptions", "FETI4ISetDefaultRealOptions", "FETI4ICreateStiffnessMatrix",
    "FETI4IAddElement", "FETI4ICreateInstance", "FETI4ISolve", "FETI4IUpdateStiffnessMatrix",
    "FETI4IUpdateStiffnessMatrixScaled",
    "FETI4IUpdateRhs", "FETI4IUpdateDirichlet", "FETI4IDestroy",
    "FETI4IGetLastError", "FETI4ISetSubdomainPartition", "FETI4IAddElements", "FETI4ISetExtendedOption", "FETI4ISetExtendedOptions",
    "FETI4IGetStats", "FETI4IGetDualSolution", "FETI4IGetSubdomainInfo", "FETI4IGetSubdomainMultipliers",
    "FETI4IGetSubdomainNodes", "FETI4IGetSubdomainSchur", "FETI4IGetSubdomainKernel", "FETI4IGetDualRhs",
    "FETI4IApplySubdomainKplus", "FETI4IApplyDualOperator", "FETI4IApplyDualOperatorMulti", "FETI4ITimeDualOperator", "FETI4ISolveResident", "FETI4ISetSolvePrecision",
    "FETI4ITiledSymvNoAlloc", "FETI4IApplyDualOperatorDevice", "FETI4IApplyPreconditionerDevice",
    "FETI4IPrimalFromDual", "FETI4IElementEnergies", "FETI4IGetTuning", "FETI4ISolveMulti",
    "FETI4ISolveMultiResident", "FETI4ISetClusterPartition", "FETI4IGetSubdomainCorners", "FETI4IGetClusterInfo",
]


class FETI4IError(RuntimeError):
    pass


_lib = None


def load(path: str = LIB_PATH):
    """Load the in-tree library; fails loudly if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FETI4IError(f"{path} is missing: build it with `python -m espreso_b200.build`")
    lib = C.CDLL(path)
    P = C.POINTER
    i32, f64 = C.c_int, C.c_double
    pi, pd, vp = P(i32), P(f64), C.c_void_p
    sig = {
        "FETI4ISetDefaultIntegerOptions": ([pi], None),
        "FETI4ISetDefaultRealOptions": ([pd], None),
        "FETI4ICreateStiffnessMatrix": ([P(vp), i32, i32], None),
        "FETI4IAddElement": ([vp, i32, i32, pi, i32, pi, pd], None),
        "FETI4ICreateInstance": ([P(vp), vp, i32, pd, pi, i32, pi, i32, pi, pd, pi, pd], None),
        "FETI4ISolve": ([vp, i32, pd], None),
        "FETI4IUpdateStiffnessMatrix": ([vp, vp], None),
        "FETI4IUpdateStiffnessMatrixScaled": ([vp, vp, i32, pd], None),
        "FETI4IUpdateRhs": ([vp, i32, pd], None),
        "FETI4IUpdateDirichlet": ([vp, i32, pi, pd], None),
        "FETI4IDestroy": ([vp], None),
        "FETI4IGetLastError": ([], C.c_char_p),
        "FETI4ISetSubdomainPartition": ([vp, i32, pi], None),
        "FETI4IAddElements": ([vp, i32, i32, i32, pi, i32, pi, pd], None),
        "FETI4ISetExtendedOption": ([i32, f64], None),
        "FETI4ISetExtendedOptions": ([vp, i32, f64], None),
        "FETI4IGetStats": ([vp, i32, pd], None),
        "FETI4IGetDualSolution": ([vp, pd, pd], None),
        "FETI4IGetSubdomainInfo": ([vp, i32, pi], None),
        "FETI4IGetSubdomainMultipliers": ([vp, i32, pi, pi, pd, pd, pd], None),
        "FETI4IGetSubdomainNodes": ([vp, i32, pi], None),
        "FETI4IGetSubdomainSchur": ([vp, i32, pd], None),
        "FETI4IGetSubdomainKernel": ([vp, i32, pd], None),
        "FETI4IGetDualRhs": ([vp, pd, pd], None),
        "FETI4IApplySubdomainKplus": ([vp, i32, pd], None),
        "FETI4IApplyDualOperator": ([vp, i32, pd, pd], None),
        "FETI4IApplyDualOperatorMulti": ([vp, i32, i32, pd, pd], None),
        "FETI4ITimeDualOperator": ([vp, i32, i32], f64),
        "FETI4ISolveResident": ([vp], f64),
        "FETI4ISetSolvePrecision": ([vp, i32], None),
        "FETI4ITiledSymvNoAlloc": ([vp, vp, vp, vp, i32, i32, vp, vp, vp, vp], i32),
        "FETI4IApplyDualOperatorDevice": ([vp, i32, vp, vp, vp], None),
        "FETI4IApplyPreconditionerDevice": ([vp, vp, vp, vp], None),
        "FETI4IPrimalFromDual": ([vp, pd, pd, i32, pd], None),
        "FETI4IElementEnergies": ([vp, i32, pd, pd, pd], None),
        "FETI4IGetTuning": ([vp], C.c_char_p),
        "FETI4ISolveMulti": ([vp, i32, i32, pd, pd], None),
        "FETI4ISolveMultiResident": ([vp, i32], f64),
        "FETI4ISetClusterPartition": ([vp, i32, pi], None),
        "FETI4IGetSubdomainCorners": ([vp, i32, pi, pi, pd], i32),
        "FETI4IGetClusterInfo": ([vp, pi], None),
    }
    for name, (args, res) in sig.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    _lib = lib
    return lib


def _ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int))


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _check(lib):
    msg = lib.FETI4IGetLastError()
    if msg:
        raise FETI4IError(msg.decode())


def tiled_symv_noalloc(tiles, tile_offset, order, vector_offset, nmatrices, max_order, x, y, dot=0, stream=0):
    """FETI4ITiledSymvNoAlloc on caller-owned device pointers (integers); returns the status code."""
    lib = load()
    rc = lib.FETI4ITiledSymvNoAlloc(C.c_void_p(tiles), C.c_void_p(tile_offset), C.c_void_p(order),
                                    C.c_void_p(vector_offset), int(nmatrices), int(max_order), C.c_void_p(x),
                                    C.c_void_p(y), C.c_void_p(dot) if dot else None,
                                    C.c_void_p(stream) if stream else None)
    if rc != 0:
        _check(lib)
        raise FETI4IError("FETI4ITiledSymvNoAlloc failed")
    return rc


def pack_symmetric_tiles(mats):
    """Pack symmetric matrices into the 32x32 upper-tile layout of FETI4ITiledSymvNoAlloc.

    Returns (tiles float64 array, tile_offset int64, order int32)."""
    out, offs, orders = [], [], []
    total = 0
    for S in mats:
        n = S.shape[0]
        T = (n + 31) // 32
        P = np.zeros((32 * T, 32 * T))
        P[:n, :n] = S
        offs.append(total)
        orders.append(n)
        for I in range(T):
            for J in range(I, T):
                out.append(P[32 * I:32 * I + 32, 32 * J:32 * J + 32].copy())
        total += T * (T + 1) // 2
    tiles = np.stack(out).ravel() if out else np.zeros(0)
    return tiles, np.array(offs, dtype=np.int64), np.array(orders, dtype=np.int32)


def default_options():
    lib = load()
    io = np.zeros(INTEGER_OPTIONS_SIZE, dtype=np.int32)
    ro = np.zeros(REAL_OPTIONS_SIZE, dtype=np.float64)
    lib.FETI4ISetDefaultIntegerOptions(_ip(io))
    lib.FETI4ISetDefaultRealOptions(_dp(ro))
    return io, ro


def set_extended(key, value):
    lib = load()
    lib.FETI4ISetExtendedOption(int(key), float(value))
    _check(lib)


class Matrix:
    """FETI4IMatrix handle filled with element matrices."""

    def __init__(self, index_base=0):
        self.lib = load()
        self.h = C.c_void_p()
        self.lib.FETI4ICreateStiffnessMatrix(C.byref(self.h), 0, int(index_base))
        _check(self.lib)

    def add_elements(self, nodes, dofs, values, etype=3):
        nodes = np.ascontiguousarray(nodes, dtype=np.int32)
        dofs = np.ascontiguousarray(dofs, dtype=np.int32)
        values = np.ascontiguousarray(values, dtype=np.float64)
        ne = nodes.shape[0]
        self.lib.FETI4IAddElements(self.h, etype, ne, nodes.shape[1], _ip(nodes), dofs.shape[1], _ip(dofs), _dp(values))
        _check(self.lib)

    def add_element(self, nodes, dofs, values, etype=3):
        nodes = np.ascontiguousarray(nodes, dtype=np.int32)
        dofs = np.ascontiguousarray(dofs, dtype=np.int32)
        values = np.ascontiguousarray(values, dtype=np.float64)
        self.lib.FETI4IAddElement(self.h, etype, nodes.size, _ip(nodes), dofs.size, _ip(dofs), _dp(values))
        _check(self.lib)

    def set_partition(self, elem2sub):
        e = np.ascontiguousarray(elem2sub, dtype=np.int32)
        self.lib.FETI4ISetSubdomainPartition(self.h, e.size, _ip(e))
        _check(self.lib)

    def set_clusters(self, sub2cluster):
        c = np.ascontiguousarray(sub2cluster, dtype=np.int32)
        self.lib.FETI4ISetClusterPartition(self.h, c.size, _ip(c))
        _check(self.lib)

    def destroy(self):
        if self.h:
            self.lib.FETI4IDestroy(self.h)
            self.h = C.c_void_p()


class Instance:
    """FETI4IInstance handle."""

    def __init__(self, matrix: Matrix, rhs, dirichlet_dofs, dirichlet_values, iopts=None, ropts=None, l2g=None):
        self.lib = load()
        io, ro = default_options()
        if iopts:
            for k, v in iopts.items():
                io[k] = v
        if ropts:
            for k, v in ropts.items():
                ro[k] = v
        self.rhs = np.ascontiguousarray(rhs, dtype=np.float64)
        n = self.rhs.size
        l2g = np.arange(n, dtype=np.int32) if l2g is None else np.ascontiguousarray(l2g, dtype=np.int32)
        di = np.ascontiguousarray(dirichlet_dofs, dtype=np.int32)
        dv = np.ascontiguousarray(np.broadcast_to(dirichlet_values, di.shape), dtype=np.float64)
        self.h = C.c_void_p()
        self.lib.FETI4ICreateInstance(C.byref(self.h), matrix.h, n, _dp(self.rhs), _ip(l2g), 0, None,
                                      di.size, _ip(di), _dp(dv), _ip(io), _dp(ro))
        _check(self.lib)
        self.n = n

    def solve(self, out=None):
        sol = np.zeros(self.n) if out is None else out
        self.lib.FETI4ISolve(self.h, sol.size, _dp(sol))
        _check(self.lib)
        return sol

    def solve_multi(self, rhs):
        """rhs (nrhs, size) -> solutions (nrhs, size), solved together."""
        R = np.ascontiguousarray(np.atleast_2d(rhs), dtype=np.float64)
        out = np.zeros_like(R)
        self.lib.FETI4ISolveMulti(self.h, R.shape[0], R.shape[1], _dp(R), _dp(out))
        _check(self.lib)
        return out

    def solve_multi_resident(self, nrhs):
        ms = self.lib.FETI4ISolveMultiResident(self.h, int(nrhs))
        _check(self.lib)
        return ms

    def solve_resident(self):
        ms = self.lib.FETI4ISolveResident(self.h)
        _check(self.lib)
        return ms

    def set_solve_precision(self, p):
        self.lib.FETI4ISetSolvePrecision(self.h, int(p))
        _check(self.lib)

    def stats(self):
        v = np.zeros(len(STAT_NAMES))
        self.lib.FETI4IGetStats(self.h, v.size, _dp(v))
        _check(self.lib)
        return dict(zip(STAT_NAMES, v.tolist()))

    def dual_solution(self):
        st = self.stats()
        lam = np.zeros(int(st["dual_size"]))
        alp = np.zeros(int(st["kernel_size"]))
        self.lib.FETI4IGetDualSolution(self.h, _dp(lam), _dp(alp))
        _check(self.lib)
        return lam, alp

    def subdomain_info(self, d):
        info = np.zeros(4, dtype=np.int32)
        self.lib.FETI4IGetSubdomainInfo(self.h, d, _ip(info))
        _check(self.lib)
        return dict(ndofs=int(info[0]), rows=int(info[1]), nk=int(info[2]), touched=int(info[3]))

    def multipliers(self, d):
        ni = self.subdomain_info(d)["rows"]
        lam = np.zeros(ni, np.int32); dof = np.zeros(ni, np.int32)
        sign = np.zeros(ni); w = np.zeros(ni); c = np.zeros(ni)
        self.lib.FETI4IGetSubdomainMultipliers(self.h, d, _ip(lam), _ip(dof), _dp(sign), _dp(w), _dp(c))
        _check(self.lib)
        return dict(lam=lam, dof=dof, sign=sign, w=w, c=c)

    def nodes(self, d):
        n = self.subdomain_info(d)["ndofs"]
        st = self.stats()
        out = np.zeros(n, np.int32)   # upper bound (ndofs >= nodes)
        self.lib.FETI4IGetSubdomainNodes(self.h, d, _ip(out))
        _check(self.lib)
        return out

    def schur(self, d):
        ni = self.subdomain_info(d)["rows"]
        S = np.zeros((ni, ni), order="F")
        self.lib.FETI4IGetSubdomainSchur(self.h, d, S.ctypes.data_as(C.POINTER(C.c_double)))
        _check(self.lib)
        return S

    def corners(self, d):
        """HYBRID_FETI corner rows of subdomain d: (cluster row, local DOF, sign) arrays."""
        n = self.lib.FETI4IGetSubdomainCorners(self.h, d, None, None, None)
        _check(self.lib)
        rows = np.zeros(n, np.int32); dofs = np.zeros(n, np.int32); signs = np.zeros(n)
        self.lib.FETI4IGetSubdomainCorners(self.h, d, _ip(rows), _ip(dofs), _dp(signs))
        _check(self.lib)
        return dict(row=rows.astype(np.int64), dof=dofs.astype(np.int64), sign=signs)

    def cluster_info(self):
        info = np.zeros(4, dtype=np.int32)
        self.lib.FETI4IGetClusterInfo(self.h, _ip(info))
        _check(self.lib)
        return dict(method=int(info[0]), clusters=int(info[1]), corner_rows=int(info[2]), kernel_size=int(info[3]))

    def kernel(self, d):
        inf = self.subdomain_info(d)
        R = np.zeros((inf["ndofs"], inf["nk"]), order="F")
        self.lib.FETI4IGetSubdomainKernel(self.h, d, R.ctypes.data_as(C.POINTER(C.c_double)))
        _check(self.lib)
        return R

    def dual_rhs(self):
        st = self.stats()
        b = np.zeros(int(st["dual_size"])); e = np.zeros(int(st["kernel_size"]))
        self.lib.FETI4IGetDualRhs(self.h, _dp(b), _dp(e))
        _check(self.lib)
        return b, e

    def kplus(self, d, x):
        y = np.array(x, dtype=np.float64, copy=True)
        self.lib.FETI4IApplySubdomainKplus(self.h, int(d), _dp(y))
        _check(self.lib)
        return y

    def apply_F(self, x, precision=FP64):
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.zeros_like(x)
        self.lib.FETI4IApplyDualOperator(self.h, int(precision), _dp(x), _dp(y))
        _check(self.lib)
        return y

    def apply_F_multi(self, X, precision=FP64):
        """F applied to the rows of X (nrhs x dual size) by the multi right-hand-side SYMM path."""
        X = np.ascontiguousarray(X, dtype=np.float64)
        Y = np.zeros_like(X)
        self.lib.FETI4IApplyDualOperatorMulti(self.h, int(precision), int(X.shape[0]), _dp(X), _dp(Y))
        _check(self.lib)
        return Y

    def time_F(self, precision=FP64, reps=10):
        ms = self.lib.FETI4ITimeDualOperator(self.h, int(precision), int(reps))
        _check(self.lib)
        return ms

    def tuning(self):
        t = self.lib.FETI4IGetTuning(self.h)
        _check(self.lib)
        return t.decode()

    def element_energies(self, u, v):
        u = np.ascontiguousarray(u, dtype=np.float64)
        v = np.ascontiguousarray(v, dtype=np.float64)
        out = np.zeros(int(self.stats()["elements"]))
        self.lib.FETI4IElementEnergies(self.h, u.size, _dp(u), _dp(v), _dp(out))
        _check(self.lib)
        return out

    def apply_F_device(self, x_ptr, y_ptr, precision=FP64, stream=0):
        """y += (this instance's subdomains' part of F) x on caller device memory (partitioned problems)."""
        self.lib.FETI4IApplyDualOperatorDevice(self.h, int(precision), x_ptr, y_ptr, stream)
        _check(self.lib)

    def apply_prec_device(self, x_ptr, y_ptr, stream=0):
        self.lib.FETI4IApplyPreconditionerDevice(self.h, x_ptr, y_ptr, stream)
        _check(self.lib)

    def primal_from_dual(self, lam, alpha):
        """This instance's part of the solution from the whole problem's lambda and its own amplitudes."""
        lam = np.ascontiguousarray(lam, dtype=np.float64)
        alpha = np.ascontiguousarray(alpha, dtype=np.float64)
        out = np.zeros(self.n)
        self.lib.FETI4IPrimalFromDual(self.h, _dp(lam), _dp(alpha), out.size, _dp(out))
        _check(self.lib)
        return out

    def set_extended(self, key, value):
        """Extended option of this instance only (FETI4ISetExtendedOptions)."""
        self.lib.FETI4ISetExtendedOptions(self.h, int(key), float(value))
        _check(self.lib)

    def update_rhs(self, rhs):
        r = np.ascontiguousarray(rhs, dtype=np.float64)
        self.lib.FETI4IUpdateRhs(self.h, r.size, _dp(r))
        _check(self.lib)

    def update_dirichlet(self, dofs, values):
        di = np.ascontiguousarray(dofs, dtype=np.int32)
        dv = np.ascontiguousarray(np.broadcast_to(values, di.shape), dtype=np.float64)
        self.lib.FETI4IUpdateDirichlet(self.h, di.size, _ip(di), _dp(dv))
        _check(self.lib)

    def update_matrix(self, matrix: Matrix):
        self.lib.FETI4IUpdateStiffnessMatrix(self.h, matrix.h)
        _check(self.lib)

    def update_matrix_scaled(self, matrix: Matrix, scale):
        """K_e := scale[e] * K_e of ``matrix`` (FETI4IUpdateStiffnessMatrixScaled)."""
        sc = np.ascontiguousarray(scale, dtype=np.float64)
        self.lib.FETI4IUpdateStiffnessMatrixScaled(self.h, matrix.h, int(sc.size), _dp(sc))
        _check(self.lib)

    def destroy(self):
        if self.h:
            self.lib.FETI4IDestroy(self.h)
            self.h = C.c_void_p()
