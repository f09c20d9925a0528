"""The FETI4I ABI from C: a plain C caller (tests/c/feti4i_caller.c, the call sequence of the reference's
apitest) compiled with gcc against include/feti4i.h and the single-process include/mpi.h stand-in, for
FETI4I_INT_WIDTH 32 (libfeti4i_b200.so) and 64 (libfeti4i_b200_i64.so).  Without a GPU it runs the host
preparation and returns b and the multipliers of subdomain 0, which must equal the Python binding's
bit for bit; on a GPU it solves and must match the binding's solution."""
import os
import subprocess

import numpy as np
import pytest

from espreso_b200 import feti4i as F
from espreso_b200 import problems

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "espreso_b200")


def _compile(width, tmp):
    exe = os.path.join(tmp, f"caller{width}")
    lib = "feti4i_b200" if width == 32 else "feti4i_b200_i64"
    cmd = ["gcc", "-std=c99", "-Wall", "-Werror", f"-DFETI4I_INT_WIDTH={width}", "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "c", "feti4i_caller.c"), "-o", exe, f"-L{LIBDIR}", f"-l{lib}",
           f"-Wl,-rpath,{LIBDIR}"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe


def _problem_file(P, path):
    dofs = P.elem_dofs()
    dd, dv = P.dirichlet_dofs()
    with open(path, "wb") as fh:
        hdr = np.array([P.elem_nodes.shape[0], 8, dofs.shape[1], P.ndofs, dd.size, int(P.elem_domain.max()) + 1])
        hdr.astype(np.int64).tofile(fh)
        for a in (P.elem_nodes, dofs, P.elem_domain, dd):
            np.asarray(a, dtype=np.int64).tofile(fh)
        for a in (P.Ke, P.rhs(), dv):
            np.asarray(a, dtype=np.float64).tofile(fh)


@pytest.fixture(scope="module")
def setup(tmp_path_factory):
    tmp = str(tmp_path_factory.mktemp("ccaller"))
    P = problems.elasticity_cube(domains=(2, 2, 1), elements=(3, 2, 3))
    path = os.path.join(tmp, "problem.bin")
    _problem_file(P, path)
    return P, path, tmp, {w: _compile(w, tmp) for w in (32, 64)}


@pytest.mark.parametrize("width", [32, 64])
def test_c_caller_host_preparation(setup, width):
    P, path, tmp, exe = setup
    out = os.path.join(tmp, f"host{width}.bin")
    r = subprocess.run([exe[width], path, out, "host"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    inst = problems.make_instance(P, iopts={F.PRECONDITIONER: F.PREC_LUMPED, F.VERBOSE_LEVEL: 0},
                                  ext={F.EXT_HOST_ONLY: 1})
    b, _ = inst.dual_rhs()
    lam = inst.multipliers(0)["lam"]
    inst.destroy()
    got = np.fromfile(out, dtype=np.float64)
    assert got.size == b.size + lam.size
    assert np.array_equal(got[:b.size], b)
    assert np.array_equal(got[b.size:].astype(np.int64), lam)


def test_int64_library_rejects_indices_beyond_32_bits():
    import ctypes
    lib = ctypes.CDLL(os.path.join(LIBDIR, "libfeti4i_b200_i64.so"))
    lib.FETI4IGetLastError.restype = ctypes.c_char_p
    m = ctypes.c_void_p()
    lib.FETI4ICreateStiffnessMatrix(ctypes.byref(m), ctypes.c_long(0), ctypes.c_long(0))
    nodes = (ctypes.c_long * 1)(1 << 40)
    dofs = (ctypes.c_long * 1)(0)
    vals = (ctypes.c_double * 1)(1.0)
    lib.FETI4IAddElement(m, ctypes.c_long(0), ctypes.c_long(1), nodes, ctypes.c_long(1), dofs, vals)
    assert b"32-bit" in lib.FETI4IGetLastError()
    lib.FETI4IDestroy(m)


@pytest.mark.gpu
@pytest.mark.parametrize("width", [32, 64])
def test_c_caller_solve(setup, width):
    P, path, tmp, exe = setup
    out = os.path.join(tmp, f"solve{width}.bin")
    r = subprocess.run([exe[width], path, out, "solve"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    inst = problems.make_instance(P, iopts={F.PRECONDITIONER: F.PREC_LUMPED, F.VERBOSE_LEVEL: 0},
                                  ropts={F.PRECISION: 1e-10})
    ref = inst.solve()
    inst.destroy()
    got = np.fromfile(out, dtype=np.float64)
    # two solves of the same instance data agree to the solver precision (the F apply sums with
    # atomics, so the last bits differ from run to run)
    assert np.linalg.norm(got - ref) <= 1e-10 * np.linalg.norm(ref)
