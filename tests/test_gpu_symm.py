"""The multi right-hand-side F apply (tile SYMM) against the single-vector FP64 F apply.

FETI4IApplyDualOperatorMulti runs the F apply of FETI4ISolveMulti on up to 32 dual vectors at once:
  * FP64 tiles: tile_symm_mma_kernel (FP64 tensor-core MMA), to 1e-12;
  * FP32 tiles on the tensor cores (3xTF32): the warp-specialised tile_symm_tc3_kernel at 32
    vectors, tile_symm_tc_kernel at 8 and 16 (and at 32 with FETI4I_SYMM_TC3=0, run in a child
    process), and the asynchronous tile_symm_tc2_kernel at 32 vectors (FETI4I_SYMM_TC2=1, child
    process), with every kind of 32-column block (stored tiles, their transposes, the blocks that
    mix both);
  * FP32 tiles on the CUDA cores (FETI4I_EXT_SYMM_TENSOR = 0).
FP32 Schur storage rounds S_i to 2^-24 relative and accumulates in FP32, so the FP32 paths agree
with the FP64 apply to 2e-5 (norm-wise per vector).  A single subdomain makes every dual row one
row of S_i, so the check also covers each 32 x 32 block of S_i separately.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

from espreso_b200 import feti4i as F
from espreso_b200 import problems

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def problems_():
    return {
        # one subdomain, Dirichlet face of 17 x 17 nodes: S of order 289 (10 tile rows)
        "single": problems.heat_cube(domains=(1, 1, 1), elements=(16, 16, 4), seed=1),
        "heat_big": problems.heat_cube(domains=(2, 2, 2), elements=(10, 10, 10), seed=3),
    }


def relerr(Y, R):
    return max(np.linalg.norm(Y[j] - R[j]) / np.linalg.norm(R[j]) for j in range(R.shape[0]))


@pytest.mark.parametrize("name", ["single", "heat_big"])
@pytest.mark.parametrize("tensor", [1, 0])
def test_symm_matches_single_apply(problems_, name, tensor):
    P = problems_[name]
    inst = problems.make_instance(P, iopts={F.VERBOSE_LEVEL: 0},
                                  ext={F.EXT_SCHUR_PRECISION: F.FP32, F.EXT_SYMM_TENSOR: tensor})
    nl = int(inst.stats()["dual_size"])
    rng = np.random.default_rng(11)
    for nrhs in (32, 16, 5):
        X = rng.standard_normal((nrhs, nl))
        R = np.array([inst.apply_F(x, F.FP64) for x in X])
        assert relerr(inst.apply_F_multi(X, F.FP64), R) <= 1e-12
        assert relerr(inst.apply_F_multi(X, F.FP32), R) <= 2e-5
    if name == "single":
        # block by block: x nonzero on one 32-row block of S, every 32-row block of y checked
        lam = inst.multipliers(0)["lam"]
        S = inst.schur(0)
        n = S.shape[0]
        for J in range(0, (n + 31) // 32, 3):
            Xl = np.zeros((32, n))
            rows = np.arange(32 * J, min(n, 32 * J + 32))
            Xl[:, rows] = rng.standard_normal((32, rows.size))
            X = np.zeros((32, nl))
            X[:, lam] = Xl
            Y = inst.apply_F_multi(X, F.FP32)[:, lam]
            Ref = Xl @ S.T
            for I in range(0, n, 32):
                blk = slice(I, min(n, I + 32))
                assert np.linalg.norm(Y[:, blk] - Ref[:, blk]) <= 2e-5 * np.linalg.norm(Ref[:, blk]) + 1e-300
    inst.destroy()


def test_symm_async_variant():
    """The same checks with the asynchronous tensor-core SYMM selected (read once per process)."""
    env = dict(os.environ, FETI4I_SYMM_TC2="1")
    r = subprocess.run([sys.executable, "-m", "pytest", "-q", "-m", "gpu", "-p", "no:cacheprovider",
                        __file__ + "::test_symm_matches_single_apply"],
                       env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]


def test_symm_register_staged_variant():
    """The same checks with tile_symm_tc_kernel serving 32 vectors (FETI4I_SYMM_TC3=0)."""
    env = dict(os.environ, FETI4I_SYMM_TC3="0")
    r = subprocess.run([sys.executable, "-m", "pytest", "-q", "-m", "gpu", "-p", "no:cacheprovider",
                        __file__ + "::test_symm_matches_single_apply"],
                       env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
