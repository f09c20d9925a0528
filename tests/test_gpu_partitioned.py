"""The partitioned dual problem on the GPU: FETI4I instances that prepare a block of the subdomains
(FETI4I_EXT_OWNED_FIRST / OWNED_COUNT) and their device operators.  One process holds two blocks and
sums their parts in place of the allreduce the processes run over NCCL (one GPU per run here): every
block operator summed over the blocks equals the whole instance's (F to 1e-12, b and e exactly as
sums, the preconditioner against the oracle's to 1e-12, the primal parts to 1e-10), and the driver's
PCG over the two blocks solves to 1e-8 against a direct solve in the whole instance's iteration count."""
import numpy as np
import pytest
import torch

from espreso_b200 import feti4i as F
from espreso_b200 import problems
from espreso_b200.partitioned import LibraryBlock, PartitionedSolver, owned_range

from helpers import direct_u, oracle_problem

pytestmark = pytest.mark.gpu


class SumBlock:
    """Several blocks of one process: their parts summed where processes would allreduce."""

    def __init__(self, blocks):
        self.blocks = blocks
        self.n_lambda = blocks[0].n_lambda
        self.device = blocks[0].device

    def coarse_blocks(self):
        return [c for b in self.blocks for c in b.coarse_blocks()]

    def dual_rhs(self):
        b = sum(blk.dual_rhs()[0] for blk in self.blocks)
        e = {}
        for blk in self.blocks:
            e.update(blk.dual_rhs()[1])
        return b, e

    def apply_F(self, x, y):
        for b in self.blocks:
            b.apply_F(x, y)

    def precondition(self, x, y):
        for b in self.blocks:
            b.precondition(x, y)

    def primal(self, lam, alpha):
        return sum(b.primal(lam, alpha) for b in self.blocks)


OPTS = dict(ropts={F.PRECISION: 1e-10})


@pytest.mark.parametrize("prec", [F.PREC_LUMPED, F.PREC_DIRICHLET, F.PREC_SUPER_DIRICHLET])
def test_two_blocks_equal_whole_instance(prec):
    schur = F.FP64
    P = problems.elasticity_cube(domains=(3, 2, 2), elements=(4, 3, 3))
    iopts = {F.PRECONDITIONER: prec, F.VERBOSE_LEVEL: 0, F.MAX_ITERATIONS: 1000}
    ext = {F.EXT_SCHUR_PRECISION: schur}
    whole = problems.make_instance(P, iopts=iopts, ext=ext, **OPTS)
    nd = int(whole.stats()["subdomains"])
    blocks = [LibraryBlock(P, *owned_range(nd, r, 2), iopts=iopts, ext=ext, precision=schur, **OPTS)
              for r in range(2)]
    assert [b.inst.stats()["subdomains"] for b in blocks] == [nd // 2, nd - nd // 2]
    dev = torch.device("cuda")
    n_lambda = blocks[0].n_lambda
    rng = np.random.default_rng(3)
    x = rng.standard_normal(n_lambda)
    xt = torch.from_numpy(x).to(dev)
    y = torch.zeros_like(xt)
    for b in blocks:
        b.apply_F(xt, y)
    ref = whole.apply_F(x, schur)
    assert np.linalg.norm(y.cpu().numpy() - ref) <= 1e-12 * np.linalg.norm(ref)
    # preconditioner: the oracle's (K, S_dir and S_sd do not depend on the regularisation)
    OP = oracle_problem(P, dirichlet_prec=True)
    z = torch.zeros_like(xt)
    for b in blocks:
        b.precondition(xt, z)
    zref = OP.precondition(x, prec)
    assert np.linalg.norm(z.cpu().numpy() - zref) <= 1e-12 * np.linalg.norm(zref)
    # right-hand sides
    bw, ew = whole.dual_rhs()
    bs = sum(b.dual_rhs()[0] for b in blocks)
    np.testing.assert_allclose(bs, bw, rtol=1e-12, atol=1e-12 * np.abs(bw).max())
    # the driver over the two blocks
    S = PartitionedSolver(SumBlock(blocks))
    lam, alpha = S.solve(precision=1e-10, max_it=1000, prec=prec)
    u = S.primal()
    uw = whole.solve()
    assert S.converged and abs(S.iterations - whole.stats()["iterations"]) <= 1
    ud = direct_u(P).ravel()
    assert np.linalg.norm(u - ud) <= 1e-8 * np.linalg.norm(ud)
    assert np.linalg.norm(u - uw) <= 1e-8 * np.linalg.norm(uw)
    # the partitioned instance refuses the internal whole-problem solve
    with pytest.raises(F.FETI4IError, match="OWNED_COUNT"):
        blocks[0].inst.solve()
    for b in blocks:
        b.destroy()
    whole.destroy()


def test_one_block_driver_matches_fetisolve():
    P = problems.heat_cube(domains=(3, 3, 2), elements=(4, 4, 4), seed=4)
    iopts = {F.PRECONDITIONER: F.PREC_LUMPED, F.VERBOSE_LEVEL: 0}
    whole = problems.make_instance(P, iopts=iopts, **OPTS)
    nd = int(whole.stats()["subdomains"])
    blk = LibraryBlock(P, 0, nd, iopts=iopts, **OPTS)
    S = PartitionedSolver(blk)
    S.solve(precision=1e-10, prec=F.PREC_LUMPED)
    u = S.primal()
    uw = whole.solve()
    assert np.linalg.norm(u - uw) <= 1e-9 * np.linalg.norm(uw)
    assert S.iterations == whole.stats()["iterations"]
    blk.destroy()
    whole.destroy()
