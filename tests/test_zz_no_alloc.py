"""FETI4ITiledSymvNoAlloc: the allocation-free batched SYMV entry point.

Some callers manage every byte of device memory themselves -- a finite-element
code that reserves its HBM pool at start-up and may not allocate while it runs.
This entry point serves them: the caller passes its own device buffers (tiles,
descriptors, x, y) and the library allocates nothing; its scratch is a static
device array of bounded size.  The test feeds it the Schur complements of a
FETI4I instance (buffers allocated here, by the caller) and checks, on two
calls in a row, that it returns what the existing F-apply entry point
(FETI4IApplyDualOperator) returns, at the FP64 tolerance of the other parity
tests (1e-13 relative).  This file is collected last on purpose.
"""
import numpy as np
import pytest

from espreso_b200 import feti4i as F
from espreso_b200 import problems

pytestmark = pytest.mark.gpu


def test_tiled_symv_no_alloc_matches_dual_operator():
    import torch

    P = problems.elasticity_cube(domains=(3, 2, 2), elements=(3, 4, 3))
    inst = problems.make_instance(P, iopts={F.PRECONDITIONER: F.PREC_LUMPED, F.VERBOSE_LEVEL: 0})
    nd = int(inst.stats()["subdomains"])
    mats = [inst.schur(d) for d in range(nd)]
    lams = [inst.multipliers(d)["lam"] for d in range(nd)]
    tiles, toff, order = F.pack_symmetric_tiles(mats)
    voff = np.concatenate([[0], np.cumsum(order)[:-1]]).astype(np.int32)
    NL = int(order.sum())
    dev = torch.device("cuda:0")
    t_tiles = torch.from_numpy(tiles).to(dev)
    t_toff = torch.from_numpy(toff).to(dev)
    t_order = torch.from_numpy(order).to(dev)
    t_voff = torch.from_numpy(voff).to(dev)
    t_y = torch.zeros(NL, dtype=torch.float64, device=dev)
    t_dot = torch.zeros(1, dtype=torch.float64, device=dev)
    rng = np.random.default_rng(7)
    n_lambda = int(inst.stats()["dual_size"])
    for call in range(2):
        x = rng.standard_normal(n_lambda)
        xL = np.concatenate([x[l] for l in lams])
        t_x = torch.from_numpy(xL).to(dev)
        torch.cuda.synchronize()
        F.tiled_symv_noalloc(t_tiles.data_ptr(), t_toff.data_ptr(), t_order.data_ptr(), t_voff.data_ptr(), nd,
                             int(order.max()), t_x.data_ptr(), t_y.data_ptr(), t_dot.data_ptr(), 0)
        torch.cuda.synchronize()
        yL = t_y.cpu().numpy()
        y = np.zeros(n_lambda)
        for d in range(nd):
            np.add.at(y, lams[d], yL[voff[d]:voff[d] + order[d]])
        ref = inst.apply_F(x, F.FP64)
        assert np.linalg.norm(y - ref) <= 1e-13 * np.linalg.norm(ref), call
        assert abs(t_dot.item() - float(xL @ yL)) <= 1e-12 * abs(float(xL @ yL))
    # a caller that understates max_order gets no product for the larger matrices: NaN in their y
    # range and in the dot, the others as before
    lo = int(order.min()) if order.max() > order.min() else int(order.min()) - 1
    F.tiled_symv_noalloc(t_tiles.data_ptr(), t_toff.data_ptr(), t_order.data_ptr(), t_voff.data_ptr(), nd, lo,
                         t_x.data_ptr(), t_y.data_ptr(), t_dot.data_ptr(), 0)
    torch.cuda.synchronize()
    yS = t_y.cpu().numpy()
    assert np.isnan(t_dot.item())
    for d in range(nd):
        seg = slice(voff[d], voff[d] + order[d])
        if order[d] > lo:
            assert np.all(np.isnan(yS[seg])), d
        else:
            assert np.allclose(yS[seg], yL[seg], rtol=1e-13, atol=1e-13 * np.abs(yL).max()), d
    with pytest.raises(F.FETI4IError, match="nmatrices"):
        F.tiled_symv_noalloc(t_tiles.data_ptr(), t_toff.data_ptr(), t_order.data_ptr(), t_voff.data_ptr(),
                             16385, int(order.max()), t_x.data_ptr(), t_y.data_ptr(), 0, 0)
    with pytest.raises(F.FETI4IError, match="max_order"):
        F.tiled_symv_noalloc(t_tiles.data_ptr(), t_toff.data_ptr(), t_order.data_ptr(), t_voff.data_ptr(),
                             nd, 4000, t_x.data_ptr(), t_y.data_ptr(), 0, 0)
    inst.destroy()
