"""The partitioned dual PCG (espreso_b200.partitioned) on CPU: world_size-2 gloo processes, each with a
block of the oracle's subdomains, against the one-process solve of the same driver and the oracle's
own PCG (lambda to 1e-10, same iteration count) and a direct solve (u to 1e-8).  The collectives are
the ones the GPU processes run over NCCL: one allreduce of the dual vector per F apply and per
preconditioner apply, the G blocks and e gathered once."""
import os
import socket

import numpy as np
import pytest

from oracle import feti as OF

PRECS = [OF.PREC_LUMPED, OF.PREC_DIRICHLET, OF.PREC_NONE]


def _problem():
    from espreso_b200 import problems
    return problems.elasticity_cube(domains=(3, 2, 2), elements=(3, 3, 2))


def _oracle(P):
    from oracle import numbering as ON
    num = ON.Numbering(P.elem_nodes, P.elem_domain, P.n_nodes, P.dpn, P.dirichlet)
    return OF.FETIProblem(num, P.elem_nodes, P.elem_domain, P.Ke, P.fe, P.coords, build_dirichlet=True)


def _run(P, OP, rank, world, group, prec):
    from espreso_b200.partitioned import PartitionedSolver, owned_range
    from tests.oracle_block import OracleBlock
    first, count = owned_range(len(OP.sub), rank, world)
    blk = OracleBlock(OP, first, count, P)
    blk.prec = prec
    S = PartitionedSolver(blk, group=group)
    lam, alpha = S.solve(precision=1e-11, max_it=500, prec=prec)
    u = S.primal()
    return lam.numpy(), alpha.numpy(), S.iterations, u, S.collectives


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        P = _problem()
        OP = _oracle(P)
        out = {prec: _run(P, OP, rank, world, dist.group.WORLD, prec) for prec in PRECS}
        q.put((rank, out))
    finally:
        dist.destroy_process_group()


@pytest.fixture(scope="module")
def two_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = {}
    for _ in procs:
        r, out = q.get(timeout=300)
        res[r] = out
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    return res


@pytest.mark.parametrize("prec", PRECS)
def test_partitioned_matches_one_process(two_ranks, prec):
    from tests.helpers import direct_u
    P = _problem()
    OP = _oracle(P)
    lam1, alpha1, it1, u1, coll1 = _run(P, OP, 0, 1, None, prec)
    assert coll1 == 0
    # the driver's one-process PCG is the oracle's Solve_RegCG
    lam_o = OP.solve(precision=1e-11, max_it=500, prec=prec)
    assert abs(OP.iterations - it1) <= 1
    assert np.linalg.norm(lam1 - lam_o) <= 1e-9 * np.linalg.norm(lam_o)
    ud = direct_u(P).ravel()
    for rank in (0, 1):
        lam, alpha, it, u, coll = two_ranks[rank][prec]
        # the allreduce adds the blocks' parts in another order than one process does, so the
        # last bits differ and the stop test may pass one iteration apart
        assert abs(it - it1) <= 1
        assert np.linalg.norm(lam - lam1) <= 1e-10 * np.linalg.norm(lam1)
        assert np.linalg.norm(u - ud) <= 1e-8 * np.linalg.norm(ud)
        # one allreduce of the dual vector per F apply (and per preconditioner apply), b and u once
        per_it = 1 if prec == OF.PREC_NONE else 2
        assert coll == 1 + 1 + per_it * it + 1
    assert two_ranks[0][prec][2] == two_ranks[1][prec][2]   # the processes take the same iterations
    # both processes hold the same replicated iterates
    assert np.array_equal(two_ranks[0][prec][0], two_ranks[1][prec][0])
