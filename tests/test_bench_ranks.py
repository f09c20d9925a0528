"""The N > 1 path of bench.py on CPU: two gloo ranks, one load case each, no exchange in the solve.

Each rank builds its own load case (rank 0 the workload's right-hand side, rank r a seeded
perturbation); the ranks meet only in the max-over-ranks timing reduction.  The check runs the
FETI4I host preprocessing on every rank (HOST_ONLY) and compares the dual right-hand sides: equal
where the load case is equal, different where it differs.
"""
import os
import socket

import numpy as np
import pytest


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
        import bench
        from espreso_b200 import feti4i as F
        from espreso_b200 import problems

        P = problems.heat_cube(domains=(2, 2, 1), elements=(3, 3, 3), seed=5)
        rhs = bench.rank_load_case(P.rhs(), rank)
        again = bench.rank_load_case(P.rhs(), rank)
        inst = problems.make_instance(P, iopts={F.VERBOSE_LEVEL: 0}, ext={F.EXT_HOST_ONLY: 1})
        inst.update_rhs(rhs)
        b, _ = inst.dual_rhs()
        inst.destroy()
        mx = bench.dist_max(dist, float(rank + 1))
        q.put((rank, np.array_equal(rhs, again), float(np.abs(rhs - P.rhs()).max()), b, mx))
    finally:
        dist.destroy_process_group()


def test_two_ranks_one_load_case_each():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = {}
    for _ in procs:
        r = q.get(timeout=300)
        out[r[0]] = r
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (_, det0, dev0, b0, mx0), (_, det1, dev1, b1, mx1) = out[0], out[1]
    assert det0 and det1                      # deterministic per rank
    assert dev0 == 0.0 and dev1 > 0.0         # rank 0: the workload's own load case
    assert mx0 == mx1 == 2.0                  # max over ranks
    assert b0.shape == b1.shape
    assert np.linalg.norm(b1 - b0) > 1e-3 * np.linalg.norm(b0)
