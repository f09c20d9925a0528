"""The opt-in PCG loop graph (FETI4I_LOOP_GRAPH=1: a CUDA graph with a WHILE node around one
iteration and an IF node for the residual replacement) against the default chunked graphs: the same
solution to 1e-10, the same iteration and replacement counts, and in mixed precision fewer kernel launches.  The switch is
read once per process, so each variant runs in its own interpreter."""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SCRIPT = r"""
import json, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
from espreso_b200 import feti4i as F, problems
P = problems.heat_cube(domains=(4, 3, 3), elements=(5, 5, 5), seed=1)
out = {}
for schur in (F.FP64, F.FP32):
    inst = problems.make_instance(P, iopts={F.PRECONDITIONER: F.PREC_LUMPED, F.VERBOSE_LEVEL: 0},
                                  ropts={F.PRECISION: 1e-10}, ext={F.EXT_SCHUR_PRECISION: schur})
    u = inst.solve()
    st = inst.stats()
    out[str(schur)] = dict(u=u.tolist(), it=st["iterations"], repl=st["replacements"], conv=st["converged"],
                           launches=st["kernel_launches"])
    inst.destroy()
print(json.dumps(out))
"""


def _run(loop):
    env = dict(os.environ, FETI4I_LOOP_GRAPH=loop)
    r = subprocess.run([sys.executable, "-c", SCRIPT, ROOT], capture_output=True, text=True, env=env, timeout=600)
    assert r.returncode == 0, r.stderr
    return json.loads(r.stdout.strip().splitlines()[-1])


def test_loop_graph_matches_chunked_graphs():
    import numpy as np
    a, b = _run("1"), _run("0")
    for key in a:
        ua, ub = np.array(a[key]["u"]), np.array(b[key]["u"])
        assert a[key]["conv"] == b[key]["conv"] == 1.0
        assert a[key]["it"] == b[key]["it"] and a[key]["repl"] == b[key]["repl"]
        assert np.linalg.norm(ua - ub) <= 1e-10 * np.linalg.norm(ub)
    # mixed precision: the replacement kernels run only in the iterations that replace
    assert a[str(1)]["launches"] < b[str(1)]["launches"]
