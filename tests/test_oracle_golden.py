"""The CPU oracle against the reference's own regression presets (.emr files).

The presets are ESPRESO's only reference-produced known answers for a FETI
solve (benchmarks/estest.py:71-101 compares them at |d|>1e-4 and
|d/v|>1e-3).  They are stored in tests/golden/emr_presets.json by
tests/golden/make_emr_fixtures.py.
"""
import json
import os

import numpy as np
import pytest

from oracle import feti, htfeti, mesh, numbering

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "emr_presets.json")))


def _close(value, ref, tol):
    d = abs(value - ref)
    return not (d > tol["abs"] and (ref == 0 or d / abs(ref) > tol["rel"]))


def _solve(g, Ke, fe, dpn, dirich, prec, hybrid=False):
    num = numbering.Numbering(g.elem_nodes, g.elem_domain, g.coords.shape[0], dpn, dirich)
    if hybrid:
        # one cluster per process of the preset: the grid's clusters
        ndom_c = int(np.prod(g.domains))
        P = htfeti.HTFETIProblem(num, g.elem_nodes, g.elem_domain, Ke, fe, g.coords,
                                 np.arange(g.ndomains) // ndom_c, build_dirichlet=(prec == feti.PREC_DIRICHLET))
    else:
        P = feti.FETIProblem(num, g.elem_nodes, g.elem_domain, Ke, fe, g.coords,
                             build_dirichlet=(prec == feti.PREC_DIRICHLET))
    P.solve(precision=1e-9, prec=prec)
    return P, P.merge(P.primal(), g.coords.shape[0])


@pytest.mark.parametrize("prec", [feti.PREC_LUMPED, feti.PREC_DIRICHLET])
def test_gravity_hexa8(prec):
    case = GOLD["gravity_hexa8"]
    g = mesh.Grid(case["clusters"], case["domains"], case["elements"], length=(100, 100, 100))
    Ke, fe = mesh.elasticity(g.coords[g.elem_nodes], 2.1e9, 0.3, body=(0, 0, 7850 * 9.8066))
    z0 = g.nodes_where(2, 0.0)
    P, u = _solve(g, Ke, fe, 3, {c: (z0, 0.0) for c in range(3)}, prec)
    mag = np.linalg.norm(u, axis=1)
    stats = {"MIN": mag.min(), "MAX": mag.max(), "AVG": mag.mean()}
    for m in case["monitors"]:
        assert _close(stats[m["stat"]], m["value"], case["tolerance"]), (m, stats)


@pytest.mark.parametrize("method", ["total", "hybrid"])
def test_pressure_hexa8_patch(method):
    case = GOLD["pressure_hexa8_" + method]
    E = 2.1e11
    g = mesh.Grid(case["clusters"], case["domains"], case["elements"], length=(100, 100, 100))
    Ke, fe = mesh.elasticity(g.coords[g.elem_nodes], E, 0.3)
    dirich = {0: (g.nodes_where(0, 0.0), 0.0), 1: (g.nodes_where(1, 0.0), 0.0), 2: (g.nodes_where(2, 0.0), 0.0)}
    # normal pressures on X1, Y1, Z1 (pressure/espreso.ecf NORMAL_PRESSURE)
    n_nodes = g.coords.shape[0]
    fnode = np.zeros((n_nodes, 3))
    faces = mesh.boundary_faces(g.elem_nodes)
    for axis, p in ((2, 70 * E / 5200), (1, 3 * 70 * E / 5200 / 7), (0, 3 * 70 * E / 5200 / 7)):
        on = np.all(np.abs(g.coords[faces][:, :, axis] - 100.0) < 1e-9, axis=1)
        F = mesh.face_pressure(g.coords[faces[on]], p)
        np.add.at(fnode, faces[on].ravel(), F.reshape(-1, 3))
    # distribute the nodal loads onto one element per node (any split gives the same global f)
    fe = np.zeros((g.elem_nodes.shape[0], 24))
    first = {}
    for e, nodes in enumerate(g.elem_nodes):
        for a, n in enumerate(nodes):
            if n not in first:
                first[n] = (e, a)
    for n, (e, a) in first.items():
        fe[e, 3 * a:3 * a + 3] = fnode[n]
    P, u = _solve(g, Ke, fe, 3, dirich, feti.PREC_LUMPED, hybrid=(method == "hybrid"))
    z1 = g.nodes_where(2, 100.0)
    mag = np.linalg.norm(u[z1], axis=1)
    stats = {"MIN": mag.min(), "MAX": mag.max()}
    for m in case["monitors"]:
        assert _close(stats[m["stat"]], m["value"], case["tolerance"]), (m, stats)


@pytest.mark.parametrize("method", ["total", "hybrid"])
def test_heat_hexa8(method):
    """Isotropic conductivity stands in for the preset's cylindrical orthotropic
    tensor: the stored monitors (Dirichlet extrema and the mean 200 fixed by the
    x -> 1-x antisymmetry) do not depend on it."""
    case = GOLD["heat_hexa8_" + method]
    g = mesh.Grid(case["clusters"], case["domains"], case["elements"], length=(1, 1, 1))
    Ke, fe = mesh.heat(g.coords[g.elem_nodes], 1.0)
    top, bottom = g.nodes_where(0, 0.0), g.nodes_where(0, 1.0)
    dirich = {0: (np.concatenate([top, bottom]), np.concatenate([np.full(top.size, 100.0), np.full(bottom.size, 300.0)]))}
    P, u = _solve(g, Ke, fe, 1, dirich, feti.PREC_DIRICHLET, hybrid=(method == "hybrid"))
    T = u[:, 0]
    stats = {("TOP", "MAX"): T[top].max(), ("BOTTOM", "MIN"): T[bottom].min(), ("ALL_ELEMENTS", "AVG"): T.mean()}
    for m in case["monitors"]:
        assert _close(stats[(m["region"], m["stat"])], m["value"], case["tolerance"]), (m, stats)


def test_oracle_matches_direct_solve():
    """FETI displacements equal a global direct solve of the same assembled system."""
    g = mesh.Grid((1, 1, 1), (2, 2, 2), (3, 3, 3), length=(1, 1, 1))
    Ke, fe = mesh.elasticity(g.coords[g.elem_nodes], 2.1e11, 0.3, body=(0, 0, -7850 * 9.81))
    x0 = g.nodes_where(0, 0.0)
    P, u = _solve(g, Ke, fe, 3, {c: (x0, 0.0) for c in range(3)}, feti.PREC_LUMPED)
    K, f = feti.global_system(g.elem_nodes, Ke, fe, g.coords.shape[0], 3)
    fd = np.concatenate([3 * x0 + c for c in range(3)])
    ud = feti.direct_solve(K, f, fd, 0.0).reshape(-1, 3)
    assert np.linalg.norm(u - ud) / np.linalg.norm(ud) < 1e-8


@pytest.mark.parametrize("physics", ["elasticity", "heat"])
def test_htfeti_oracle_matches_direct_solve(physics):
    """HTFETI with corner-glued clusters gives the displacements of a global direct solve."""
    g = mesh.Grid((2, 1, 2), (2, 2, 1), (2, 3, 2), length=(1, 1, 1))
    if physics == "elasticity":
        dpn = 3
        Ke, fe = mesh.elasticity(g.coords[g.elem_nodes], 2.1e11, 0.3, body=(0, 0, -7850 * 9.81))
        x0 = g.nodes_where(0, 0.0)
        dirich = {c: (x0, 0.0) for c in range(3)}
        fd = np.concatenate([3 * x0 + c for c in range(3)])
    else:
        dpn = 1
        Ke, fe = mesh.heat(g.coords[g.elem_nodes], 1.0)
        x0 = g.nodes_where(2, 0.0)
        dirich = {0: (x0, 0.0)}
        fe = fe + 1.0 / 8 * np.ones_like(fe)
        fd = x0
    P, u = _solve(g, Ke, fe, dpn, dirich, feti.PREC_LUMPED, hybrid=True)
    K, f = feti.global_system(g.elem_nodes, Ke, fe, g.coords.shape[0], dpn)
    ud = feti.direct_solve(K, f, fd, 0.0).reshape(-1, dpn)
    assert P.n_kern == (6 if dpn == 3 else 1) * 4        # one kernel block per cluster
    assert np.linalg.norm(u - ud) / np.linalg.norm(ud) < 1e-8


def test_corner_rule_surface_cursor():
    """Corner nodes follow fetidata.cpp:146-188: surface intervals shared by two or more
    domains take every len/3-th node until the first single-domain surface interval; from
    there on every interval takes its middle node."""
    g = mesh.Grid((1, 1, 1), (2, 2, 1), (3, 3, 2), length=(1, 1, 1))
    num = numbering.Numbering(g.elem_nodes, g.elem_domain, g.coords.shape[0], 1, {0: (g.nodes_where(2, 0.0), 0.0)})
    corners = htfeti.corner_nodes(num)
    ext = [i for i, e in enumerate(num.interval_ext) if e]
    multi = [i for i, (d, _) in enumerate(num.intervals) if len(d) > 1]
    holders = {num.node_doms[n] for n, _ in corners}
    assert holders == {num.intervals[i][0] for i in multi}
    first_single = next((i for i in ext if len(num.intervals[i][0]) == 1), None)
    for i in multi:
        nodes = set(num.intervals[i][1].tolist())
        k = sum(1 for n, _ in corners if n in nodes)
        if i in ext and (first_single is None or i < first_single) and len(nodes) >= 2:
            assert k >= 2
        else:
            assert k == 1
