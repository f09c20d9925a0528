"""Extract the reference's HEXA8 regression presets into emr_presets.json.

Reads the ``.emr`` monitor tables and the benchmark arguments from the
reference checkout (``benchmarks/**``) and stores the numbers, the case
geometry and the monitor definitions as a small JSON fixture, so that the
tests never need the reference tree at run time.

    python tests/golden/make_emr_fixtures.py <path of the reference checkout>
"""
import json
import os
import sys

CASES = {
    # name: (relative emr path, args from tested.py, physics, monitors)
    "gravity_hexa8": ("benchmarks/linearElasticity3D/steadystate/gravity/HEXA8.emr",
                      [2, 2, 1, 1, 2, 2, 5, 5, 5], "elasticity",
                      [("ALL_NODES", "MIN", "DISPLACEMENT"), ("ALL_NODES", "MAX", "DISPLACEMENT"),
                       ("ALL_NODES", "AVG", "DISPLACEMENT")]),
    "pressure_hexa8_total": ("benchmarks/linearElasticity3D/steadystate/pressure/HEXA8.TOTAL_FETI.emr",
                             [2, 2, 1, 1, 2, 2, 5, 5, 5], "elasticity",
                             [("Z1", "MIN", "DISPLACEMENT"), ("Z1", "MAX", "DISPLACEMENT")]),
    "heat_hexa8_total": ("benchmarks/diffusion3D/steadystate/simple/HEXA8.TOTAL_FETI.emr",
                         [3, 2, 1, 1, 2, 3, 4, 3, 4], "heat",
                         [("TOP", "MAX", "TEMPERATURE"), ("BOTTOM", "MIN", "TEMPERATURE"),
                          ("ALL_ELEMENTS", "AVG", "TEMPERATURE")]),
    # HYBRID_FETI runs of the same cases: one cluster per process, clusters = args[0:3]
    "pressure_hexa8_hybrid": ("benchmarks/linearElasticity3D/steadystate/pressure/HEXA8.HYBRID_FETI.emr",
                              [2, 2, 1, 1, 2, 2, 5, 5, 5], "elasticity",
                              [("Z1", "MIN", "DISPLACEMENT"), ("Z1", "MAX", "DISPLACEMENT")]),
    "heat_hexa8_hybrid": ("benchmarks/diffusion3D/steadystate/simple/HEXA8.HYBRID_FETI.emr",
                          [3, 2, 1, 1, 2, 3, 4, 3, 4], "heat",
                          [("TOP", "MAX", "TEMPERATURE"), ("BOTTOM", "MIN", "TEMPERATURE"),
                           ("ALL_ELEMENTS", "AVG", "TEMPERATURE")]),
}


def parse_emr(path):
    with open(path) as fh:
        lines = [ln for ln in fh.read().splitlines() if ln.strip()]
    last = lines[-1]
    vals = []
    for tok in last.split(";")[3:]:
        tok = tok.strip()
        if tok and tok != "-":
            vals.append(float(tok))
    return vals


def main(ref):
    out = {}
    for name, (rel, args, physics, mons) in CASES.items():
        vals = parse_emr(os.path.join(ref, rel))
        out[name] = {
            "source": rel,
            "clusters": args[0:3], "domains": args[3:6], "elements": args[6:9],
            "physics": physics,
            "monitors": [{"region": r, "stat": s, "property": p, "value": v}
                         for (r, s, p), v in zip(mons, vals)],
            "tolerance": {"abs": 1e-4, "rel": 1e-3},
        }
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "emr_presets.json")
    with open(dst, "w") as fh:
        json.dump(out, fh, indent=1)
    print("wrote", dst)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_emr_fixtures.py <path of the reference checkout>")
    main(sys.argv[1])
