#!/usr/bin/env python3
"""Writes strut_validation_cases.json: Strut's own fiber beam-column validation models
(tests/validation/{force,disp}_beam_column{2,3}d_fiber_cantilever/*.json of the reference
project), each given a transient analysis block so that it runs on the transient path.

The models are the reference's as they stand (nodes, constraints, materials, FiberSection2d /
FiberSection3d patches, element type, geomTransf, integration); the conversion replaces the static
analysis block and its point load by: a lumped mass on the free node's translations, 5 % mass-
proportional damping, a seeded Kanai-Tajimi ground motion along the point load's direction
(PGA 0.5 g, dt 0.01 s, 300 steps) and Newton with NormDispIncr 1e-8 on BandGeneral.  Recorders
that this path records (node displacement, element force, section force and deformation) are
kept.

    python tests/golden/make_strut_validation_cases.py [/path/to/reference]
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))

from strut_b200 import workloads as W  # noqa: E402

NAMES = ["force_beam_column2d_fiber_cantilever", "disp_beam_column2d_fiber_cantilever",
         "force_beam_column3d_fiber_cantilever", "disp_beam_column3d_fiber_cantilever"]
STEPS, DT = 300, 0.01
MASS = {2: 2.0e4, 3: 4.0e4}  # kg on each translation of the free node (ndm 2, 3)


def convert(case: dict, seed: int) -> dict:
    out = {k: v for k, v in case.items() if k not in ("analysis", "loads", "enabled", "benchmark_size",
                                                       "parity_tolerance_by_recorder")}
    ndm = int(case["model"]["ndm"])
    load = case["loads"][0]
    free = [n for n in case["nodes"] if not n.get("constraints")]
    out["masses"] = [{"node": n["id"], "dof": d, "value": MASS[ndm]} for n in free for d in range(1, ndm + 1)]
    rec = W.kanai_tajimi_record(seed, STEPS + 1, DT, wg=15.0, zg=0.6, pga_g=0.5)
    out["time_series"] = [{"type": "Path", "tag": 1, "dt": DT, "values": [float(v) for v in rec]}]
    out["pattern"] = {"type": "UniformExcitation", "tag": 1, "direction": int(load["dof"]), "accel": 1}
    out["rayleigh"] = {"alphaM": 0.5}
    out["analysis"] = {"type": "transient_nonlinear", "steps": STEPS, "dt": DT,
                       "integrator": {"type": "Newmark", "gamma": 0.5, "beta": 0.25},
                       "algorithm": "Newton", "test_type": "NormDispIncr", "tol": 1.0e-8, "max_iters": 20,
                       "system": "BandGeneral"}
    out["recorders"] = [r for r in case.get("recorders", [])
                        if r["type"] in ("node_displacement", "element_force", "section_force", "section_deformation")]
    return out


def main():
    ref = Path(sys.argv[1]) if len(sys.argv) > 1 else Path("/root/reference")
    cases = {}
    for k, name in enumerate(NAMES):
        case = json.loads((ref / "tests" / "validation" / name / f"{name}.json").read_text())
        cases[name] = convert(case, 9100 + k)
    (HERE / "strut_validation_cases.json").write_text(json.dumps(cases) + "\n")


if __name__ == "__main__":
    main()
