#!/usr/bin/env python3
"""Regenerates the golden fixtures in this folder from the CPU oracle.

The reference engine (Mojo) cannot be built or run here, so the fixtures are the oracle's
outputs on small seeded inputs; they pin the oracle against regressions (CPU tests compare bit
for bit) and give the GPU tests fixed targets (compared within the documented tolerances).

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))

import numpy as np  # noqa: E402

from oracle import binding  # noqa: E402
from strut_b200 import model as M  # noqa: E402
from strut_b200 import workloads as W  # noqa: E402
from tests.helpers import ALTERNATING, lcg_strains, mixed_section_case, path_array  # noqa: E402

MATERIALS = [
    {"id": 1, "type": "Steel02", "params": dict(W.STEEL)},
    {"id": 2, "type": "Concrete02", "params": dict(W.CORE)},
    {"id": 3, "type": "Concrete02", "params": dict(W.COVER)},
    {"id": 4, "type": "Steel01", "params": {"Fy": 350.0e6, "E0": 200.0e9, "b": 0.01}},
]


def material_fixtures():
    out = []
    for mat in MATERIALS:
        strains = lcg_strains(100 + mat["id"], 200, 0.004, "cyclic")
        res = binding.material_path(M.uniaxial_material(mat), strains)
        out.append({"material": mat, "strains": strains.tolist(), "stress_tangent": res.tolist()})
    return out


def section_fixtures():
    out = []
    case = mixed_section_case(ALTERNATING)
    mats, nm, fibs, nf = M.section_fibers(case["section"], case["materials"])
    res = binding.section_path(mats, nm, fibs, nf, path_array(case))
    out.append({"case": case, "response": res.tolist()})
    sec = W.rc_section(1, 0.5, 0.5)
    mats_json = [{"id": 1, "type": "Concrete02", "params": dict(W.CORE)},
                 {"id": 2, "type": "Concrete02", "params": dict(W.COVER)},
                 {"id": 3, "type": "Steel02", "params": dict(W.STEEL)}]
    k = lcg_strains(7, 80, 0.004, "cyclic")
    e = -0.0004 + 0.2 * lcg_strains(8, 80, 0.001, "walk")
    path = [{"eps0": float(a), "kappa": float(b)} for a, b in zip(e, k)]
    case2 = {"materials": mats_json, "section": sec, "deformation_path": path}
    mats, nm, fibs, nf = M.section_fibers(sec, mats_json)
    res = binding.section_path(mats, nm, fibs, nf, path_array(case2))
    out.append({"case": case2, "response": res.tolist()})
    return out


def transient_fixture():
    case = W.rc_frame_case(stories=2, bays=1, steps=60, seed=42, pga_g=0.45)
    m = M.Model(case)
    disp, ef, iters, rc, failed = binding.run_transient(m, 60)
    assert rc == 0
    return {"case": case, "disp": disp.tolist(), "eforce": ef.tolist(), "iters": iters.tolist()}


def main():
    binding.build()
    binding.set_simd_width(8)
    (HERE / "material_paths.json").write_text(json.dumps(material_fixtures()))
    (HERE / "section_paths.json").write_text(json.dumps(section_fixtures()))
    (HERE / "transient_2x1.json").write_text(json.dumps(transient_fixture()))
    print("wrote fixtures to", HERE)


if __name__ == "__main__":
    main()
