"""Shared helpers for the test-suite (cases and comparisons)."""
from __future__ import annotations

import numpy as np


def lcg_strains(seed: int, n: int, scale: float, kind: str = "walk") -> np.ndarray:
    """Deterministic strain scenarios in the spirit of Strut's material micro-benchmark
    (src/mojo/material_compare_micro.mojo:288-368): a 64-bit LCG drives a random walk or a
    cyclic ramp with growing amplitude."""
    mask = (1 << 64) - 1
    state = (seed * 2862933555777941757 + 3037000493) & mask
    out = np.zeros(n)
    x = 0.0
    for i in range(n):
        state = (state * 6364136223846793005 + 1442695040888963407) & mask
        r = (state >> 11) / float(1 << 53)
        if kind == "walk":
            x += (r - 0.5) * scale
        else:
            amp = scale * (1.0 + i / n * 4.0)
            x = amp * np.sin(2.0 * np.pi * i / 37.0) + (r - 0.5) * scale * 0.1
        out[i] = x
    return out


def mixed_section_case(order):
    """Restated from tests/unit/test_fiber_section.py:263-361 of the reference."""
    layers = []
    for material, y, area in order:
        layers.append({"type": "straight", "material": material, "num_bars": 1, "bar_area": area,
                       "y_start": y, "z_start": 0.0, "y_end": y, "z_end": 0.0})
    return {
        "materials": [
            {"id": 1, "type": "Concrete02", "params": {"fpc": -32.0, "epsc0": -0.0021, "fpcu": -18.0,
                                                        "epscu": -0.0058, "rat": 0.12, "ft": 2.8, "Ets": 180.0}},
            {"id": 2, "type": "Concrete02", "params": {"fpc": -36.0, "epsc0": -0.0024, "fpcu": -21.0,
                                                        "epscu": -0.0064, "rat": 0.1, "ft": 3.1, "Ets": 220.0}},
            {"id": 3, "type": "Steel02", "params": {"Fy": 420.0, "E0": 200000.0, "b": 0.012, "R0": 18.0,
                                                     "cR1": 0.925, "cR2": 0.15, "a1": 0.01, "a2": 1.0,
                                                     "a3": 0.01, "a4": 1.0}},
            {"id": 4, "type": "Steel02", "params": {"Fy": 460.0, "E0": 200000.0, "b": 0.01, "R0": 20.0,
                                                     "cR1": 0.92, "cR2": 0.18, "a1": 0.015, "a2": 1.0,
                                                     "a3": 0.015, "a4": 1.0}},
        ],
        "section": {"id": 9, "type": "FiberSection2d", "params": {"patches": [], "layers": layers}},
        "deformation_path": [
            {"eps0": -8.0e-4, "kappa": 6.0e-3},
            {"eps0": -1.6e-3, "kappa": 1.0e-2},
            {"eps0": -2.0e-4, "kappa": -4.0e-3},
            {"eps0": 4.0e-4, "kappa": -8.0e-3},
            {"eps0": -6.0e-4, "kappa": 5.0e-3},
        ],
    }


ALTERNATING = [(1, -0.30, 0.0042), (3, -0.24, 0.00045), (2, -0.10, 0.0040), (4, -0.04, 0.00055),
               (3, 0.04, 0.00045), (1, 0.10, 0.0042), (4, 0.24, 0.00055), (2, 0.30, 0.0040)]
GROUPED = [(1, -0.30, 0.0042), (1, 0.10, 0.0042), (2, -0.10, 0.0040), (2, 0.30, 0.0040),
           (3, -0.24, 0.00045), (3, 0.04, 0.00045), (4, -0.04, 0.00055), (4, 0.24, 0.00055)]


def path_array(case):
    return np.array([[p["eps0"], p["kappa"]] for p in case["deformation_path"]])


def rel_err_of_peak(a, b):
    """max |a - b| / max |b| over a history (the 'within x of peak response' measure)."""
    a = np.asarray(a)
    b = np.asarray(b)
    peak = np.max(np.abs(b))
    if peak == 0.0:
        return float(np.max(np.abs(a - b)))
    return float(np.max(np.abs(a - b)) / peak)


def planar_frame_3d(case2: dict) -> dict:
    """The same plane frame as a 3D model: the 2D plane becomes the global x-z plane, the
    out-of-plane dofs (y translation, rotations about x and z) are restrained, and each
    member's vecxz makes its local y the 2D local y, so the 3D beam-columns bend about local z
    exactly as the 2D ones do.  Displacement records map (ux, uy, rz) -> (ux, uz, -ry)."""
    import copy

    c = copy.deepcopy(case2)
    c["model"] = {"ndm": 3, "ndf": 6}
    for n in c["nodes"]:
        x, y = n["x"], n["y"]
        n["x"], n["y"], n["z"] = x, 0.0, y
        base = bool(n.get("constraints"))
        n["constraints"] = [1, 2, 3, 4, 5, 6] if base else [2, 4, 6]
    nodes = {n["id"]: n for n in c["nodes"]}
    for e in c["elements"]:
        e["type"] = e["type"].replace("2d", "3d")
        a, b = nodes[e["nodes"][0]], nodes[e["nodes"][1]]
        vertical = abs(b["z"] - a["z"]) > 0.0
        e["vecxz"] = [0.0, 1.0, 0.0] if vertical else [0.0, -1.0, 0.0]
    for s in c["sections"]:
        s["type"] = "FiberSection3d"
        s["params"]["G"] = 12.5e9
        s["params"]["J"] = 0.01
    for m in c["masses"]:
        m["dof"] = {1: 1, 2: 3}[m["dof"]]
    for r in c["recorders"]:
        if r["type"] == "node_displacement":
            r["dofs"] = [1, 3, 5]
    return c


def single_element_3d(etype: str, geom: str = "Linear", end=(3.0, 1.0, 2.0), vecxz=None,
                      nonlinear: bool = True) -> dict:
    """One free-free 3D beam-column (node 1 at the origin, node 2 at ``end``) with the RC
    FiberSection3d of the synthetic frames, or an all-elastic copy of its fiber layout."""
    from strut_b200 import workloads as W

    if nonlinear:
        mats = [{"id": 1, "type": "Concrete02", "params": dict(W.CORE)},
                {"id": 2, "type": "Concrete02", "params": dict(W.COVER)},
                {"id": 3, "type": "Steel02", "params": dict(W.STEEL)}]
        sec = W.rc_section(1, 0.4, 0.6, three_d=True)
    else:
        mats = [{"id": 1, "type": "Elastic", "params": {"E": 3.0e10}}]
        sec = W.rc_section(1, 0.4, 0.6, core_mat=1, cover_mat=1, steel_mat=1, three_d=True)
    el = {"id": 1, "type": etype, "nodes": [1, 2], "section": 1, "geomTransf": geom,
          "integration": "Lobatto", "num_int_pts": 5}
    if vecxz is not None:
        el["vecxz"] = list(vecxz)
    return {"model": {"ndm": 3, "ndf": 6},
            "nodes": [{"id": 1, "x": 0.0, "y": 0.0, "z": 0.0},
                      {"id": 2, "x": end[0], "y": end[1], "z": end[2]}],
            "materials": mats, "sections": [sec], "elements": [el],
            "masses": [{"node": 2, "dof": 1, "value": 1.0}],
            "analysis": {"type": "transient_nonlinear", "dt": 0.01, "steps": 1,
                         "test_type": "NormDispIncr", "tol": 1e-8}}


def equal_dof_floors_2d(case2: dict) -> dict:
    """The 2D frame with every floor's horizontal displacement tied to its first node by
    equalDOF (Transformation handler); the tied nodes' horizontal masses move to that node."""
    import copy

    c = copy.deepcopy(case2)
    by_y = {}
    for n in c["nodes"]:
        if n.get("constraints"):
            continue
        by_y.setdefault(n["y"], []).append(n["id"])
    mpcs = []
    moved = {}
    for y, ids in by_y.items():
        master = ids[0]
        for nid in ids[1:]:
            mpcs.append({"type": "equalDOF", "retained_node": master, "constrained_node": nid,
                         "dofs": [1]})
            moved[nid] = master
    masses = []
    extra = {}
    for m in c["masses"]:
        if m["dof"] == 1 and m["node"] in moved:
            extra[moved[m["node"]]] = extra.get(moved[m["node"]], 0.0) + m["value"]
        else:
            masses.append(m)
    for m in masses:
        if m["dof"] == 1 and m["node"] in extra:
            m["value"] += extra[m["node"]]
    c["masses"] = masses
    c["mp_constraints"] = mpcs
    c["analysis"]["constraints"] = "Transformation"
    return c


def transformation_matrix(m_red, m_full):
    """T with u_free(m_full) = T u_free(m_red) for a model and its copy without constraints."""
    import numpy as np

    T = np.zeros((m_full.num_free, m_red.num_free))
    for dof in range(m_red.num_dofs):
        f2 = m_full.free_index[dof]
        if f2 < 0:
            continue
        f = m_red.free_index[dof]
        if f >= 0:
            T[f2, f] = 1.0
        elif dof in m_red.slaves:
            for md, c in m_red.slaves[dof]:
                if m_red.free_index[md] >= 0:
                    T[f2, m_red.free_index[md]] += c
    return T


def band_to_dense(band, n, bw):
    import numpy as np

    K = np.zeros((n, n))
    for i in range(n):
        for o in range(band.shape[1]):
            j = i + o - bw
            if 0 <= j < n:
                K[i, j] = band[i, o]
    return K
