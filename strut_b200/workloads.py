"""Synthetic RC-frame workloads in Strut's JSON schema (seeded, no external data).

* ``rc_frame_case``: a 2D reinforced-concrete moment frame of forceBeamColumn2d elements with
  fiber sections (confined Concrete02 core, unconfined Concrete02 cover, Steel02 bars), lumped
  floor masses, Rayleigh damping fitted to two modes of the initial stiffness, Newmark
  (gamma 0.5, beta 0.25), Newton with NormDispIncr, BandGeneral.
* ``kanai_tajimi_record``: Gaussian white noise through the Kanai-Tajimi filter
  H(s) = (wg^2 + 2 zg wg s) / (s^2 + 2 zg wg s + wg^2) (bilinear transform), a trapezoid
  envelope (rise, hold, decay) and scaling to a target peak ground acceleration.
* ``batched_frames``: the 256-frame batch (stories U{3..12}, bays U{2..5}, wg U(8, 25) rad/s,
  PGA U(0.2, 0.6) g, record i seeded with 1000 + i).
* ``rc_frame3d_case``: a 3D RC moment frame (z vertical) of forceBeamColumn3d or
  dispBeamColumn3d elements with FiberSection3d sections (same fiber layout as the 2D
  sections, plus G and J for torsion), masses on the three translations of every floor node,
  one or two horizontal records.

Builder choices that the workload description leaves open (recorded here): cover 0.04 m; the
cover concrete is fpc -30 MPa, epsc0 -0.002, fpcu 0, epscu -0.004 with the core's rat, ft and
Ets; masses act on both translational dofs of every floor node; Rayleigh is written as
``{alphaM, betaKInit}``; no gravity load.
"""
from __future__ import annotations

import math

import numpy as np

from .integration import beam_integration_rule

G = 9.81

CORE = {"fpc": -30.0e6, "epsc0": -0.002, "fpcu": -6.0e6, "epscu": -0.006,
        "rat": 0.1, "ft": 3.0e6, "Ets": 1500.0e6}
COVER = {"fpc": -30.0e6, "epsc0": -0.002, "fpcu": 0.0, "epscu": -0.004,
         "rat": 0.1, "ft": 3.0e6, "Ets": 1500.0e6}
STEEL = {"Fy": 420.0e6, "E0": 200.0e9, "b": 0.01, "R0": 18.0, "cR1": 0.925, "cR2": 0.15}
BAR_AREA = 500.0e-6
COVER_T = 0.04


def rc_section_208(sec_id: int, width: float, depth: float, core_mat=1, cover_mat=2,
                   steel_mat=3, G: float = 12.5e9) -> dict:
    """FiberSection3d with ~200 fibers: a 12x12 confined core, 20-fiber top and bottom cover
    layers, 8-fiber side covers, 2 x 4 bars (208 fibers)."""
    h2, b2, c = 0.5 * depth, 0.5 * width, COVER_T
    b, h = min(width, depth), max(width, depth)
    beta = 1.0 / 3.0 - 0.21 * (b / h) * (1.0 - (b / h) ** 4 / 12.0)
    return {
        "id": sec_id,
        "type": "FiberSection3d",
        "params": {
            "patches": [
                {"type": "rect", "material": core_mat, "num_subdiv_y": 12, "num_subdiv_z": 12,
                 "y_i": -(h2 - c), "z_i": -(b2 - c), "y_j": h2 - c, "z_j": b2 - c},
                {"type": "rect", "material": cover_mat, "num_subdiv_y": 1, "num_subdiv_z": 20,
                 "y_i": h2 - c, "z_i": -b2, "y_j": h2, "z_j": b2},
                {"type": "rect", "material": cover_mat, "num_subdiv_y": 1, "num_subdiv_z": 20,
                 "y_i": -h2, "z_i": -b2, "y_j": -(h2 - c), "z_j": b2},
                {"type": "rect", "material": cover_mat, "num_subdiv_y": 8, "num_subdiv_z": 1,
                 "y_i": -(h2 - c), "z_i": b2 - c, "y_j": h2 - c, "z_j": b2},
                {"type": "rect", "material": cover_mat, "num_subdiv_y": 8, "num_subdiv_z": 1,
                 "y_i": -(h2 - c), "z_i": -b2, "y_j": h2 - c, "z_j": -(b2 - c)},
            ],
            "layers": [
                {"type": "straight", "material": steel_mat, "num_bars": 4, "bar_area": BAR_AREA,
                 "y_start": h2 - c, "z_start": -(b2 - c), "y_end": h2 - c, "z_end": b2 - c},
                {"type": "straight", "material": steel_mat, "num_bars": 4, "bar_area": BAR_AREA,
                 "y_start": -(h2 - c), "z_start": -(b2 - c), "y_end": -(h2 - c), "z_end": b2 - c},
            ],
            "G": G,
            "J": beta * b ** 3 * h,
        },
    }


def rc_section(sec_id: int, width: float, depth: float, core_mat=1, cover_mat=2, steel_mat=3,
               three_d: bool = False, G: float = 12.5e9):
    """10x10 confined core, two 20-fiber cover layers, 2 x 4 bars: 148 fibers.  With three_d
    the section is a FiberSection3d whose torsional constant is the rectangle's
    J = beta * b^3 * h (beta from b/h) with shear modulus G."""
    h2, b2, c = 0.5 * depth, 0.5 * width, COVER_T
    if three_d:
        sec = rc_section(sec_id, width, depth, core_mat, cover_mat, steel_mat)
        sec["type"] = "FiberSection3d"
        b, h = min(width, depth), max(width, depth)
        beta = 1.0 / 3.0 - 0.21 * (b / h) * (1.0 - (b / h) ** 4 / 12.0)
        sec["params"]["G"] = G
        sec["params"]["J"] = beta * b ** 3 * h
        return sec
    return {
        "id": sec_id,
        "type": "FiberSection2d",
        "params": {
            "patches": [
                {"type": "rect", "material": core_mat, "num_subdiv_y": 10, "num_subdiv_z": 10,
                 "y_i": -(h2 - c), "z_i": -(b2 - c), "y_j": h2 - c, "z_j": b2 - c},
                {"type": "rect", "material": cover_mat, "num_subdiv_y": 1, "num_subdiv_z": 20,
                 "y_i": h2 - c, "z_i": -b2, "y_j": h2, "z_j": b2},
                {"type": "rect", "material": cover_mat, "num_subdiv_y": 1, "num_subdiv_z": 20,
                 "y_i": -h2, "z_i": -b2, "y_j": -(h2 - c), "z_j": b2},
            ],
            "layers": [
                {"type": "straight", "material": steel_mat, "num_bars": 4, "bar_area": BAR_AREA,
                 "y_start": h2 - c, "z_start": -(b2 - c), "y_end": h2 - c, "z_end": b2 - c},
                {"type": "straight", "material": steel_mat, "num_bars": 4, "bar_area": BAR_AREA,
                 "y_start": -(h2 - c), "z_start": -(b2 - c), "y_end": -(h2 - c), "z_end": b2 - c},
            ],
        },
    }


def kanai_tajimi_record(seed: int, n: int, dt: float, wg: float = 15.0, zg: float = 0.6,
                        pga_g: float = 0.35, rise: float = 2.0, hold: float = 10.0,
                        decay: float = 8.0) -> np.ndarray:
    """Ground acceleration samples [m/s^2], n samples at dt."""
    from scipy import signal

    rng = np.random.default_rng(seed)
    w = rng.standard_normal(n)
    b_s = [2.0 * zg * wg, wg * wg]
    a_s = [1.0, 2.0 * zg * wg, wg * wg]
    bz, az = signal.bilinear(b_s, a_s, fs=1.0 / dt)
    ag = signal.lfilter(bz, az, w)
    t = np.arange(n) * dt
    env = np.where(t < rise, t / rise,
                   np.where(t < rise + hold, 1.0,
                            np.clip(1.0 - (t - rise - hold) / decay, 0.0, 1.0)))
    ag = ag * env
    peak = np.max(np.abs(ag))
    if peak > 0.0:
        ag = ag * (pga_g * G / peak)
    return ag


def _section_initial_props(sec: dict, mats: dict):
    """EA, ES, EI about the area centroid from the fibers' initial tangents."""
    from .model import discretize_section

    cells = discretize_section(sec["params"])
    area = sum(c[2] for c in cells)
    ybar = sum(c[2] * c[0] for c in cells) / area
    EA = ES = EI = 0.0
    for (y, _z, a, m) in cells:
        mat = mats[m]
        if mat["type"] == "Concrete02":
            E = 2.0 * mat["params"]["fpc"] / mat["params"]["epsc0"]
        elif mat["type"] in ("Steel02", "Steel01"):
            E = mat["params"]["E0"]
        else:
            E = mat["params"]["E"]
        yr = y - ybar
        EA += E * a
        ES += -E * a * yr
        EI += E * a * yr * yr
    return EA, ES, EI


def initial_stiffness(case: dict) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """Dense initial K_ff, lumped M_ff diagonal and free map of a frame case (numpy)."""
    nodes = case["nodes"]
    idx = {n["id"]: i for i, n in enumerate(nodes)}
    ndof = 3 * len(nodes)
    fixed = np.zeros(ndof, dtype=bool)
    for i, n in enumerate(nodes):
        for d in n.get("constraints", []) or []:
            fixed[3 * i + d - 1] = True
    free = np.where(~fixed)[0]
    mats = {m["id"]: m for m in case["materials"]}
    secs = {s["id"]: _section_initial_props(s, mats) for s in case["sections"]}
    K = np.zeros((ndof, ndof))
    for e in case["elements"]:
        ni, nj = idx[e["nodes"][0]], idx[e["nodes"][1]]
        x1, y1 = nodes[ni]["x"], nodes[ni]["y"]
        x2, y2 = nodes[nj]["x"], nodes[nj]["y"]
        L = math.hypot(x2 - x1, y2 - y1)
        c, s = (x2 - x1) / L, (y2 - y1) / L
        EA, ES, EI = secs[e["section"]]
        fs = np.linalg.inv(np.array([[EA, ES], [ES, EI]]))
        xis, ws = beam_integration_rule(e.get("integration", "Lobatto"), e.get("num_int_pts", 3))
        F = np.zeros((3, 3))
        for xi, w in zip(xis, ws):
            b = np.array([[1.0, 0.0, 0.0], [0.0, xi - 1.0, xi]])
            F += w * L * b.T @ fs @ b
        kb = np.linalg.inv(F)
        a = np.array([[-1, 0, 0, 1, 0, 0],
                      [0, 1 / L, 1, 0, -1 / L, 0],
                      [0, 1 / L, 0, 0, -1 / L, 1]], dtype=float)
        kl = a.T @ kb @ a
        T = np.zeros((6, 6))
        for o in (0, 3):
            T[o:o + 2, o:o + 2] = [[c, s], [-s, c]]
            T[o + 2, o + 2] = 1.0
        kg = T.T @ kl @ T
        dofs = [3 * ni, 3 * ni + 1, 3 * ni + 2, 3 * nj, 3 * nj + 1, 3 * nj + 2]
        K[np.ix_(dofs, dofs)] += kg
    M = np.zeros(ndof)
    for m in case.get("masses", []):
        M[3 * idx[m["node"]] + m["dof"] - 1] += m["value"]
    return K[np.ix_(free, free)], M[free], free


def rayleigh_from_modes(case: dict, zeta: float = 0.05, modes=(1, 3)):
    """alphaM, betaK giving ``zeta`` in the two given modes of the initial system."""
    from scipy import linalg

    K, M, _free = initial_stiffness(case)
    m_idx = np.where(M > 0.0)[0]
    z_idx = np.where(M == 0.0)[0]
    if len(z_idx):
        Kmm = K[np.ix_(m_idx, m_idx)]
        Kmz = K[np.ix_(m_idx, z_idx)]
        Kzz = K[np.ix_(z_idx, z_idx)]
        Kc = Kmm - Kmz @ np.linalg.solve(Kzz, Kmz.T)
    else:
        Kc = K
    lam = linalg.eigh(Kc, np.diag(M[m_idx]), eigvals_only=True)
    w = np.sqrt(np.sort(lam))
    wi, wj = w[modes[0] - 1], w[modes[1] - 1]
    alpha = 2.0 * zeta * wi * wj / (wi + wj)
    beta = 2.0 * zeta / (wi + wj)
    return float(alpha), float(beta), w


def rc_frame_case(stories: int = 3, bays: int = 3, story_h: float = 3.6, bay_w: float = 6.0,
                  nip: int = 5, floor_mass: float = 60.0e3, dt: float = 0.01, steps: int = 2000,
                  seed: int = 1000, wg: float = 15.0, zg: float = 0.6, pga_g: float = 0.35,
                  tol: float = 1.0e-8, max_iters: int = 20, element: str = "forceBeamColumn2d",
                  system: str = "BandGeneral", zeta: float = 0.05, record=None,
                  geom: str = "Linear") -> dict:
    nodes = []
    nid = 1
    grid = {}
    for i in range(stories + 1):
        for j in range(bays + 1):
            n = {"id": nid, "x": j * bay_w, "y": i * story_h}
            if i == 0:
                n["constraints"] = [1, 2, 3]
            nodes.append(n)
            grid[(i, j)] = nid
            nid += 1
    elements = []
    eid = 1
    for i in range(stories):
        for j in range(bays + 1):
            elements.append({"id": eid, "type": element, "nodes": [grid[(i, j)], grid[(i + 1, j)]],
                             "section": 1, "geomTransf": geom, "integration": "Lobatto",
                             "num_int_pts": nip})
            eid += 1
    for i in range(1, stories + 1):
        for j in range(bays):
            elements.append({"id": eid, "type": element, "nodes": [grid[(i, j)], grid[(i, j + 1)]],
                             "section": 2, "geomTransf": geom, "integration": "Lobatto",
                             "num_int_pts": nip})
            eid += 1
    masses = []
    for i in range(1, stories + 1):
        for j in range(bays + 1):
            masses.append({"node": grid[(i, j)], "dof": 1, "value": floor_mass})
            masses.append({"node": grid[(i, j)], "dof": 2, "value": floor_mass})
    n_samples = steps + 1
    if record is None:
        record = kanai_tajimi_record(seed, n_samples, dt, wg=wg, zg=zg, pga_g=pga_g)
    case = {
        "schema_version": "1.0",
        "metadata": {"name": f"rc_frame_{stories}s{bays}b_seed{seed}", "units": "SI"},
        "model": {"ndm": 2, "ndf": 3},
        "nodes": nodes,
        "materials": [
            {"id": 1, "type": "Concrete02", "params": dict(CORE)},
            {"id": 2, "type": "Concrete02", "params": dict(COVER)},
            {"id": 3, "type": "Steel02", "params": dict(STEEL)},
        ],
        "sections": [rc_section(1, 0.5, 0.5), rc_section(2, 0.4, 0.6)],
        "elements": elements,
        "masses": masses,
        "time_series": [{"type": "Path", "tag": 1, "dt": dt, "values": [float(v) for v in record]}],
        "pattern": {"type": "UniformExcitation", "tag": 1, "direction": 1, "accel": 1},
        "analysis": {"type": "transient_nonlinear", "steps": steps, "dt": dt,
                     "integrator": {"type": "Newmark", "gamma": 0.5, "beta": 0.25},
                     "algorithm": "Newton", "test_type": "NormDispIncr", "tol": tol,
                     "max_iters": max_iters, "system": system, "numberer": "RCM"},
        "recorders": [
            {"type": "node_displacement", "nodes": [grid[(stories, 0)]], "dofs": [1, 2, 3],
             "output": "roof"},
            {"type": "element_force", "elements": [1], "output": "base_col"},
        ],
    }
    alpha, beta, _w = rayleigh_from_modes(case, zeta=zeta)
    case["rayleigh"] = {"alphaM": alpha, "betaKInit": beta}
    return case


def _section3d_initial_flex(sec: dict, mats: dict) -> np.ndarray:
    """3x3 initial flexibility (N, My, Mz) of a FiberSection3d from the fibers' initial
    tangents, about the area centroid (fiber3d.mojo:191-256 sums with E0)."""
    from .model import discretize_section

    cells = discretize_section(sec["params"])
    area = sum(c[2] for c in cells)
    ybar = sum(c[2] * c[0] for c in cells) / area
    zbar = sum(c[2] * c[1] for c in cells) / area
    ks = np.zeros((3, 3))
    for (y, z, a, m) in cells:
        mat = mats[m]
        if mat["type"] == "Concrete02":
            E = 2.0 * mat["params"]["fpc"] / mat["params"]["epsc0"]
        elif mat["type"] in ("Steel02", "Steel01"):
            E = mat["params"]["E0"]
        else:
            E = mat["params"]["E"]
        yr, zr = y - ybar, z - zbar
        ea = E * a
        ks += ea * np.array([[1.0, zr, -yr], [zr, zr * zr, -zr * yr], [-yr, -zr * yr, yr * yr]])
    return np.linalg.inv(ks)


def _rotation3d(p1, p2, vecxz=None) -> np.ndarray:
    """Local axes rows (x, y, z) as in elements/utils.mojo:77-140."""
    d = np.asarray(p2, float) - np.asarray(p1, float)
    lx = d / np.linalg.norm(d)
    if vecxz is None:
        v = np.array([1.0, 0.0, 0.0])
        if abs(lx @ v) >= 0.9:
            v = np.array([0.0, 1.0, 0.0])
            if abs(lx @ v) >= 0.9:
                v = np.array([0.0, 0.0, 1.0])
    else:
        v = np.asarray(vecxz, float)
    ly = np.cross(v, lx)
    ly /= np.linalg.norm(ly)
    lz = np.cross(lx, ly)
    return np.array([lx, ly, lz])


def initial_stiffness_3d(case: dict) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """Dense initial K_ff, lumped M_ff diagonal and free map of a 3D frame case (numpy): the
    force-based element flexibility from the sections' initial tangents, GJ/L torsion."""
    nodes = case["nodes"]
    idx = {n["id"]: i for i, n in enumerate(nodes)}
    ndof = 6 * len(nodes)
    fixed = np.zeros(ndof, dtype=bool)
    for i, n in enumerate(nodes):
        for d in n.get("constraints", []) or []:
            fixed[6 * i + d - 1] = True
    free = np.where(~fixed)[0]
    mats = {m["id"]: m for m in case["materials"]}
    # the frame alone: slab shells (if any) do not enter the Rayleigh coefficients
    fsecs = [s for s in case["sections"] if s["type"] == "FiberSection3d"]
    flex = {s["id"]: _section3d_initial_flex(s, mats) for s in fsecs}
    gj = {s["id"]: s["params"]["G"] * s["params"]["J"] for s in fsecs}
    K = np.zeros((ndof, ndof))
    for e in case["elements"]:
        if e["type"] == "shell":
            continue
        ni, nj = idx[e["nodes"][0]], idx[e["nodes"][1]]
        p1 = [nodes[ni][k] for k in ("x", "y", "z")]
        p2 = [nodes[nj][k] for k in ("x", "y", "z")]
        L = float(np.linalg.norm(np.subtract(p2, p1)))
        fs = flex[e["section"]]
        xis, ws = beam_integration_rule(e.get("integration", "Lobatto"), e.get("num_int_pts", 3))
        F = np.zeros((5, 5))
        for xi, w in zip(xis, ws):
            b = np.array([[1.0, 0.0, 0.0, 0.0, 0.0],
                          [0.0, 0.0, 0.0, xi - 1.0, xi],
                          [0.0, xi - 1.0, xi, 0.0, 0.0]])
            F += w * L * b.T @ fs @ b
        kb = np.linalg.inv(F)
        a = np.zeros((6, 12))
        a[0, 0], a[0, 6] = -1.0, 1.0
        a[1, 1], a[1, 5], a[1, 7] = 1.0 / L, 1.0, -1.0 / L
        a[2, 1], a[2, 7], a[2, 11] = 1.0 / L, -1.0 / L, 1.0
        a[3, 2], a[3, 4], a[3, 8] = -1.0 / L, 1.0, 1.0 / L
        a[4, 2], a[4, 8], a[4, 10] = -1.0 / L, 1.0 / L, 1.0
        a[5, 3], a[5, 9] = -1.0, 1.0
        kb6 = np.zeros((6, 6))
        kb6[:5, :5] = kb
        kb6[5, 5] = gj[e["section"]] / L
        kl = a.T @ kb6 @ a
        R = _rotation3d(p1, p2, e.get("vecxz"))
        T = np.kron(np.eye(4), R)
        kg = T.T @ kl @ T
        dofs = [6 * ni + k for k in range(6)] + [6 * nj + k for k in range(6)]
        K[np.ix_(dofs, dofs)] += kg
    M = np.zeros(ndof)
    for m in case.get("masses", []):
        M[6 * idx[m["node"]] + m["dof"] - 1] += m["value"]
    mpcs = case.get("mp_constraints") or []
    if mpcs:
        # Transformation: u = T u_r, the slaves following their retained dofs
        slave = {}
        for c in mpcs:
            ri, ci = idx[c["retained_node"]], idx[c["constrained_node"]]
            for row, cd in enumerate(c["constrained_dofs"]):
                slave[6 * ci + cd - 1] = [(6 * ri + rd - 1, c["matrix"][row][col])
                                          for col, rd in enumerate(c["retained_dofs"])]
        keep = [d for d in range(ndof) if not fixed[d] and d not in slave]
        col = {d: k for k, d in enumerate(keep)}
        T = np.zeros((ndof, len(keep)))
        for d in keep:
            T[d, col[d]] = 1.0
        for d, terms in slave.items():
            for md, c in terms:
                T[d, col[md]] += c
        Kr = T.T @ K @ T
        Mr = np.diag(T.T @ np.diag(M) @ T)
        return Kr, Mr, np.asarray(keep)
    return K[np.ix_(free, free)], M[free], free


def rc_frame3d_case(stories: int = 2, bays_x: int = 2, bays_y: int = 2, story_h: float = 3.6,
                    bay_w: float = 6.0, nip: int = 5, floor_mass: float = 60.0e3,
                    dt: float = 0.01, steps: int = 2000, seed: int = 1000, wg: float = 15.0,
                    zg: float = 0.6, pga_g: float = 0.35, tol: float = 1.0e-8,
                    max_iters: int = 20, element: str = "forceBeamColumn3d",
                    system: str = "BandGeneral", zeta: float = 0.05, geom: str = "Linear",
                    bidirectional: bool = False, record_elements=(1,), diaphragm: bool = False,
                    beam_element: str | None = None, sections=None,
                    diaphragm_mass: float | None = None, slabs: dict | None = None,
                    slab_mesh: int = 1) -> dict:
    """3D RC frame: columns along z, beams along x and y, base fixed in all six dofs.  With
    ``diaphragm`` every floor is a rigid diaphragm (perp_dirn 3) retained by its central node,
    which carries the floor's horizontal masses and rotational inertia; the other nodes keep
    their vertical mass only.  ``beam_element`` (default: ``element``) sets the beams' type;
    ``sections`` replaces the (column, beam) sections; ``diaphragm_mass`` is the floor's total
    horizontal mass (default: floor_mass per node).  ``slab_mesh`` m > 1 meshes every bay's slab
    with m x m shells: the floor grid gets nodes every bay_w / m, beams are split at them (one
    element per segment), columns stay at the bay corners, and the Rayleigh coefficients are
    those of the same frame with whole-bay beams and no slab."""
    ms = max(1, int(slab_mesh))
    if ms > 1:
        coarse = rc_frame3d_case(stories, bays_x, bays_y, story_h, bay_w, nip, floor_mass, dt, steps,
                                 seed, wg, zg, pga_g, tol, max_iters, element, system, zeta, geom,
                                 bidirectional, record_elements, diaphragm, beam_element, sections,
                                 diaphragm_mass, None, 1)
    bays_x, bays_y, bay_w = bays_x * ms, bays_y * ms, bay_w / ms
    nodes = []
    grid = {}
    nid = 1
    for k in range(stories + 1):
        for j in range(bays_y + 1):
            for i in range(bays_x + 1):
                if k == 0 and (i % ms or j % ms):
                    continue  # no column below a slab-only node
                n = {"id": nid, "x": i * bay_w, "y": j * bay_w, "z": k * story_h}
                if k == 0:
                    n["constraints"] = [1, 2, 3, 4, 5, 6]
                nodes.append(n)
                grid[(k, j, i)] = nid
                nid += 1
    elements = []
    eid = 1

    def add(n1, n2, sec, etype=element):
        nonlocal eid
        elements.append({"id": eid, "type": etype, "nodes": [n1, n2], "section": sec,
                         "geomTransf": geom, "integration": "Lobatto", "num_int_pts": nip})
        eid += 1

    for k in range(stories):
        for j in range(0, bays_y + 1, ms):
            for i in range(0, bays_x + 1, ms):
                add(grid[(k, j, i)], grid[(k + 1, j, i)], 1)
    bt = beam_element or element
    for k in range(1, stories + 1):
        for j in range(0, bays_y + 1, ms):
            for i in range(bays_x):
                add(grid[(k, j, i)], grid[(k, j, i + 1)], 2, bt)
        for j in range(bays_y):
            for i in range(0, bays_x + 1, ms):
                add(grid[(k, j, i)], grid[(k, j + 1, i)], 2, bt)
    if slabs:
        # one ShellMITC4 per bay and floor on the beam-column joints (counter-clockwise seen
        # from +z), ElasticMembranePlateSection {E, nu, h, rho}
        for k in range(1, stories + 1):
            for j in range(bays_y):
                for i in range(bays_x):
                    elements.append({"id": eid, "type": "shell", "section": 3,
                                     "nodes": [grid[(k, j, i)], grid[(k, j, i + 1)],
                                               grid[(k, j + 1, i + 1)], grid[(k, j + 1, i)]]})
                    eid += 1
    masses = []
    mpcs = []
    jm, im = bays_y // 2, bays_x // 2
    for k in range(1, stories + 1):
        if not diaphragm:
            for j in range(bays_y + 1):
                for i in range(bays_x + 1):
                    for d in (1, 2, 3):
                        masses.append({"node": grid[(k, j, i)], "dof": d, "value": floor_mass})
            continue
        master = grid[(k, jm, im)]
        xm, ym = im * bay_w, jm * bay_w
        total, inertia = 0.0, 0.0
        n_floor = (bays_x + 1) * (bays_y + 1)
        m_node = floor_mass if diaphragm_mass is None else diaphragm_mass / n_floor
        for j in range(bays_y + 1):
            for i in range(bays_x + 1):
                node = grid[(k, j, i)]
                masses.append({"node": node, "dof": 3, "value": m_node})
                dx, dy = i * bay_w - xm, j * bay_w - ym
                total += m_node
                inertia += m_node * (dx * dx + dy * dy)
                if node == master:
                    continue
                mpcs.append({"type": "rigidDiaphragm", "retained_node": master,
                             "constrained_node": node, "perp_dirn": 3,
                             "constrained_dofs": [1, 2, 6], "retained_dofs": [1, 2, 6],
                             "matrix": [[1.0, 0.0, -dy], [0.0, 1.0, dx], [0.0, 0.0, 1.0]],
                             "dx": dx, "dy": dy, "dz": 0.0})
        masses += [{"node": master, "dof": 1, "value": total},
                   {"node": master, "dof": 2, "value": total},
                   {"node": master, "dof": 6, "value": inertia}]
    n_samples = steps + 1
    series = [{"type": "Path", "tag": 1, "dt": dt,
               "values": [float(v) for v in kanai_tajimi_record(seed, n_samples, dt, wg=wg,
                                                               zg=zg, pga_g=pga_g)]}]
    pattern = {"type": "UniformExcitation", "tag": 1, "direction": 1, "accel": 1}
    if bidirectional:
        series.append({"type": "Path", "tag": 2, "dt": dt,
                       "values": [float(v) for v in kanai_tajimi_record(
                           seed + 500000, n_samples, dt, wg=wg, zg=zg, pga_g=pga_g)]})
        pattern = [pattern, {"type": "UniformExcitation", "tag": 2, "direction": 2, "accel": 2}]
    top = grid[(stories, bays_y, bays_x)]
    case = {
        "schema_version": "1.0",
        "metadata": {"name": f"rc_frame3d_{stories}s{bays_x}x{bays_y}b_seed{seed}",
                     "units": "SI"},
        "model": {"ndm": 3, "ndf": 6},
        "nodes": nodes,
        "materials": [
            {"id": 1, "type": "Concrete02", "params": dict(CORE)},
            {"id": 2, "type": "Concrete02", "params": dict(COVER)},
            {"id": 3, "type": "Steel02", "params": dict(STEEL)},
        ],
        "sections": list(sections) if sections else [rc_section(1, 0.5, 0.5, three_d=True),
                                                      rc_section(2, 0.4, 0.6, three_d=True)] + ([{"id": 3, "type": "ElasticMembranePlateSection", "params": dict(slabs)}] if slabs else []),
        "elements": elements,
        "masses": masses,
        "time_series": series,
        "pattern": pattern,
        "analysis": {"type": "transient_nonlinear", "steps": steps, "dt": dt,
                     "integrator": {"type": "Newmark", "gamma": 0.5, "beta": 0.25},
                     "algorithm": "Newton", "test_type": "NormDispIncr", "tol": tol,
                     "max_iters": max_iters, "system": system, "numberer": "RCM"},
        "recorders": [
            {"type": "node_displacement", "nodes": [top], "dofs": [1, 2, 3, 4, 5, 6],
             "output": "roof"},
        ],
    }
    if mpcs:
        case["mp_constraints"] = mpcs
        case["analysis"]["constraints"] = "Transformation"
    if record_elements:
        case["recorders"].append({"type": "element_force", "elements": list(record_elements),
                                  "output": "elements"})
    if ms > 1:
        case["rayleigh"] = dict(coarse["rayleigh"])
        return case
    K, M, _free = initial_stiffness_3d(case)
    m_idx = np.where(M > 0.0)[0]
    z_idx = np.where(M == 0.0)[0]
    Kmm = K[np.ix_(m_idx, m_idx)]
    Kmz = K[np.ix_(m_idx, z_idx)]
    Kzz = K[np.ix_(z_idx, z_idx)]
    Kc = Kmm - Kmz @ np.linalg.solve(Kzz, Kmz.T)
    from scipy import linalg

    lam = linalg.eigh(Kc, np.diag(M[m_idx]), eigvals_only=True)
    w = np.sqrt(np.sort(lam))
    wi, wj = w[0], w[2]
    case["rayleigh"] = {"alphaM": float(2.0 * zeta * wi * wj / (wi + wj)),
                        "betaKInit": float(2.0 * zeta / (wi + wj))}
    return case


def tall_frame3d_case(stories: int = 20, bays: int = 6, steps: int = 4000, dt: float = 0.005,
                      seed: int = 7000, pga_g: float = 0.4, record_elements=(1,)) -> dict:
    """The large single-instance 3D RC frame: 20 stories x 6x6 bays of 7 m, story height
    3.5 m (1029 nodes, 980 forceBeamColumn3d columns, 1680 dispBeamColumn3d beams), 5 Lobatto
    points and 208-fiber sections, a rigid diaphragm per floor carrying 400 t, two horizontal
    seeded Kanai-Tajimi records at PGA 0.4 g, dt 0.005 s.  Builder choices: columns
    0.7 x 0.7 m, beams 0.5 x 0.7 m; the diaphragm's rotational inertia is that of the floor's
    nodes with the floor mass spread evenly over them, which also carry it vertically."""
    return rc_frame3d_case(stories=stories, bays_x=bays, bays_y=bays, story_h=3.5, bay_w=7.0,
                           nip=5, dt=dt, steps=steps, seed=seed, pga_g=pga_g,
                           element="forceBeamColumn3d", beam_element="dispBeamColumn3d",
                           diaphragm=True, diaphragm_mass=400.0e3, bidirectional=True,
                           sections=[rc_section_208(1, 0.7, 0.7), rc_section_208(2, 0.5, 0.7)],
                           record_elements=record_elements)


SLAB = {"E": 30.0e9, "nu": 0.2, "h": 0.2, "rho": 0.0}


def slab_frame3d_case(stories: int, bays: int, steps: int = 4000, dt: float = 0.005, seed: int = 8000,
                      pga_g: float = 0.45, wg: float = 15.0, record_elements=(1,)) -> dict:
    """A frame of the batched slab-frame set: a 3D RC frame of `stories` stories and bays x bays
    bays of 7 m (story height 3.5 m), forceBeamColumn3d columns (0.7 x 0.7 m) and dispBeamColumn3d
    beams (0.5 x 0.7 m) with 5 Lobatto points and 208-fiber sections, ShellMITC4 floor slabs on an
    ElasticMembranePlateSection (E 30 GPa, nu 0.2, h 0.2 m, massless) meshed 2 x 2 per bay, a rigid
    diaphragm per floor carrying 400 t, two horizontal seeded Kanai-Tajimi records at `pga_g`."""
    sec = [rc_section_208(1, 0.7, 0.7), rc_section_208(2, 0.5, 0.7),
           {"id": 3, "type": "ElasticMembranePlateSection", "params": dict(SLAB)}]
    return rc_frame3d_case(stories=stories, bays_x=bays, bays_y=bays, story_h=3.5, bay_w=7.0, nip=5, dt=dt,
                           steps=steps, seed=seed, pga_g=pga_g, wg=wg, element="forceBeamColumn3d",
                           beam_element="dispBeamColumn3d", diaphragm=True, diaphragm_mass=400.0e3,
                           bidirectional=True, sections=sec, slabs=dict(SLAB), slab_mesh=2,
                           record_elements=record_elements)


def slab_frame_params(n: int, base_seed: int = 8000, max_bays: int = 6):
    """Sizes and records of the batched slab-frame set: stories U{10..30}, bays U{4..max_bays},
    PGA U(0.3, 0.6) g, wg U(8, 25) rad/s, record i seeded with base_seed + i."""
    out = []
    for i in range(n):
        rng = np.random.default_rng(base_seed + i)
        out.append(dict(stories=int(rng.integers(10, 31)), bays=int(rng.integers(4, max_bays + 1)),
                        pga_g=float(rng.uniform(0.3, 0.6)), wg=float(rng.uniform(8.0, 25.0)),
                        seed=base_seed + i))
    return out


def batched_frame_params(n: int = 256, base_seed: int = 1000):
    out = []
    for i in range(n):
        rng = np.random.default_rng(base_seed + i)
        stories = int(rng.integers(3, 13))
        bays = int(rng.integers(2, 6))
        wg = float(rng.uniform(8.0, 25.0))
        pga = float(rng.uniform(0.2, 0.6))
        out.append(dict(stories=stories, bays=bays, wg=wg, pga_g=pga, seed=base_seed + i))
    return out


def batched_frames(n: int = 256, steps: int = 2000, dt: float = 0.01, base_seed: int = 1000,
                   **kw):
    return [rc_frame_case(stories=p["stories"], bays=p["bays"], wg=p["wg"], pga_g=p["pga_g"],
                          seed=p["seed"], steps=steps, dt=dt, **kw)
            for p in batched_frame_params(n, base_seed)]
