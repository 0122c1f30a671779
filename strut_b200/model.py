"""Strut JSON case -> C-ABI model description.

This is the host-side set-up that Strut's loader performs before the transient loop
(``src/mojo/solver/run_case/loader.mojo``): material definitions with Strut's defaults and
sign conventions (loader.mojo:913-1100), fiber discretisation of patches / layers / direct
fibers (``src/mojo/sections/fiber2d.mojo:3504-3944``), beam integration rules,
natural-order DOF numbering of the transient path (loader.mojo:2393-2450, RCM not applied),
lumped masses (loader.mojo:1984-2000), Rayleigh coefficients and one UniformExcitation with a
Path time series (``transient_nonlinear.mojo:1823-1852``).

The schema is Strut's own (``docs/harness.md``).  One documented extension: ``pattern`` may
be a list of up to two UniformExcitation patterns (bidirectional records), which Strut's CPU
path cannot express.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np

from . import _abi as A
from .integration import beam_integration_rule


class ModelError(ValueError):
    """Invalid or unsupported input (Strut would abort with the same message)."""


# ---------------------------------------------------------------------------------------
# materials (loader.mojo:913-1100)
# ---------------------------------------------------------------------------------------
def uniaxial_material(mat: dict) -> A.StrutUniMaterial:
    t = mat["type"]
    p = mat.get("params", {})
    m = A.StrutUniMaterial()
    vals = [0.0] * 11
    if t == "Elastic":
        E = float(p["E"])
        if E <= 0.0:
            raise ModelError("Elastic material E must be > 0")
        m.type = A.MAT_ELASTIC
        vals[0] = E
    elif t == "Steel01":
        Fy, E0, b = float(p["Fy"]), float(p["E0"]), float(p["b"])
        if Fy <= 0.0:
            raise ModelError("Steel01 Fy must be > 0")
        if E0 <= 0.0:
            raise ModelError("Steel01 E0 must be > 0")
        if b < 0.0 or b >= 1.0:
            raise ModelError("Steel01 b must be in [0, 1)")
        m.type = A.MAT_STEEL01
        vals[0:3] = [Fy, E0, b]
    elif t == "Steel02":
        Fy, E0, b = float(p["Fy"]), float(p["E0"]), float(p["b"])
        if Fy < 0.0:
            raise ModelError("Steel02 Fy must be >= 0")
        if E0 <= 0.0:
            raise ModelError("Steel02 E0 must be > 0")
        if b < 0.0 or b >= 1.0:
            raise ModelError("Steel02 b must be in [0, 1)")
        has_r0, has_cr1, has_cr2 = "R0" in p, "cR1" in p, "cR2" in p
        has_a = [k in p for k in ("a1", "a2", "a3", "a4")]
        has_sig = "sigInit" in p
        if not (has_r0 == has_cr1 == has_cr2):
            raise ModelError("Steel02 requires R0, cR1, cR2 together")
        if not all(h == has_a[0] for h in has_a):
            raise ModelError("Steel02 requires a1, a2, a3, a4 together")
        if has_a[0] and not has_r0:
            raise ModelError("Steel02 a1-a4 require R0, cR1, cR2")
        if has_sig and not has_a[0]:
            raise ModelError("Steel02 sigInit requires a1-a4 and R0/cR1/cR2")
        R0, cR1, cR2 = 15.0, 0.925, 0.15
        if has_r0:
            R0, cR1, cR2 = float(p["R0"]), float(p["cR1"]), float(p["cR2"])
        if R0 <= 0.0:
            raise ModelError("Steel02 R0 must be > 0")
        if cR2 <= 0.0:
            raise ModelError("Steel02 cR2 must be > 0")
        a1, a2, a3, a4 = 0.0, 1.0, 0.0, 1.0
        if has_a[0]:
            a1, a2, a3, a4 = (float(p[k]) for k in ("a1", "a2", "a3", "a4"))
        if a2 <= 0.0:
            raise ModelError("Steel02 a2 must be > 0")
        if a4 <= 0.0:
            raise ModelError("Steel02 a4 must be > 0")
        sig_init = float(p["sigInit"]) if has_sig else 0.0
        m.type = A.MAT_STEEL02
        vals = [Fy, E0, b, R0, cR1, cR2, a1, a2, a3, a4, sig_init]
    elif t == "Concrete01":
        fpc, epsc0 = float(p["fpc"]), float(p["epsc0"])
        fpcu, epscu = float(p["fpcu"]), float(p["epscu"])
        if fpc > 0.0:
            fpc = -fpc
        if epsc0 > 0.0:
            epsc0 = -epsc0
        if fpcu > 0.0:
            fpcu = -fpcu
        if epscu > 0.0:
            epscu = -epscu
        if fpc >= 0.0:
            raise ModelError("Concrete01 fpc must be < 0")
        if epsc0 >= 0.0:
            raise ModelError("Concrete01 epsc0 must be < 0")
        if epscu >= 0.0:
            raise ModelError("Concrete01 epscu must be < 0")
        if epscu >= epsc0:
            raise ModelError("Concrete01 epscu must be < epsc0")
        if fpcu > 0.0 or fpcu < fpc:
            raise ModelError("Concrete01 fpcu must be between fpc and 0")
        m.type = A.MAT_CONCRETE01
        vals[0:4] = [fpc, epsc0, fpcu, epscu]
    elif t == "Concrete02":
        fpc, epsc0 = float(p["fpc"]), float(p["epsc0"])
        fpcu, epscu = float(p["fpcu"]), float(p["epscu"])
        if fpc > 0.0:
            fpc = -fpc
        if epsc0 > 0.0:
            epsc0 = -epsc0
        if fpcu > 0.0:
            fpcu = -fpcu
        if epscu > 0.0:
            epscu = -epscu
        if fpc >= 0.0:
            raise ModelError("Concrete02 fpc must be < 0")
        if epsc0 >= 0.0:
            raise ModelError("Concrete02 epsc0 must be < 0")
        if epscu >= 0.0:
            raise ModelError("Concrete02 epscu must be < 0")
        if epscu >= epsc0:
            raise ModelError("Concrete02 epscu must be < epsc0")
        if fpcu > 0.0 or fpcu < fpc:
            raise ModelError("Concrete02 fpcu must be between fpc and 0")
        has = ["rat" in p, "ft" in p, "Ets" in p]
        if not (has[0] == has[1] == has[2]):
            raise ModelError("Concrete02 requires rat, ft, Ets together")
        rat = 0.1
        ft = 0.1 * fpc
        if ft < 0.0:
            ft = -ft
        Ets = 0.1 * fpc / epsc0
        if has[0]:
            rat, ft, Ets = float(p["rat"]), float(p["ft"]), float(p["Ets"])
        if rat == 1.0:
            raise ModelError("Concrete02 rat must not be 1")
        if ft < 0.0:
            raise ModelError("Concrete02 ft must be >= 0")
        if Ets <= 0.0:
            raise ModelError("Concrete02 Ets must be > 0")
        m.type = A.MAT_CONCRETE02
        vals[0:7] = [fpc, epsc0, fpcu, epscu, rat, ft, Ets]
    else:
        raise ModelError(f"unsupported uniaxial material type for this path: {t}")
    for i, v in enumerate(vals):
        m.p[i] = v
    return m


# ---------------------------------------------------------------------------------------
# fiber discretisation (fiber2d.mojo:3504-3944)
# ---------------------------------------------------------------------------------------
def discretize_section(params: dict):
    """List of (y, z, area, material_id) in Strut's append order (patches, layers, fibers)."""
    cells = []
    for patch in params.get("patches", []):
        ptype = patch["type"]
        if ptype == "quad":
            ptype = "quadr"
        ny, nz = int(patch["num_subdiv_y"]), int(patch["num_subdiv_z"])
        if ny <= 0 or nz <= 0:
            raise ModelError(f"FiberSection2d patch {ptype} requires num_subdiv_y and num_subdiv_z > 0")
        mat = int(patch["material"])
        if ptype == "rect":
            y_i, z_i, y_j, z_j = (float(patch[k]) for k in ("y_i", "z_i", "y_j", "z_j"))
            y_min, y_max = (y_i, y_j) if y_i <= y_j else (y_j, y_i)
            z_min, z_max = (z_i, z_j) if z_i <= z_j else (z_j, z_i)
            dy_total = y_max - y_min
            dz_total = z_max - z_min
            if dy_total <= 0.0 or dz_total <= 0.0:
                raise ModelError("FiberSection2d patch rect must have non-zero side lengths")
            dy = dy_total / float(ny)
            dz = dz_total / float(nz)
            area = dy * dz
            for iy in range(ny):
                y = y_min + (float(iy) + 0.5) * dy
                for iz in range(nz):
                    z = z_min + (float(iz) + 0.5) * dz
                    cells.append((y, z, area, mat))
        elif ptype == "quadr":
            yi, zi = float(patch["y_i"]), float(patch["z_i"])
            yj, zj = float(patch["y_j"]), float(patch["z_j"])
            yk, zk = float(patch["y_k"]), float(patch["z_k"])
            yl, zl = float(patch["y_l"]), float(patch["z_l"])

            def bil(u, v, a, b, c, d):
                return (1.0 - u) * (1.0 - v) * a + u * (1.0 - v) * b + u * v * c + (1.0 - u) * v * d

            for iy in range(ny):
                u0 = float(iy) / float(ny)
                u1 = float(iy + 1) / float(ny)
                uc = 0.5 * (u0 + u1)
                for iz in range(nz):
                    v0 = float(iz) / float(nz)
                    v1 = float(iz + 1) / float(nz)
                    vc = 0.5 * (v0 + v1)
                    y00, z00 = bil(u0, v0, yi, yj, yk, yl), bil(u0, v0, zi, zj, zk, zl)
                    y10, z10 = bil(u1, v0, yi, yj, yk, yl), bil(u1, v0, zi, zj, zk, zl)
                    y11, z11 = bil(u1, v1, yi, yj, yk, yl), bil(u1, v1, zi, zj, zk, zl)
                    y01, z01 = bil(u0, v1, yi, yj, yk, yl), bil(u0, v1, zi, zj, zk, zl)
                    twice = (y00 * z10 + y10 * z11 + y11 * z01 + y01 * z00
                             - z00 * y10 - z10 * y11 - z11 * y01 - z01 * y00)
                    area = abs(twice) * 0.5
                    if area <= 0.0:
                        raise ModelError("FiberSection2d patch quadr generated zero-area cell")
                    yc = bil(uc, vc, yi, yj, yk, yl)
                    zc = bil(uc, vc, zi, zj, zk, zl)
                    cells.append((yc, zc, area, mat))
        else:
            raise ModelError(f"unsupported FiberSection2d patch type: {ptype}")
    for layer in params.get("layers", []):
        if layer["type"] != "straight":
            raise ModelError(f"unsupported FiberSection2d layer type: {layer['type']}")
        nb = int(layer["num_bars"])
        if nb <= 0:
            raise ModelError("FiberSection2d layer straight requires num_bars > 0")
        ba = float(layer["bar_area"])
        if ba <= 0.0:
            raise ModelError("FiberSection2d layer straight requires bar_area > 0")
        ys, zs = float(layer["y_start"]), float(layer["z_start"])
        ye, ze = float(layer["y_end"]), float(layer["z_end"])
        mat = int(layer["material"])
        if nb == 1:
            cells.append((0.5 * (ys + ye), 0.5 * (zs + ze), ba, mat))
        else:
            for i in range(nb):
                t = float(i) / float(nb - 1)
                cells.append((ys + (ye - ys) * t, zs + (ze - zs) * t, ba, mat))
    for f in params.get("fibers", []):
        if float(f["area"]) <= 0.0:
            raise ModelError("FiberSection2d fiber area must be > 0")
        cells.append((float(f["y"]), float(f["z"]), float(f["area"]), int(f["material"])))
    if not cells:
        raise ModelError("FiberSection2d produced no fibers")
    return cells


def _struct_array(ctype, items):
    arr = (ctype * max(len(items), 1))()
    for i, it in enumerate(items):
        arr[i] = it
    return arr


def _excitation_list(case: dict):
    pat = case.get("pattern")
    if pat is None:
        return []
    pats = pat if isinstance(pat, list) else [pat]
    out = []
    for p in pats:
        if p.get("type") != "UniformExcitation":
            raise ModelError(f"unsupported pattern type for transient path: {p.get('type')}")
        out.append(p)
    if len(out) > 2:
        raise ModelError("at most two UniformExcitation patterns are supported")
    return out


@dataclass
class Model:
    """One analysis instance built from a Strut JSON case."""

    case: dict
    node_ids: list = field(default_factory=list)
    _keep: list = field(default_factory=list)

    def __post_init__(self):
        self._build()

    # -----------------------------------------------------------------------------------
    def _build(self):
        case = self.case
        model = case.get("model", {})
        self.ndm = int(model.get("ndm", 2))
        self.ndf = int(model.get("ndf", 3))
        if (self.ndm, self.ndf) not in ((2, 3), (3, 6)):
            raise ModelError("this path implements frames with ndm=2, ndf=3 or ndm=3, ndf=6")
        nodes = case["nodes"]
        self.node_ids = [int(n["id"]) for n in nodes]
        self.node_index = {nid: i for i, nid in enumerate(self.node_ids)}
        nn = len(nodes)
        self.num_nodes = nn
        self.num_dofs = nn * self.ndf
        self.coords = np.zeros(self.ndm * nn)
        constrained = np.zeros(self.num_dofs, dtype=bool)
        for i, n in enumerate(nodes):
            self.coords[self.ndm * i] = float(n["x"])
            self.coords[self.ndm * i + 1] = float(n["y"])
            if self.ndm == 3:
                if "z" not in n:
                    raise ModelError("z is required when ndm=3")
                self.coords[self.ndm * i + 2] = float(n["z"])
            for d in n.get("constraints", []) or []:
                d = int(d)
                if d < 1 or d > self.ndf:
                    raise ModelError("constraint dof out of range")
                constrained[i * self.ndf + d - 1] = True
        mpcs = case.get("mp_constraints") or []

        # materials
        mats = case.get("materials", [])
        self.mat_index = {}
        mat_structs = []
        for m in mats:
            self.mat_index[int(m["id"])] = len(mat_structs)
            mat_structs.append(uniaxial_material(m))
        self.materials = mat_structs

        # sections
        self.section_index = {}
        fibers = []
        sections = []
        want = "FiberSection2d" if self.ndm == 2 else "FiberSection3d"
        self.plate_sections = {}
        for s in case.get("sections", []):
            if s["type"] == "ElasticMembranePlateSection" and self.ndm == 3:
                prm = s.get("params", {})
                E, nu, h = float(prm.get("E", 0.0)), float(prm.get("nu", 0.0)), float(prm.get("h", 0.0))
                if not (E > 0.0 and h > 0.0 and -1.0 < nu < 0.5):
                    raise ModelError("ElasticMembranePlateSection needs E > 0, h > 0, -1 < nu < 0.5")
                self.plate_sections[int(s["id"])] = (E, nu, h, float(prm.get("rho", 0.0)))
                continue
            if s["type"] != want:
                raise ModelError(f"unsupported section type for this path: {s['type']}")
            cells = discretize_section(s.get("params", {}))
            off = len(fibers)
            for (y, z, a, mid) in cells:
                if mid not in self.mat_index:
                    raise ModelError("FiberSection2d requires uniaxial material for all fibers")
                f = A.StrutFiber()
                f.y, f.z, f.area, f.material = y, z, a, self.mat_index[mid]
                fibers.append(f)
            sec = A.StrutFiberSection()
            sec.fiber_offset, sec.fiber_count = off, len(cells)
            sec.dim = self.ndm
            if self.ndm == 3:
                prm = s.get("params", {})
                sec.G = float(prm.get("G", 0.0))
                sec.J = float(prm.get("J", 0.0))
                if not (sec.G > 0.0 and sec.J > 0.0):
                    raise ModelError("FiberSection3d beam-column use requires positive params.G and params.J")
            self.section_index[int(s["id"])] = len(sections)
            sections.append(sec)
        self.fibers = fibers
        self.sections = sections

        # elements and integration rules
        rules = {}
        rule_structs = []
        elems = []
        self.elem_ids = []
        shells = []
        self.shell_ids = []
        for e in case.get("elements", []):
            et = e["type"]
            if et == "shell" and self.ndm == 3:
                # ShellMITC4 on an ElasticMembranePlateSection (elements/shell4.mojo:10-363)
                sid = int(e["section"])
                if sid not in self.plate_sections:
                    raise ModelError("shell requires an ElasticMembranePlateSection")
                nodes4 = [self.node_index[int(x)] for x in e["nodes"]]
                if len(nodes4) != 4:
                    raise ModelError("shell requires 4 nodes")
                sh = A.StrutShellElement()
                for k, ni in enumerate(nodes4):
                    sh.nodes[k] = ni
                    for a in range(6):
                        sh.dof[6 * k + a] = ni * 6 + a
                sh.E, sh.nu, sh.h = self.plate_sections[sid][:3]
                shells.append(sh)
                self.shell_ids.append(int(e["id"]))
                continue
            tags = {"forceBeamColumn2d": (A.ELEM_FORCE_BEAM_COLUMN_2D, 2),
                    "dispBeamColumn2d": (A.ELEM_DISP_BEAM_COLUMN_2D, 2),
                    "forceBeamColumn3d": (A.ELEM_FORCE_BEAM_COLUMN_3D, 3),
                    "dispBeamColumn3d": (A.ELEM_DISP_BEAM_COLUMN_3D, 3)}
            if et not in tags or tags[et][1] != self.ndm:
                raise ModelError(f"unsupported element type for this path: {et}")
            tag = tags[et][0]
            geom = e.get("geomTransf", "Linear")
            if geom == "Linear":
                g = A.GEOM_LINEAR
            elif geom == "PDelta":
                g = A.GEOM_PDELTA
            elif geom == "Corotational" and self.ndm == 3:
                g = A.GEOM_COROTATIONAL
            elif self.ndm == 3:
                raise ModelError(f"{et} supports geomTransf Linear, PDelta, or Corotational")
            else:
                raise ModelError(f"{et} supports geomTransf Linear | PDelta")
            integ = e.get("integration", "Lobatto")
            nip = int(e.get("num_int_pts", 3))
            if nip > A.MAX_INT_PTS:
                raise ModelError("num_int_pts above the supported maximum")
            key = (integ, nip)
            if key not in rules:
                xis, ws = beam_integration_rule(integ, nip)
                r = A.StrutBeamIntegration()
                r.num_int_pts = nip
                for i in range(nip):
                    r.xi[i] = xis[i]
                    r.w[i] = ws[i]
                rules[key] = len(rule_structs)
                rule_structs.append(r)
            sid = int(e["section"])
            if sid not in self.section_index:
                raise ModelError(f"{et} requires FiberSection2d")
            ni, nj = (self.node_index[int(x)] for x in e["nodes"])
            el = A.StrutFrameElement()
            el.type, el.node_i, el.node_j = tag, ni, nj
            el.section = self.section_index[sid]
            el.geom = g
            el.integration = rules[key]
            for a in range(self.ndf):
                el.dof[a] = ni * self.ndf + a
                el.dof[self.ndf + a] = nj * self.ndf + a
            if "vecxz" in e and e["vecxz"] is not None:
                vx = [float(x) for x in e["vecxz"]]
                el.vecxz[0], el.vecxz[1], el.vecxz[2] = vx
                el.has_vecxz = 1
            self.elem_ids.append(int(e["id"]))
            elems.append(el)
        self.elements = elems
        self.shells = shells
        self._shell_sections = [int(e["section"]) for e in case.get("elements", []) if e["type"] == "shell"]
        self.integrations = rule_structs
        self.elem_index = {eid: i for i, eid in enumerate(self.elem_ids)}

        # multi-point constraints, Transformation handler (loader.mojo:2239-2340)
        self.slaves = self._mp_constraints(mpcs, case, constrained)
        slave_set = set(self.slaves)
        # natural-order free numbering, slaves and fixed dofs skipped (loader.mojo:2439-2446)
        self.free_index = np.full(self.num_dofs, -1, dtype=np.int32)
        nf = 0
        for dof in range(self.num_dofs):
            if not constrained[dof] and dof not in slave_set:
                self.free_index[dof] = nf
                nf += 1
        if nf == 0:
            raise ModelError("no free dofs")
        self.num_free = nf

        # masses and loads
        self.mass = np.zeros(self.num_dofs)
        for m in case.get("masses", []) or []:
            d = int(m["dof"])
            if d < 1 or d > self.ndf:
                raise ModelError("mass dof out of range")
            self.mass[self.node_index[int(m["node"])] * self.ndf + d - 1] += float(m["value"])
        # shell mass: rho h area / 4 on each node's translations (loader.mojo:2060-2100)
        for sh, sid in zip(self.shells, self._shell_sections):
            rho = self.plate_sections[sid][3]
            if rho == 0.0:
                continue
            P = [self.coords[3 * sh.nodes[k]: 3 * sh.nodes[k] + 3] for k in range(4)]
            a = (P[1] - P[0]) + (P[2] - P[3])
            b = (P[3] - P[0]) + (P[2] - P[1])
            cr = np.cross(a, b)
            area = 0.25 * float(np.sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]))
            if area <= 0.0:
                raise ModelError("shell area must be > 0")
            lumped = rho * self.plate_sections[sid][2] * area / 4.0
            for d in range(3):
                for k in range(4):
                    self.mass[sh.nodes[k] * 6 + d] += lumped
        self.mass_rayleigh = self.mass.copy()
        self.f_const = np.zeros(self.num_dofs)
        for ld in case.get("loads", []) or []:
            d = int(ld["dof"])
            self.f_const[self.node_index[int(ld["node"])] * self.ndf + d - 1] += float(ld["value"])

        ray = case.get("rayleigh", {}) or {}
        self.alpha_m = float(ray.get("alphaM", 0.0))
        self.beta_k = float(ray.get("betaK", 0.0))
        self.beta_k_init = float(ray.get("betaKInit", 0.0))
        self.beta_k_comm = float(ray.get("betaKComm", 0.0))

        an = case.get("analysis", {})
        if an.get("type", "transient_nonlinear") != "transient_nonlinear":
            raise ModelError("this path runs transient_nonlinear analyses")
        self.dt = float(an.get("dt", 0.0))
        if self.dt <= 0.0:
            raise ModelError("transient_nonlinear requires dt > 0")
        self.steps = int(an.get("steps", 1))
        integ = an.get("integrator", {}) or {}
        if integ.get("type", "Newmark") != "Newmark":
            raise ModelError("transient_nonlinear only supports Newmark integrator")
        self.gamma = float(integ.get("gamma", 0.5))
        self.beta = float(integ.get("beta", 0.25))
        if self.beta <= 0.0:
            raise ModelError("Newmark beta must be > 0")
        amap = {"Newton": A.ALGORITHM_NEWTON, "ModifiedNewton": A.ALGORITHM_MODIFIED_NEWTON,
                "ModifiedNewtonInitial": A.ALGORITHM_MODIFIED_NEWTON_INITIAL}
        alg = an.get("algorithm", "Newton")
        if alg not in amap:
            raise ModelError(f"this path implements Newton, ModifiedNewton and ModifiedNewtonInitial, not {alg}")
        self.algorithm = amap[alg]
        tmap = {
            "MaxDispIncr": A.TEST_MAX_DISP_INCR,
            "NormDispIncr": A.TEST_NORM_DISP_INCR,
            "NormUnbalance": A.TEST_NORM_UNBALANCE,
            "EnergyIncr": A.TEST_ENERGY_INCR,
        }
        tt = an.get("test_type", "NormUnbalance")
        if tt not in tmap:
            raise ModelError(f"unsupported test_type: {tt}")
        self.test_type = tmap[tt]
        self.tol = float(an.get("tol", 1.0e-10))
        self.max_iters = int(an.get("max_iters", 20))
        # solver chain (transient_nonlinear.mojo:758-830): attempts tried in turn on a step that
        # does not converge; an absent chain is resolved by the library (Strut's rule)
        self.attempts = []
        for at in an.get("solver_chain", []) or []:
            a_alg = at.get("algorithm", "Newton")
            if a_alg not in amap:
                raise ModelError(f"solver_chain: this path implements Newton, ModifiedNewton and "
                                 f"ModifiedNewtonInitial, not {a_alg}")
            a_tt = at.get("test_type", tt)
            if a_tt not in tmap:
                raise ModelError(f"solver_chain: unsupported test_type {a_tt}")
            self.attempts.append((amap[a_alg], tmap[a_tt], int(at.get("max_iters", self.max_iters)),
                                  float(at.get("tol", self.tol))))
        if len(self.attempts) > A.MAX_ATTEMPTS:
            raise ModelError(f"solver_chain: at most {A.MAX_ATTEMPTS} attempts")
        system = an.get("system", an.get("solver", "")) or "BandGeneral"
        if system in ("BandGEN", "BandGen"):
            system = "BandGeneral"
        if system == "BandGeneral":
            self.system = A.SYSTEM_BAND_GENERAL
        elif system == "BandSPD":
            self.system = A.SYSTEM_BAND_SPD
        else:
            raise ModelError(f"this path implements BandGeneral and BandSPD, not {system}")

        # excitations: Path time series with dt
        ts_by_tag = {}
        for ts in case.get("time_series", []) or []:
            ts_by_tag[int(ts["tag"])] = ts
        self.excitations = []
        for p in _excitation_list(case):
            direction = int(p["direction"])
            if direction < 1 or direction > self.ndm:
                raise ModelError("UniformExcitation direction out of range")
            ts = ts_by_tag.get(int(p["accel"]))
            if ts is None:
                raise ModelError("UniformExcitation missing accel time_series")
            if ts.get("type") not in ("Path", "PathFile"):
                raise ModelError("UniformExcitation accel must be a Path time series")
            if "dt" not in ts:
                raise ModelError("Path time series on this path must give dt")
            vals = np.ascontiguousarray(ts["values"], dtype=np.float64)
            self.excitations.append(
                dict(
                    direction=direction,
                    values=vals,
                    dt=float(ts["dt"]),
                    factor=float(ts.get("factor", 1.0)),
                    start_time=float(ts.get("start_time", 0.0)),
                    use_last=bool(ts.get("use_last", False)),
                )
            )

        # recorders (transient_nonlinear.mojo:1550-1700): each needs displacement columns (full
        # dof indices) and element-force columns of the device history, shared between recorders
        rec_dofs, rec_elems = [], []
        dof_col, elem_col = {}, {}

        def dcol(dof):
            if dof not in dof_col:
                dof_col[dof] = len(rec_dofs)
                rec_dofs.append(dof)
            return dof_col[dof]

        def ecol(e):
            if e not in elem_col:
                elem_col[e] = len(rec_elems)
                rec_elems.append(e)
            return elem_col[e]

        def node_of(nid, what):
            if int(nid) not in self.node_index:
                raise ModelError(f"{what}: node {nid} not found")
            return self.node_index[int(nid)]

        def dof_of(d, what):
            d = int(d)
            if d < 1 or d > self.ndf:
                raise ModelError(f"{what}: dof {d} out of range 1..{self.ndf}")
            return d - 1

        sec_recs, sec_col = [], {}

        def scol(e, ip, kind):
            key = (e, ip, kind)
            if key not in sec_col:
                sec_col[key] = len(sec_recs)
                sec_recs.append(key)
            return sec_col[key]

        self.recorder_plan = []
        for r in case.get("recorders", []) or []:
            t = r["type"]
            out = str(r.get("output", t))
            if t in ("node_displacement", "envelope_node_displacement"):
                for nid in r["nodes"]:
                    ni = node_of(nid, t)
                    cols = [dcol(ni * self.ndf + dof_of(d, t)) for d in r["dofs"]]
                    self.recorder_plan.append({"type": t, "file": f"{out}_node{int(nid)}.out", "disp_cols": cols})
            elif t in ("element_force", "envelope_element_force"):
                for eid in r["elements"]:
                    if int(eid) not in self.elem_index:
                        raise ModelError(f"{t}: element {eid} not found")
                    c = ecol(self.elem_index[int(eid)])
                    self.recorder_plan.append({"type": t, "file": f"{out}_ele{int(eid)}.out", "elem_col": c})
            elif t == "drift":
                i_node, j_node = int(r["i_node"]), int(r["j_node"])
                ii, jj = node_of(i_node, t), node_of(j_node, t)
                d = dof_of(r["dof"], t)
                perp = int(r["perp_dirn"])
                if perp < 1 or perp > 3 or (perp == 3 and self.ndm < 3):
                    raise ModelError("drift perp_dirn must be in 1..ndm")
                dx = self.coords[self.ndm * jj + perp - 1] - self.coords[self.ndm * ii + perp - 1]
                if dx == 0.0:
                    raise ModelError("drift denominator is zero")
                self.recorder_plan.append({"type": t, "file": f"{out}_i{i_node}_j{j_node}.out",
                                           "i_col": dcol(ii * self.ndf + d), "j_col": dcol(jj * self.ndf + d),
                                           "dx": float(dx)})
            elif t in ("section_force", "section_deformation"):
                # one file per element and section (transient_nonlinear.mojo:1631-1655)
                kind = A.SECTION_FORCE if t == "section_force" else A.SECTION_DEFORMATION
                for eid in r["elements"]:
                    if int(eid) not in self.elem_index:
                        raise ModelError(f"{t}: element {eid} not found")
                    ei = self.elem_index[int(eid)]
                    el = self.elements[ei]
                    nip = int(self.integrations[el.integration].num_int_pts)
                    for sec_no in r["sections"]:
                        if int(sec_no) < 1 or int(sec_no) > nip:
                            raise ModelError("section recorder section index out of range")
                        if int(el.type) == A.ELEM_FORCE_BEAM_COLUMN_3D:
                            # Strut's recorder re-runs this element's state determination at
                            # the step's displacements (helpers.mojo:2223-2246): the element is
                            # recorded, whose record pass does exactly that
                            ecol(ei)
                        c = scol(ei, int(sec_no) - 1, kind)
                        self.recorder_plan.append({"type": t, "file": f"{out}_ele{int(eid)}_sec{int(sec_no)}.out",
                                                   "sec_col": c})
            else:
                raise ModelError(f"recorder type {t!r} is not on this path")
        self.record_dofs = np.asarray(rec_dofs, dtype=np.int32)
        self.record_elements = np.asarray(rec_elems, dtype=np.int32)
        self.record_sections = (A.StrutSectionRecord * max(len(sec_recs), 1))()
        for k, (e, ip, kind) in enumerate(sec_recs):
            self.record_sections[k] = A.StrutSectionRecord(e, ip, kind, 0)
        self.num_record_sections = len(sec_recs)

    def _mp_constraints(self, mpcs, case, constrained):
        """{slave dof: [(retained dof, coefficient), ...]} in constraint order."""
        if not mpcs:
            return {}
        an = case.get("analysis", {})
        handler = an.get("constraints", "Plain")
        if handler not in ("Transformation", "Lagrange"):
            raise ModelError("mp_constraints require analysis.constraints=Transformation or Lagrange")
        ndf = self.ndf
        slaves = {}
        mpc_constrained_nodes = set()
        for m in mpcs:
            cn = int(m["constrained_node"])
            if cn in self.node_index:
                mpc_constrained_nodes.add(self.node_index[cn])
        for m in mpcs:
            t = m.get("type")
            if t not in ("equalDOF", "rigidDiaphragm"):
                raise ModelError(f"unsupported mp constraint type: {t}")
            rn, cn = int(m["retained_node"]), int(m["constrained_node"])
            if rn not in self.node_index:
                raise ModelError(f"{t} retained_node not found")
            if cn not in self.node_index:
                raise ModelError(f"{t} constrained_node not found")
            ri, ci = self.node_index[rn], self.node_index[cn]
            if ri in mpc_constrained_nodes:
                raise ModelError(f"{t} retained_node cannot also be constrained")
            if t == "equalDOF":
                dofs = [int(d) for d in m.get("dofs", [])]
                if not dofs:
                    raise ModelError("equalDOF requires non-empty dofs")
                for d in dofs:
                    if d < 1 or d > ndf:
                        raise ModelError("equalDOF dof out of range")
                    sd = ci * ndf + d - 1
                    if sd in slaves:
                        raise ModelError("equalDOF constrained dof already controlled")
                    slaves[sd] = [(ri * ndf + d - 1, 1.0)]
            else:
                if not ((self.ndm == 3 and ndf == 6) or (self.ndm == 2 and ndf == 3)):
                    raise ModelError("rigidDiaphragm requires a 3D/6DOF or 2D/3DOF model")
                perp = int(m.get("perp_dirn", 0))
                if perp < 1 or perp > 3:
                    raise ModelError("rigidDiaphragm perp_dirn must be in 1..3")
                cdofs = [int(d) for d in m.get("constrained_dofs", [])]
                rdofs = [int(d) for d in m.get("retained_dofs", [])]
                mat = m.get("matrix", [])
                if not cdofs or not rdofs:
                    raise ModelError("rigidDiaphragm requires constrained_dofs and retained_dofs")
                if len(cdofs) > 3 or len(rdofs) > 3:
                    raise ModelError("rigidDiaphragm holds at most 3 constrained and 3 retained dofs")
                if len(mat) != len(cdofs):
                    raise ModelError("rigidDiaphragm matrix rows must match constrained_dofs")
                for row, cd in enumerate(cdofs):
                    if len(mat[row]) != len(rdofs):
                        raise ModelError("rigidDiaphragm matrix columns must match retained_dofs")
                    if cd < 1 or cd > ndf:
                        raise ModelError("rigidDiaphragm dof out of range")
                    sd = ci * ndf + cd - 1
                    if sd in slaves:
                        raise ModelError("rigidDiaphragm constrained dof already controlled")
                    terms = []
                    for col, rd in enumerate(rdofs):
                        if rd < 1 or rd > ndf:
                            raise ModelError("rigidDiaphragm dof out of range")
                        terms.append((ri * ndf + rd - 1, float(mat[row][col])))
                    slaves[sd] = terms
                    constrained[sd] = True
        for sd, terms in slaves.items():
            for md, _c in terms:
                if md in slaves:
                    raise ModelError("a retained dof cannot itself be constrained")
        return slaves

    # -----------------------------------------------------------------------------------
    def desc(self) -> A.StrutModelDesc:
        """The C struct; the Model keeps every buffer it points to alive."""
        d = A.StrutModelDesc()
        keep = []

        def dptr(arr):
            arr = np.ascontiguousarray(arr, dtype=np.float64)
            keep.append(arr)
            return arr.ctypes.data_as(C.POINTER(C.c_double))

        def iptr(arr):
            arr = np.ascontiguousarray(arr, dtype=np.int32)
            keep.append(arr)
            return arr.ctypes.data_as(C.POINTER(C.c_int32))

        d.ndm, d.ndf = self.ndm, self.ndf
        d.num_nodes, d.num_dofs = self.num_nodes, self.num_dofs
        d.node_coords = dptr(self.coords)
        mats = _struct_array(A.StrutUniMaterial, self.materials)
        fibs = _struct_array(A.StrutFiber, self.fibers)
        secs = _struct_array(A.StrutFiberSection, self.sections)
        rules = _struct_array(A.StrutBeamIntegration, self.integrations)
        elems = _struct_array(A.StrutFrameElement, self.elements)
        keep += [mats, fibs, secs, rules, elems]
        d.num_materials, d.materials = len(self.materials), mats
        d.num_fibers, d.fibers = len(self.fibers), fibs
        d.num_sections, d.sections = len(self.sections), secs
        d.num_integrations, d.integrations = len(self.integrations), rules
        d.num_elements, d.elements = len(self.elements), elems
        d.num_free = self.num_free
        d.free_index = iptr(self.free_index)
        d.mass = dptr(self.mass)
        d.mass_rayleigh = dptr(self.mass_rayleigh)
        d.f_const = dptr(self.f_const)
        d.alpha_m, d.beta_k = self.alpha_m, self.beta_k
        d.beta_k_init, d.beta_k_comm = self.beta_k_init, self.beta_k_comm
        d.dt, d.gamma, d.beta = self.dt, self.gamma, self.beta
        d.tol, d.max_iters = self.tol, self.max_iters
        d.test_type, d.system = self.test_type, self.system
        d.algorithm = self.algorithm
        d.num_attempts = len(self.attempts)
        for k, (a_alg, a_tt, a_mi, a_tol) in enumerate(self.attempts):
            d.attempts[k].algorithm, d.attempts[k].test_type = a_alg, a_tt
            d.attempts[k].max_iters, d.attempts[k].tol = a_mi, a_tol
        d.num_excitations = len(self.excitations)
        for i, x in enumerate(self.excitations):
            ex = d.excitation[i]
            ex.direction = x["direction"]
            ex.count = len(x["values"])
            ex.values = dptr(x["values"])
            ex.dt, ex.factor, ex.start_time = x["dt"], x["factor"], x["start_time"]
            ex.use_last = 1 if x["use_last"] else 0
        d.num_record_dofs = len(self.record_dofs)
        d.record_dofs = iptr(self.record_dofs)
        d.num_record_elements = len(self.record_elements)
        d.record_elements = iptr(self.record_elements)
        d.num_record_sections = self.num_record_sections
        d.record_sections = C.cast(self.record_sections, C.POINTER(A.StrutSectionRecord))
        sl = sorted(self.slaves)
        d.num_slaves = len(sl)
        ptr, mdof, coef = [0], [], []
        for sd in sl:
            for md, c in self.slaves[sd]:
                mdof.append(md)
                coef.append(c)
            ptr.append(len(mdof))
        d.slave_dof = iptr(np.asarray(sl, dtype=np.int32))
        d.slave_ptr = iptr(np.asarray(ptr, dtype=np.int32))
        d.slave_master = iptr(np.asarray(mdof, dtype=np.int32))
        d.slave_coef = dptr(np.asarray(coef, dtype=np.float64))
        d.num_shells = len(self.shells)
        if self.shells:
            sh = _struct_array(A.StrutShellElement, self.shells)
            keep.append(sh)
            d.shells = C.cast(sh, C.POINTER(A.StrutShellElement))
        self._keep = keep
        return d

    # convenience -----------------------------------------------------------------------
    @property
    def num_fibers_total(self) -> int:
        """Fiber-state slots of the whole model (sections x integration points)."""
        tot = 0
        for el in self.elements:
            nip = self.integrations[el.integration].num_int_pts
            tot += nip * self.sections[el.section].fiber_count
        return tot

    def free_dofs_of_records(self):
        return [int(self.free_index[d]) for d in self.record_dofs]


def material_struct(mat: dict) -> A.StrutUniMaterial:
    return uniaxial_material(mat)


def section_fibers(case_section: dict, materials: list):
    """(StrutUniMaterial array, StrutFiber array) for one FiberSection2d section-path case."""
    idx = {int(m["id"]): i for i, m in enumerate(materials)}
    mats = [uniaxial_material(m) for m in materials]
    cells = discretize_section(case_section.get("params", {}))
    fibs = []
    for (y, z, a, mid) in cells:
        f = A.StrutFiber()
        f.y, f.z, f.area, f.material = y, z, a, idx[mid]
        fibs.append(f)
    return _struct_array(A.StrutUniMaterial, mats), len(mats), _struct_array(A.StrutFiber, fibs), len(fibs)


def math_isclose(a, b, rel_tol, abs_tol):  # small helper shared by tests
    return math.isclose(a, b, rel_tol=rel_tol, abs_tol=abs_tol)
