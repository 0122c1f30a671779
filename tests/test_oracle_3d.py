"""The 3D part of the CPU oracle: FiberSection3d, dispBeamColumn3d, forceBeamColumn3d.

* the reference's own 3D section tests (tests/unit/test_fiber_section.py:475-632), with their
  tolerances;
* a nonlinear FiberSection3d bent about z only equals the FiberSection2d of the same fibers;
* element invariants: for an elastic section the force-based and displacement-based 3D
  elements give the same (exact) tangent, which is symmetric and has the rigid-body modes in
  its null space; for the RC section each element's tangent matches central differences of
  its own resisting force;
* a plane frame written as a 3D model reproduces the 2D oracle's transient history
  (displacements within 1e-10 of peak, identical Newton iteration counts).
"""
import math

import numpy as np
import pytest

from strut_b200 import model as M
from strut_b200 import workloads as W
from tests.helpers import lcg_strains, planar_frame_3d, single_element_3d


def _section3d(case):
    mats, nm, fibs, nf = M.section_fibers(case["section"], case["materials"])
    return mats, nm, fibs, nf


def _run3d(oracle, case, path):
    mats, nm, fibs, nf = _section3d(case)
    return oracle.section3d_path(mats, nm, fibs, nf, path)


def _expected_elastic_3d(case, eps0, ky, kz):
    # tests/unit/test_fiber_section.py:426-473
    e_by_mat = {m["id"]: m["params"]["E"] for m in case["materials"] if m["type"] == "Elastic"}
    fibers = M.discretize_section(case["section"]["params"])
    a_sum = sum(a for y, z, a, m in fibers)
    y_bar = sum(a * y for y, z, a, m in fibers) / a_sum
    z_bar = sum(a * z for y, z, a, m in fibers) / a_sum
    out = np.zeros(9)
    for y, z, area, mat in fibers:
        e = e_by_mat[mat]
        yr, zr = y - y_bar, z - z_bar
        fs = e * (eps0 + zr * ky - yr * kz) * area
        ks = e * area
        out += [fs, fs * zr, -fs * yr, ks, ks * zr, -ks * yr, ks * zr * zr, -ks * zr * yr,
                ks * yr * yr]
    return out


def test_section3d_rect_patch_elastic_aggregation(oracle):
    # tests/unit/test_fiber_section.py:475-512
    case = {"materials": [{"id": 1, "type": "Elastic", "params": {"E": 2.8e10}}],
            "section": {"id": 1, "type": "FiberSection3d", "params": {"patches": [
                {"type": "rect", "material": 1, "num_subdiv_y": 6, "num_subdiv_z": 5,
                 "y_i": -0.3, "z_i": -0.2, "y_j": 0.3, "z_j": 0.2}], "layers": []}}}
    got = _run3d(oracle, case, [[1.2e-4, -7.5e-4, 2.5e-3]])[0]
    exp = _expected_elastic_3d(case, 1.2e-4, -7.5e-4, 2.5e-3)
    for i in (0, 1, 2, 3, 6, 8):
        assert math.isclose(got[i], exp[i], rel_tol=1e-10, abs_tol=1e-10)
    for i in (4, 5, 7):
        assert math.isclose(got[i], exp[i], rel_tol=1e-8, abs_tol=1e-6)
    # the uniform-modulus elastic family reports k12 = k13 = 0 exactly (fiber3d.mojo:243-253)
    assert got[4] == 0.0 and got[5] == 0.0


def test_section3d_inline_fibers_elastic_aggregation(oracle):
    # tests/unit/test_fiber_section.py:515-558
    case = {"materials": [{"id": 1, "type": "Elastic", "params": {"E": 2.8e10}},
                          {"id": 2, "type": "Elastic", "params": {"E": 2.0e11}}],
            "section": {"id": 2, "type": "FiberSection3d", "params": {
                "patches": [], "layers": [], "fibers": [
                    {"y": -0.3, "z": -0.15, "area": 0.012, "material": 1},
                    {"y": -0.1, "z": 0.12, "area": 0.01, "material": 1},
                    {"y": 0.2, "z": -0.08, "area": 0.009, "material": 2},
                    {"y": 0.35, "z": 0.18, "area": 0.011, "material": 2}]}}}
    got = _run3d(oracle, case, [[9.0e-5, -6.5e-4, 1.8e-3]])[0]
    exp = _expected_elastic_3d(case, 9.0e-5, -6.5e-4, 1.8e-3)
    for i in range(9):
        assert math.isclose(got[i], exp[i], rel_tol=1e-10, abs_tol=1e-10)


def test_section3d_tangent_matches_finite_difference(oracle):
    # tests/unit/test_fiber_section.py:563-632
    case = {"materials": [{"id": 1, "type": "Elastic", "params": {"E": 3.0e10}},
                          {"id": 2, "type": "Elastic", "params": {"E": 2.2e11}}],
            "section": {"id": 7, "type": "FiberSection3d", "params": {
                "patches": [{"type": "quadr", "material": 1, "num_subdiv_y": 4, "num_subdiv_z": 3,
                             "y_i": -0.35, "z_i": -0.2, "y_j": -0.3, "z_j": 0.22,
                             "y_k": 0.28, "z_k": 0.18, "y_l": 0.33, "z_l": -0.25}],
                "layers": [{"type": "straight", "material": 2, "num_bars": 3, "bar_area": 0.0004,
                            "y_start": -0.25, "z_start": 0.16, "y_end": 0.1, "z_end": 0.2}]}}}
    e0, ky, kz, d = 8.0e-5, -1.2e-3, 1.7e-3, 1.0e-7
    base = _run3d(oracle, case, [[e0, ky, kz]])[0]
    pe = _run3d(oracle, case, [[e0 + d, ky, kz]])[0]
    py = _run3d(oracle, case, [[e0, ky + d, kz]])[0]
    pz = _run3d(oracle, case, [[e0, ky, kz + d]])[0]
    fd = {}
    for name, p in (("e", pe), ("y", py), ("z", pz)):
        fd[name] = (p[:3] - base[:3]) / d
    k = {"11": base[3], "12": base[4], "13": base[5], "22": base[6], "23": base[7], "33": base[8]}
    pairs = [("11", fd["e"][0]), ("12", fd["y"][0]), ("13", fd["z"][0]),
             ("12", fd["e"][1]), ("22", fd["y"][1]), ("23", fd["z"][1]),
             ("13", fd["e"][2]), ("23", fd["y"][2]), ("33", fd["z"][2])]
    for key, val in pairs:
        assert math.isclose(k[key], val, rel_tol=1e-5, abs_tol=1e-2)


def test_section3d_bending_about_z_equals_section2d(oracle):
    """Nonlinear RC fibers: (eps0, 0, kz) on the 3D section gives the 2D section's N, M and
    tangent along a cyclic path (sums in different orders: rel 1e-12)."""
    sec2 = W.rc_section(1, 0.4, 0.6)
    mats = [{"id": 1, "type": "Concrete02", "params": dict(W.CORE)},
            {"id": 2, "type": "Concrete02", "params": dict(W.COVER)},
            {"id": 3, "type": "Steel02", "params": dict(W.STEEL)}]
    m2, n2, f2, nf2 = M.section_fibers(sec2, mats)
    sec3 = W.rc_section(1, 0.4, 0.6, three_d=True)
    m3, n3, f3, nf3 = M.section_fibers(sec3, mats)
    kappa = lcg_strains(7, 300, 4.0e-3, "cyclic") * 0.01
    eps0 = lcg_strains(8, 300, 1.0e-4, "walk") - 2.0e-4
    r2 = oracle.section_path(m2, n2, f2, nf2, np.stack([eps0, kappa], 1))
    r3 = oracle.section3d_path(m3, n3, f3, nf3, np.stack([eps0, np.zeros_like(eps0), kappa], 1))
    pairs = [(r2[:, 0], r3[:, 0]), (r2[:, 1], r3[:, 2]), (r2[:, 2], r3[:, 3]),
             (r2[:, 3], r3[:, 5]), (r2[:, 4], r3[:, 8])]
    for a, b in pairs:
        assert np.max(np.abs(a - b)) <= 1e-12 * np.max(np.abs(a))


@pytest.mark.parametrize("geom", ["Linear", "PDelta", "Corotational"])
def test_elastic_force_and_disp_3d_agree(oracle, geom):
    rng = np.random.default_rng(0)
    u = rng.normal(0.0, 1e-4, 12)
    mf = M.Model(single_element_3d("forceBeamColumn3d", geom, nonlinear=False))
    md = M.Model(single_element_3d("dispBeamColumn3d", geom, nonlinear=False))
    kf, ff = oracle.element_state(mf, 0, u)
    kd, fd = oracle.element_state(md, 0, u)
    scale = np.abs(kf).max()
    assert np.abs(kf - kd).max() <= 1e-12 * scale
    assert np.abs(ff - fd).max() <= 1e-12 * np.abs(ff).max()
    assert np.abs(kf - kf.T).max() <= 1e-13 * scale
    if geom == "Linear":
        assert np.abs(kf @ u - ff).max() <= 1e-12 * np.abs(ff).max()
        # rigid translation and rigid rotation about the element's first node
        ur = np.zeros(12)
        ur[[0, 6]], ur[[1, 7]], ur[[2, 8]] = 1e-3, -2e-3, 5e-4
        assert np.abs(oracle.element_state(mf, 0, ur)[1]).max() <= 1e-12 * np.abs(ff).max()
        w = np.array([1e-4, -2e-4, 3e-4])
        xj = np.array([3.0, 1.0, 2.0])
        ur = np.zeros(12)
        ur[3:6] = w
        ur[6:9] = np.cross(w, xj)
        ur[9:12] = w
        assert np.abs(kf @ ur).max() <= 1e-9 * scale * 1e-4


@pytest.mark.parametrize("etype", ["forceBeamColumn3d", "dispBeamColumn3d"])
def test_nonlinear_3d_tangent_matches_central_differences(oracle, etype):
    m = M.Model(single_element_3d(etype, "Linear", nonlinear=True, vecxz=(0.3, 0.4, -1.0)))
    u = np.random.default_rng(1).normal(0.0, 2e-4, 12)
    k, _f = oracle.element_state(m, 0, u)
    h = 1e-9
    kfd = np.zeros((12, 12))
    for j in range(12):
        up, um = u.copy(), u.copy()
        up[j] += h
        um[j] -= h
        kfd[:, j] = (oracle.element_state(m, 0, up)[1] - oracle.element_state(m, 0, um)[1]) / (2 * h)
    assert np.abs(k - kfd).max() <= 1e-8 * np.abs(k).max()


@pytest.mark.parametrize("element", ["forceBeamColumn2d", "dispBeamColumn2d"])
def test_plane_frame_as_3d_model_matches_2d(oracle, element):
    steps = 150
    c2 = W.rc_frame_case(stories=2, bays=2, steps=steps, element=element, seed=11, pga_g=0.4)
    c3 = planar_frame_3d(c2)
    d2, _e2, i2, rc2, _ = oracle.run_transient(M.Model(c2), steps)
    d3, _e3, i3, rc3, _ = oracle.run_transient(M.Model(c3), steps)
    assert rc2 == 0 and rc3 == 0
    assert np.array_equal(i2, i3)
    for j, sgn in enumerate((1.0, 1.0, -1.0)):
        assert np.abs(d2[:, j] - sgn * d3[:, j]).max() <= 1e-10 * np.abs(d2[:, j]).max()


def test_frame3d_bidirectional_runs(oracle):
    case = W.rc_frame3d_case(stories=2, bays_x=1, bays_y=1, steps=60, bidirectional=True,
                             seed=3)
    d, e, it, rc, failed = oracle.run_transient(M.Model(case), 60)
    assert rc == 0, failed
    assert e.shape == (60, 1, 12)
    # both horizontal directions respond
    assert np.abs(d[:, 0]).max() > 1e-4 and np.abs(d[:, 1]).max() > 1e-4
