"""The CPU oracle against the known-answer tests of the reference's own test-suite.

Each test restates a reference test (tests/unit/*.py of the Strut project) with the oracle in
place of the Mojo binary; expectations and tolerances are the reference test's.
"""
import math

import numpy as np
import pytest

from strut_b200 import _abi as A
from strut_b200 import model as M
from strut_b200 import workloads as W
from tests.helpers import ALTERNATING, GROUPED, lcg_strains, mixed_section_case, path_array


def _expected_elastic(case, eps0, kappa):
    # tests/unit/test_fiber_section.py:161-187
    e_by_mat = {m["id"]: m["params"]["E"] for m in case["materials"] if m["type"] == "Elastic"}
    fibers = M.discretize_section(case["section"]["params"])
    a_sum = sum(a for y, z, a, m in fibers)
    y_bar = sum(a * y for y, z, a, m in fibers) / a_sum
    n = mz = k11 = k12 = k22 = 0.0
    for y, z, area, mat in fibers:
        e = e_by_mat[mat]
        y_rel = y - y_bar
        stress = e * (eps0 - y_rel * kappa)
        fs = stress * area
        ks = e * area
        n += fs
        mz += -fs * y_rel
        k11 += ks
        k12 += -ks * y_rel
        k22 += ks * y_rel * y_rel
    return [n, mz, k11, k12, k22]


def _section_path(oracle, case):
    mats, nm, fibs, nf = M.section_fibers(case["section"], case["materials"])
    return oracle.section_path(mats, nm, fibs, nf, path_array(case))


def test_rect_patch_elastic_aggregation(oracle):
    # tests/unit/test_fiber_section.py:189-223
    case = {
        "materials": [{"id": 1, "type": "Elastic", "params": {"E": 30000000000.0}}],
        "section": {"id": 1, "type": "FiberSection2d", "params": {"patches": [
            {"type": "rect", "material": 1, "num_subdiv_y": 6, "num_subdiv_z": 4,
             "y_i": -0.3, "z_i": -0.2, "y_j": 0.3, "z_j": 0.2}], "layers": []}},
        "deformation_path": [{"eps0": 1.2e-4, "kappa": 2.5e-3}],
    }
    got = _section_path(oracle, case)[0]
    exp = _expected_elastic(case, 1.2e-4, 2.5e-3)
    for i in (0, 1, 2, 4):
        assert math.isclose(got[i], exp[i], rel_tol=1e-10, abs_tol=1e-10)
    assert math.isclose(got[3], exp[3], rel_tol=1e-8, abs_tol=1e-6)


def test_straight_layer_single_bar_midpoint(oracle):
    # tests/unit/test_fiber_section.py:226-257
    case = {
        "materials": [{"id": 1, "type": "Elastic", "params": {"E": 200000000000.0}}],
        "section": {"id": 1, "type": "FiberSection2d", "params": {"patches": [], "layers": [
            {"type": "straight", "material": 1, "num_bars": 1, "bar_area": 0.0005,
             "y_start": -0.1, "z_start": 0.0, "y_end": 0.3, "z_end": 0.0}]}},
        "deformation_path": [{"eps0": 0.0, "kappa": 0.02}],
    }
    got = _section_path(oracle, case)[0]
    assert abs(got[0]) <= 1e-12 and abs(got[1]) <= 1e-12
    assert got[2] > 0.0
    assert abs(got[3]) <= 1e-12 and abs(got[4]) <= 1e-12


def test_quadr_patch_elastic_aggregation(oracle):
    # tests/unit/test_fiber_section.py:260-300
    case = {
        "materials": [{"id": 1, "type": "Elastic", "params": {"E": 3.0e10}}],
        "section": {"id": 2, "type": "FiberSection2d", "params": {"patches": [
            {"type": "quadr", "material": 1, "num_subdiv_y": 4, "num_subdiv_z": 3,
             "y_i": -0.4, "z_i": 0.2, "y_j": -0.2, "z_j": -0.2, "y_k": 0.4, "z_k": -0.1,
             "y_l": 0.2, "z_l": 0.3}], "layers": []}},
        "deformation_path": [{"eps0": 8.0e-5, "kappa": -1.5e-3}],
    }
    got = _section_path(oracle, case)[0]
    exp = _expected_elastic(case, 8.0e-5, -1.5e-3)
    for i in range(5):
        assert math.isclose(got[i], exp[i], rel_tol=1e-10, abs_tol=1e-10)


def test_mixed_material_order_is_response_invariant(oracle):
    # tests/unit/test_fiber_section.py:364-387
    a = _section_path(oracle, mixed_section_case(ALTERNATING))
    g = _section_path(oracle, mixed_section_case(GROUPED))
    assert a.shape == g.shape == (5, 5)
    np.testing.assert_allclose(a, g, rtol=1e-10, atol=1e-8)


@pytest.mark.parametrize("width", [1, 4, 8])
def test_simd_width_changes_only_rounding(oracle, width):
    """Strut's section sums depend on the host SIMD width (chunked reduction); every width
    gives the same response to rounding."""
    case = mixed_section_case(ALTERNATING)
    oracle.set_simd_width(8)
    ref = _section_path(oracle, case)
    oracle.set_simd_width(width)
    try:
        got = _section_path(oracle, case)
    finally:
        oracle.set_simd_width(8)
    np.testing.assert_allclose(got, ref, rtol=1e-13, atol=1e-9)


MATS = [
    {"id": 1, "type": "Steel02", "params": dict(W.STEEL)},
    {"id": 2, "type": "Concrete02", "params": dict(W.CORE)},
    {"id": 3, "type": "Concrete02", "params": dict(W.COVER)},
    {"id": 4, "type": "Steel01", "params": {"Fy": 350.0e6, "E0": 200.0e9, "b": 0.01}},
    {"id": 5, "type": "Elastic", "params": {"E": 30.0e9}},
    {"id": 6, "type": "Steel02", "params": {"Fy": 420.0, "E0": 200000.0, "b": 0.012, "R0": 18.0,
                                             "cR1": 0.925, "cR2": 0.15, "a1": 0.01, "a2": 1.0,
                                             "a3": 0.01, "a4": 1.0, "sigInit": 50.0}},
    {"id": 7, "type": "Concrete01", "params": {"fpc": -30.0e6, "epsc0": -0.002, "fpcu": -6.0e6,
                                                "epscu": -0.006}},
]


@pytest.mark.parametrize("mat", MATS, ids=[m["type"] + str(m["id"]) for m in MATS])
@pytest.mark.parametrize("kind", ["walk", "cyclic"])
def test_scalar_path_matches_fiber_runtime(oracle, mat, kind):
    """material_compare_micro (src/mojo/material_compare_micro.mojo:740-753, 845-940): the scalar
    uniaxial path and the fiber runtime agree on LCG strain scenarios within atol 1e-10 +
    rtol 1e-9 * scale.  The fiber runtime is driven through a one-fiber section."""
    scale = 0.004 if mat["type"] != "Steel02" or mat["id"] != 6 else 0.004
    strains = lcg_strains(mat["id"] * 7 + (1 if kind == "walk" else 2), 400, scale, kind)
    m = M.uniaxial_material(mat)
    scalar = oracle.material_path(m, strains)
    sec = {"id": 1, "type": "FiberSection2d", "params": {"patches": [], "layers": [], "fibers": [
        {"y": 0.0, "z": 0.0, "area": 1.0, "material": mat["id"]}]}}
    mats, nm, fibs, nf = M.section_fibers(sec, [mat])
    ek = np.stack([strains, np.zeros_like(strains)], axis=1)
    fiber = oracle.section_path(mats, nm, fibs, nf, ek)
    stress_scale = max(1.0, float(np.max(np.abs(scalar[:, 0]))))
    # Steel02 with sigInit: the scalar path shifts the strain it compares against, the section
    # path adds sigInit / E0 as well; both report the same stress.
    np.testing.assert_allclose(fiber[:, 0], scalar[:, 0], rtol=1e-9, atol=1e-10 * stress_scale)


def test_steel02_known_points(oracle):
    """Elastic branch returns E0, monotonic loading approaches the hardening slope b*E0 and the
    stress stays below Fy*(1+b*mu) (Menegotto-Pinto envelope)."""
    m = M.uniaxial_material({"id": 1, "type": "Steel02", "params": dict(W.STEEL)})
    Fy, E0, b = W.STEEL["Fy"], W.STEEL["E0"], W.STEEL["b"]
    eps_y = Fy / E0
    strains = np.linspace(0.0, 20 * eps_y, 401)[1:]
    out = oracle.material_path(m, strains)
    assert math.isclose(out[0, 1], E0, rel_tol=1e-3)
    assert math.isclose(out[-1, 1], b * E0, rel_tol=0.05)
    assert np.all(out[:, 0] <= Fy * (1.0 + b * strains / eps_y) + 1e-6)
    # unloading from the plateau is elastic again
    back = oracle.material_path(m, np.concatenate([strains, [strains[-1] - 0.1 * eps_y]]))
    assert math.isclose(back[-1, 1], E0, rel_tol=0.05)


def test_concrete02_known_points(oracle):
    """Compression envelope: peak fc at epsc0 with zero tangent, linear softening to fcu at
    epscu; tension: linear to ft then softening with -Ets (concrete02.mojo:3-31)."""
    p = W.CORE
    m = M.uniaxial_material({"id": 1, "type": "Concrete02", "params": dict(p)})
    out = oracle.material_path(m, [p["epsc0"]])
    assert math.isclose(out[0, 0], p["fpc"], rel_tol=1e-12)
    assert abs(out[0, 1]) < 1e-3
    out = oracle.material_path(m, [p["epsc0"], p["epscu"]])
    assert math.isclose(out[1, 0], p["fpcu"], rel_tol=1e-12)
    Ec0 = 2 * p["fpc"] / p["epsc0"]
    eps_t = p["ft"] / Ec0
    out = oracle.material_path(m, [0.5 * eps_t, 1.5 * eps_t])
    assert math.isclose(out[0, 0], 0.5 * p["ft"], rel_tol=1e-12)
    assert math.isclose(out[1, 1], -p["Ets"], rel_tol=1e-12)


def _cantilever_case(E=30.0e9, element="forceBeamColumn2d", nip=3, L=4.0):
    return {
        "model": {"ndm": 2, "ndf": 3},
        "nodes": [{"id": 1, "x": 0.0, "y": 0.0, "constraints": [1, 2, 3]}, {"id": 2, "x": L, "y": 0.0}],
        "materials": [{"id": 1, "type": "Elastic", "params": {"E": E}}],
        "sections": [{"id": 1, "type": "FiberSection2d", "params": {"patches": [
            {"type": "rect", "material": 1, "num_subdiv_y": 16, "num_subdiv_z": 2,
             "y_i": -0.25, "z_i": -0.15, "y_j": 0.25, "z_j": 0.15}], "layers": []}}],
        "elements": [{"id": 1, "type": element, "nodes": [1, 2], "section": 1, "geomTransf": "Linear",
                      "integration": "Lobatto", "num_int_pts": nip}],
        "masses": [{"node": 2, "dof": 1, "value": 1.0}, {"node": 2, "dof": 2, "value": 1.0}],
        "analysis": {"type": "transient_nonlinear", "dt": 0.01, "steps": 1},
    }


@pytest.mark.parametrize("element", ["forceBeamColumn2d", "dispBeamColumn2d"])
def test_cantilever_tip_stiffness_and_equilibrium(oracle, element):
    """test_force_beam_column2d.py:516-537 restated on the state determination: end forces are
    in equilibrium and the tip stiffness of an elastic fiber cantilever is 3EI/L^3 (exact for
    both elements at 3 Lobatto points with a uniform section)."""
    E, L = 30.0e9, 4.0
    m = M.Model(_cantilever_case(E=E, element=element, L=L))
    u = np.zeros(m.num_free)
    u[1] = 1.0e-3  # tip transverse displacement
    f, band, bw = oracle.state_determination(m, u)
    # second moment of the discretised fibers (16 layers: bh^3/12 * (1 - 1/16^2))
    cells = M.discretize_section(_cantilever_case()["sections"][0]["params"])
    I = sum(a * y * y for y, z, a, mat in cells)
    k_tip = 3.0 * E * I / L ** 3
    # equilibrium of the element forces: the free tip dofs carry the element's node-2 forces
    Kff = np.zeros((m.num_free, m.num_free))
    for i in range(m.num_free):
        for o in range(band.shape[1]):
            j = i + o - bw
            if 0 <= j < m.num_free:
                Kff[i, j] = band[i, o]
    # remove the a0*M term added on the diagonal of the effective band
    a0 = 1.0 / (0.25 * 0.01 * 0.01)
    Kff[0, 0] -= a0
    Kff[1, 1] -= a0
    # condensed tip translational stiffness (rotation free)
    kc = Kff[1, 1] - Kff[1, 2] * Kff[2, 1] / Kff[2, 2]
    assert math.isclose(kc, k_tip, rel_tol=1e-7)
    np.testing.assert_allclose(Kff @ u, f, rtol=1e-9, atol=1e-6)


def test_transient_small_frame_runs_and_is_deterministic(oracle):
    case = W.rc_frame_case(stories=2, bays=1, steps=120, seed=7, pga_g=0.5)
    m = M.Model(case)
    d1, e1, it1, rc1, fs1 = oracle.run_transient(m, 120)
    d2, e2, it2, rc2, fs2 = oracle.run_transient(m, 120)
    assert rc1 == 0 and fs1 == -1
    assert np.array_equal(d1, d2) and np.array_equal(e1, e2) and np.array_equal(it1, it2)
    assert 1 <= it1.min() and it1.max() <= case["analysis"]["max_iters"]
    assert np.max(np.abs(d1[:, 0])) > 1e-4


def test_nonconvergence_is_reported_not_aborted(oracle):
    """Strut aborts when Newton fails (transient_nonlinear.mojo:2849); the oracle returns
    STRUT_NONCONVERGED with the failing step instead."""
    case = W.rc_frame_case(stories=2, bays=1, steps=20, seed=3, pga_g=0.5, tol=1e-30, max_iters=2)
    m = M.Model(case)
    _d, _e, it, rc, failed = oracle.run_transient(m, 20)
    assert rc == A.STRUT_NONCONVERGED
    assert failed == 0
    assert it[0] == 2


def test_concrete01_known_points(oracle):
    """Kent-Scott-Park envelope (concrete01.mojo:3-20): parabola to fpc at epsc0 (zero tangent),
    linear to fpcu at epscu, constant beyond; no tension; unloading towards the end strain."""
    m = M.uniaxial_material({"id": 1, "type": "Concrete01",
                             "params": {"fpc": -30.0e6, "epsc0": -0.002, "fpcu": -6.0e6,
                                        "epscu": -0.006}})
    out = oracle.material_path(m, [-0.001])
    assert math.isclose(out[0, 0], -30.0e6 * (2 * 0.5 - 0.25), rel_tol=1e-12)
    out = oracle.material_path(m, [-0.002, -0.004, -0.008])
    # at epsc0 itself the softening branch applies (strain > epsc0 is false)
    assert math.isclose(out[0, 0], -30.0e6, rel_tol=1e-12)
    assert math.isclose(out[0, 1], -24.0e6 / 0.004, rel_tol=1e-12)
    assert math.isclose(out[1, 0], -30.0e6 + (-24.0e6 / 0.004) * (-0.004 + 0.002), rel_tol=1e-12)
    assert out[2, 0] == -6.0e6 and out[2, 1] == 0.0
    out = oracle.material_path(m, [0.001])
    assert out[0, 0] == 0.0 and out[0, 1] == 0.0
    # unloading from -0.003 is linear with the unloading slope and stays non-positive
    out = oracle.material_path(m, [-0.003, -0.0025, 0.0])
    assert out[1, 0] > out[0, 0] and out[1, 0] <= 0.0 and out[1, 1] > 0.0
    assert out[2, 0] == 0.0
