"""Section force / deformation recorders (transient_nonlinear.mojo:1631-1655, 3537-3605): the
recorder plan (files `<output>_ele<id>_sec<n>.out`, one column per element, section and kind),
and the oracle's values checked against the element formulations they come from:

* forceBeamColumn2d: the section forces are the basic forces interpolated, so N is the same at
  every point and Mz is linear in the point's position xi;
* dispBeamColumn2d: eps0 is constant along the element and kappa linear in xi (cubic Hermite
  displacement field);
* a section index outside the element's points is rejected as Strut rejects it."""
import numpy as np
import pytest

from strut_b200 import model as M
from strut_b200 import recorders as R
from strut_b200 import workloads as W

STEPS = 60


def section_case(element):
    case = W.rc_frame_case(stories=2, bays=2, steps=STEPS, seed=31, pga_g=0.5, element=element)
    case["recorders"] = [
        {"type": "section_force", "elements": [1], "sections": [1, 2, 3, 4, 5], "output": "sf"},
        {"type": "section_deformation", "elements": [1], "sections": [1, 2, 3, 4, 5], "output": "sd"},
        {"type": "node_displacement", "nodes": [case["nodes"][-1]["id"]], "dofs": [1], "output": "d"},
    ]
    return case


def point_xi(model, record):
    """Positions xi of the recorded element's integration points."""
    el = model.elements[model.record_sections[record].element]
    r = model.integrations[el.integration]
    return np.array([r.xi[k] for k in range(int(r.num_int_pts))])


def test_plan_files_and_columns():
    m = M.Model(section_case("forceBeamColumn2d"))
    files = [r["file"] for r in m.recorder_plan if r["type"].startswith("section_")]
    assert files == [f"sf_ele1_sec{k}.out" for k in range(1, 6)] + [f"sd_ele1_sec{k}.out" for k in range(1, 6)]
    assert m.num_record_sections == 10
    bad = section_case("forceBeamColumn2d")
    bad["recorders"][0]["sections"] = [6]
    with pytest.raises(M.ModelError):
        M.Model(bad)


def _linear_fit_residual(x, y):
    A = np.stack([np.ones_like(x), x], axis=1)
    coef, *_ = np.linalg.lstsq(A, y, rcond=None)
    return float(np.max(np.abs(A @ coef - y)))


def test_force_based_sections_follow_the_basic_forces(oracle):
    m = M.Model(section_case("forceBeamColumn2d"))
    *_, rc, failed, sec = oracle.run_transient(m, STEPS, sections=True)
    assert rc == 0
    force = sec[:, :5, :]  # steps x point x (N, Mz)
    assert np.max(np.abs(force[:, :, 0])) > 0.0
    # N equal at every point, Mz = (xi - 1) q1 + xi q2 linear in the point's position
    scale = np.max(np.abs(force))
    xs = point_xi(m, 0)
    for s in range(STEPS):
        assert np.max(np.abs(force[s, :, 0] - force[s, 0, 0])) <= 1e-9 * scale
        assert _linear_fit_residual(xs, force[s, :, 1]) <= 1e-9 * scale


def test_displacement_based_sections_follow_the_hermite_field(oracle):
    m = M.Model(section_case("dispBeamColumn2d"))
    *_, rc, failed, sec = oracle.run_transient(m, STEPS, sections=True)
    assert rc == 0
    defo = sec[:, 5:, :]  # steps x point x (eps0, kappa)
    xs = point_xi(m, 5)
    scale = np.max(np.abs(defo), axis=(0, 1))
    assert np.all(scale > 0.0)
    for s in range(STEPS):
        assert np.max(np.abs(defo[s, :, 0] - defo[s, 0, 0])) <= 1e-9 * scale[0]
        assert _linear_fit_residual(xs, defo[s, :, 1]) <= 1e-9 * scale[1]


def test_files_from_oracle_history(oracle, tmp_path):
    m = M.Model(section_case("dispBeamColumn2d"))
    d, e, it, rc, failed, sec = oracle.run_transient(m, STEPS, sections=True)
    paths = R.write_outputs(m, d, e, tmp_path, sections=sec)
    names = sorted(p.name for p in paths)
    assert "sf_ele1_sec1.out" in names and "sd_ele1_sec5.out" in names
    rows = (tmp_path / "sf_ele1_sec3.out").read_text().splitlines()
    assert len(rows) == STEPS
    vals = np.array([[float(v) for v in r.split()] for r in rows])
    np.testing.assert_array_equal(vals, sec[:, 2, :])
