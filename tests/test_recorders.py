"""Strut's transient recorder files (transient_nonlinear.mojo:1550-1700, 3225-3500;
helpers.mojo:2581-2588, 3113-3200) written from a recorded history: names, rows, drift and
envelopes, on an oracle history."""
import numpy as np
import pytest

from strut_b200 import model as M
from strut_b200 import recorders as R
from strut_b200 import workloads as W


def recorder_case(steps=30, element="forceBeamColumn2d"):
    case = W.rc_frame_case(stories=3, bays=2, steps=steps, seed=77, pga_g=0.4, element=element)
    col0 = sorted((n for n in case["nodes"] if n["x"] == 0.0), key=lambda n: n["y"])
    base, first, roof = col0[0]["id"], col0[1]["id"], col0[-1]["id"]
    case["recorders"] = [
        {"type": "node_displacement", "nodes": [roof, first], "dofs": [1, 3], "output": "disp"},
        {"type": "element_force", "elements": [1, 2], "output": "force"},
        {"type": "drift", "i_node": base, "j_node": first, "dof": 1, "perp_dirn": 2, "output": "drift1"},
        {"type": "drift", "i_node": first, "j_node": roof, "dof": 1, "perp_dirn": 2, "output": "drift_top"},
        {"type": "envelope_element_force", "elements": [1], "output": "env"},
        {"type": "envelope_node_displacement", "nodes": [roof], "dofs": [1, 2], "output": "envd"},
        {"type": "element_force", "elements": [2], "output": "force"},  # shares force_ele2.out
    ]
    return case, (base, first, roof)


def test_plan_names_and_columns():
    case, (base, first, roof) = recorder_case()
    m = M.Model(case)
    names = [r["file"] for r in m.recorder_plan]
    assert names[:2] == [f"disp_node{roof}.out", f"disp_node{first}.out"]
    assert f"drift1_i{base}_j{first}.out" in names and "env_ele1.out" in names
    # shared columns: element 2 and the roof dofs appear once in the device history
    assert len(m.record_elements) == len(set(m.record_elements.tolist())) == 2
    assert len(m.record_dofs) == len(set(m.record_dofs.tolist()))


def test_files_from_oracle_history(oracle, tmp_path):
    case, (base, first, roof) = recorder_case()
    m = M.Model(case)
    steps = 30
    d, e, _it, rc, _f = oracle.run_transient(m, steps)
    assert rc == 0
    paths = R.write_outputs(m, d, e, tmp_path)
    files = {p.name: p for p in paths}
    ndf = m.ndf
    col = {int(x): j for j, x in enumerate(m.record_dofs)}
    ni = {nid: m.node_index[nid] for nid in (base, first, roof)}
    # node displacement rows: one per step, the requested dofs in order
    rows = R.read_rows(files[f"disp_node{roof}.out"])
    assert rows.shape == (steps, 2)
    assert np.array_equal(rows[:, 0], d[:, col[ni[roof] * ndf]])
    assert np.array_equal(rows[:, 1], d[:, col[ni[roof] * ndf + 2]])
    # element force: 2 ndf global end forces per step; the shared file holds both recorders' rows
    rows = R.read_rows(files["force_ele1.out"])
    assert rows.shape == (steps, 2 * ndf) and np.array_equal(rows, e[:, 0, :])
    rows = R.read_rows(files["force_ele2.out"])
    assert rows.shape == (2 * steps, 2 * ndf)
    assert np.array_equal(rows[0::2], e[:, 1, :]) and np.array_equal(rows[1::2], e[:, 1, :])
    # drift: (u_j - u_i) / (y_j - y_i)
    dy = m.coords[2 * ni[first] + 1] - m.coords[2 * ni[base] + 1]
    rows = R.read_rows(files[f"drift1_i{base}_j{first}.out"])
    ref = (d[:, col[ni[first] * ndf]] - d[:, col[ni[base] * ndf]]) / dy
    assert rows.shape == (steps, 1) and np.array_equal(rows[:, 0], ref)
    # envelopes: minima, maxima, absolute maxima over the steps
    rows = R.read_rows(files["env_ele1.out"])
    assert rows.shape == (3, 2 * ndf)
    assert np.array_equal(rows[0], e[:, 0, :].min(0)) and np.array_equal(rows[1], e[:, 0, :].max(0))
    assert np.array_equal(rows[2], np.abs(e[:, 0, :]).max(0))
    rows = R.read_rows(files[f"envd_node{roof}.out"])
    assert np.array_equal(rows[2], np.abs(d[:, [col[ni[roof] * ndf], col[ni[roof] * ndf + 1]]]).max(0))


def test_values_round_trip():
    vals = [0.0, -1.6666666666666667e-05, 1e300, 3.141592653589793, -0.1]
    line = R.format_values_line(vals)
    assert line.endswith("\n") and [float(x) for x in line.split()] == vals


def test_bad_recorders_are_rejected():
    case, (base, first, roof) = recorder_case()
    case["recorders"] = [{"type": "drift", "i_node": base, "j_node": first, "dof": 1, "perp_dirn": 1,
                          "output": "x"}]
    with pytest.raises(M.ModelError):
        M.Model(case)  # both nodes at x = 0: zero denominator
    case["recorders"] = [{"type": "node_displacement", "nodes": [roof], "dofs": [4], "output": "x"}]
    with pytest.raises(M.ModelError):
        M.Model(case)
