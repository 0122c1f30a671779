"""Section force / deformation recorders on the GPU against the oracle: the recorded points of a
forceBeamColumn2d and of a dispBeamColumn2d frame (the basic-state and the displacement-field
forms), every value within 1e-7 of its history's peak (peaks floored at 1e-6 of the recorder's
largest of its kind, as for the other histories)."""
import numpy as np
import pytest

from strut_b200 import model as M
from tests.test_section_recorders import STEPS, section_case

pytestmark = pytest.mark.gpu


def worst_of_peak(g, r):
    g2 = g.reshape(g.shape[0], -1)
    r2 = r.reshape(r.shape[0], -1)
    peaks = np.max(np.abs(r2), axis=0)
    floor = 1e-6 * float(peaks.max())
    return float(np.max(np.max(np.abs(g2 - r2), axis=0) / np.maximum(peaks, floor)))


@pytest.mark.parametrize("element", ["forceBeamColumn2d", "dispBeamColumn2d"])
def test_section_histories_match_the_oracle(gpu_lib, oracle, element):
    m = M.Model(section_case(element))
    with gpu_lib.Analysis([m]) as an:
        st = an.run(STEPS)
        gs = an.section_history(0)
        _gd, _ge, gi = an.history(0)
    assert st.steps_done == STEPS
    _d, _e, ri, rc, failed, rs = oracle.run_transient(m, STEPS, sections=True)
    assert rc == 0
    assert gs.shape == rs.shape
    assert np.max(np.abs(rs)) > 0.0
    kinds = np.array([m.record_sections[k].kind for k in range(m.num_record_sections)])
    for kind in (0, 1):  # forces and deformations apart: each its own scale
        assert worst_of_peak(gs[:, kinds == kind], rs[:, kinds == kind]) <= 1e-7, kind
    assert np.array_equal(gi, ri)
