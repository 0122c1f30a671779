"""Strut's own fiber beam-column validation models (tests/validation/*_fiber_cantilever of the
reference project) through this library's JSON loader and the C ABI, GPU against the oracle.
tests/golden/make_strut_validation_cases.py gave each a transient analysis block (mass, damping,
a seeded ground motion along its point load's direction, Newton at NormDispIncr 1e-8); every
displacement, element-force and (3D files) section force / deformation history within 1e-7 of
peak, Newton iteration counts identical."""
import json
from pathlib import Path

import numpy as np
import pytest

from strut_b200 import model as M
from tests.test_gpu_records import compare_histories

pytestmark = pytest.mark.gpu

CASES = json.loads((Path(__file__).resolve().parent / "golden" / "strut_validation_cases.json").read_text())


@pytest.mark.parametrize("name", sorted(CASES))
def test_strut_validation_model(gpu_lib, oracle, name):
    m = M.Model(CASES[name])
    with gpu_lib.Analysis([m]) as an:
        st = an.run(m.steps)
        gd, ge, gi = an.history(0)
        gs = an.section_history(0)
    assert st.steps_done == m.steps
    rd, re, ri, rc, failed, rs = oracle.run_transient(m, m.steps, sections=True)
    assert rc == 0, f"oracle failed at step {failed}"
    worst_d, worst_e, n_diff = compare_histories(gd, ge, gi, rd, re, ri)
    assert worst_d <= 1e-7 and worst_e <= 1e-7, (worst_d, worst_e)
    assert n_diff == 0
    assert np.max(np.abs(rd)) > 0.0
    if m.num_record_sections:
        # forces and deformations apart, each history's peak floored at 1e-6 of the largest of
        # its kind (the cantilevers' axial components hold rounding noise only)
        kinds = np.array([m.record_sections[k].kind for k in range(m.num_record_sections)])
        for kind in (0, 1):
            sel = kinds == kind
            if sel.any():
                worst_s, _, _ = compare_histories(gs[:, sel], ge, gi, rs[:, sel], re, ri)
                assert worst_s <= 1e-7, (kind, worst_s)
