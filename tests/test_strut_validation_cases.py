"""Strut's own fiber beam-column validation models, given a transient analysis block
(tests/golden/make_strut_validation_cases.py), load through the JSON model builder and run on the
CPU oracle; the GPU comparison is tests/test_gpu_strut_cases.py."""
import json
from pathlib import Path

import pytest

from strut_b200 import model as M

CASES = json.loads((Path(__file__).resolve().parent / "golden" / "strut_validation_cases.json").read_text())


@pytest.mark.parametrize("name", sorted(CASES))
def test_loads_and_runs_on_the_oracle(oracle, name):
    m = M.Model(CASES[name])
    assert m.num_free > 0 and len(m.record_dofs) > 0
    _d, _e, it, rc, failed = oracle.run_transient(m, 50)
    assert rc == 0, f"failed at step {failed}"
    assert it.min() >= 1
