"""Recorder files written from the device history agree with those written from the oracle's
(within 1e-7 of each file's peak, as the histories)."""
import numpy as np
import pytest

from strut_b200 import model as M
from strut_b200 import recorders as R
from tests.test_recorders import recorder_case

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("element", ["forceBeamColumn2d", "dispBeamColumn2d"])
def test_recorder_files_gpu_vs_oracle(gpu_lib, oracle, element):
    case, _ = recorder_case(steps=60, element=element)
    m = M.Model(case)
    with gpu_lib.Analysis([m]) as an:
        an.run(60)
        gd, ge, _gi = an.history(0)
    rd, re, _ri, rc, _f = oracle.run_transient(m, 60)
    assert rc == 0
    got = R.recorder_outputs(m, gd, ge)
    ref = R.recorder_outputs(m, rd, re)
    assert list(got) == list(ref)
    for name in ref:
        a = np.array([[float(x) for x in ln.split()] for ln in got[name].splitlines()])
        b = np.array([[float(x) for x in ln.split()] for ln in ref[name].splitlines()])
        assert a.shape == b.shape, name
        assert np.max(np.abs(a - b)) <= 1e-7 * max(np.max(np.abs(b)), 1e-30), name
