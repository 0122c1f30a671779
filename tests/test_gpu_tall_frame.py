"""The 20-story 6x6-bay rigid-diaphragm frame (the large single instance: 3000 free dofs, half
band 155, the band factored in global memory) on its 4000-step record until it gives out,
against the oracle's histories in both rounding orders (tests/golden/make_tall_frame_golden.py):
identical Newton iteration counts and displacement / element-force histories within 1e-7 of peak
over the first 200 steps, and the same stop (an element state determination that fails,
STRUT_ELEMENT_FAILED) within a step of where the oracle stops: from step 200 on, the orders
themselves disagree on the step."""
import json
from pathlib import Path

import numpy as np
import pytest

from strut_b200 import _abi as A
from strut_b200 import model as M
from strut_b200 import workloads as W

pytestmark = pytest.mark.gpu

GOLD = json.loads((Path(__file__).resolve().parent / "golden" / "tall_frame3d_4000_first215.json").read_text())
AGREE = 200  # steps over which both rounding orders agree with each other


def _worst(a, b):
    """max |a - b| over the largest |b| of each column (floored at 1e-6 of the largest)."""
    peak = np.max(np.abs(b), axis=0)
    peak = np.maximum(peak, 1e-6 * np.max(peak))
    return float(np.max(np.abs(a - b) / peak))


def test_tall_frame3d_until_it_stops(gpu_lib):
    m = M.Model(W.tall_frame3d_case(steps=GOLD["record_steps"]))
    with gpu_lib.Analysis([m]) as an:
        st = an.run(GOLD["steps"], check=False)
        gd, ge, gi = an.history(0)
        assert an.band_info(0)[0] > 100  # the global-memory band path
    assert st.status == A.STRUT_ELEMENT_FAILED
    gpu_stop = st.failed_step + 1  # 1-based step of the failure
    ge = ge.reshape(ge.shape[0], -1)
    stops = []
    for order, r in GOLD["orders"].items():
        rd, re, ri = np.array(r["disp"]), np.array(r["eforce"]), np.array(r["iters"])
        assert r["status"] == A.STRUT_ELEMENT_FAILED, order
        stops.append(r["failed_step"] + 1)
        n = AGREE
        assert np.array_equal(gi[:n], ri[:n]), (order, np.nonzero(gi[:n] != ri[:n])[0][:5])
        assert _worst(gd[:n], rd[:n]) <= 1e-7, order
        assert _worst(ge[:n], re[:n]) <= 1e-7, order
    assert min(abs(gpu_stop - s) for s in stops) <= 1, (gpu_stop, stops)
