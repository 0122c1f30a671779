"""Frames of the batched slab-frame set (3D RC frames with rigid diaphragms and 2 x 2 ShellMITC4
slabs per bay, two horizontal records) on the GPU against the oracle.  Their bands live in global
memory; the 5 x 5 and 6 x 6-bay floors (half bands 368 and 515) take the wide factorisation
variant (16-column panels, 640 threads), the 4 x 4-bay floor (251) the standard one.  The
oracle's BandGeneral restarts densely on every one of these systems (its pivot test fails), which
the partial-pivot band LU reproduces.  Histories within 1e-7 of peak, identical iteration
counts; a batch of the three in one handle gives each its own run's histories bit for bit."""
import numpy as np
import pytest

from strut_b200 import model as M
from strut_b200 import workloads as W
from tests.test_gpu_records import compare_histories

pytestmark = pytest.mark.gpu

SIZES = [(3, 5, 368), (3, 6, 515), (4, 4, 251)]


def _case(stories, bays, steps):
    c = W.slab_frame3d_case(stories, bays, steps=steps, seed=8100 + stories + bays)
    c["recorders"][0]["nodes"] = [n["id"] for n in c["nodes"][-5:]]
    return c


@pytest.mark.parametrize("stories,bays,bw", SIZES)
def test_slab_frame_against_the_oracle(gpu_lib, oracle, stories, bays, bw):
    steps = 6
    m = M.Model(_case(stories, bays, steps))
    with gpu_lib.Analysis([m]) as an:
        assert an.band_info(0)[0] == bw
        st = an.run(steps)
        gd, ge, gi = an.history(0)
    assert st.steps_done == steps
    rd, re, ri, rc, failed = oracle.run_transient(m, steps)
    assert rc == 0, f"oracle failed at step {failed}"
    worst_d, worst_e, n_diff = compare_histories(gd, ge, gi, rd, re, ri)
    assert worst_d <= 1e-7 and worst_e <= 1e-7, (worst_d, worst_e)
    assert n_diff == 0


def test_uneven_slab_frames_in_one_handle(gpu_lib):
    steps = 4
    models = [M.Model(_case(s, b, steps)) for s, b, _bw in SIZES]
    alone = []
    for m in models:
        with gpu_lib.Analysis([m]) as an:
            an.run(steps)
            alone.append(an.history(0))
    with gpu_lib.Analysis(models) as an:
        an.run(steps)
        for i, (d, e, it) in enumerate(alone):
            d2, e2, it2 = an.history(i)
            assert np.array_equal(it, it2) and np.array_equal(d, d2) and np.array_equal(e, e2)
