"""Attempt fan-out of forceBeamColumn2d (StrutTuning.fan_out) against the sequential order.

A forceBeamColumn2d element tries an increment with three schemes at up to four subdivision
levels, each attempt from the accepted state (force_beam_column2d.mojo:1669-1763).  With
fan_out the twelve attempts of every pass of an element whose last state determination needed
a subdivision run on twelve CTAs (later passes through the launch's attempt queue) and the
first success in Strut's order is kept.  Frames 0, 21 and 37 of the
256-frame batch subdivide in their first 400 steps (the oracle counts 116, 153 and 121
cut-back passes there), so their histories exercise the fan-out; they must be bit for bit those
of the sequential order, with every element CTA size, and within 1e-7 of peak of the oracle's
under one of its roundings: frame 0 bifurcates at rounding level near step 300 (the oracle with
separately rounded and with contracted multiply-adds differ there by 1.3 % of peak, while its
SIMD widths 8 and 1 agree to 3e-9), and the GPU, which contracts, follows the contracted
oracle."""
import numpy as np
import pytest

from strut_b200 import model as M
from strut_b200 import workloads as W
from tests.test_gpu_records import nearest_order, record_everything

pytestmark = pytest.mark.gpu

FRAMES = (0, 21, 37)
STEPS = 400


def _cases():
    params = W.batched_frame_params(256, base_seed=1000)
    return [record_everything(W.rc_frame_case(stories=params[i]["stories"], bays=params[i]["bays"],
                                              wg=params[i]["wg"], pga_g=params[i]["pga_g"],
                                              seed=params[i]["seed"], steps=STEPS)) for i in FRAMES]


def _run(gpu_lib, models, **tuning):
    with gpu_lib.Analysis(models) as an:
        an.set_tuning(**tuning)
        t = an.tuning()
        for k, v in tuning.items():
            assert getattr(t, k) == v
        st = an.run(STEPS)
        return st, [an.history(i) for i in range(len(models))]


def test_fan_out_is_the_sequential_order_bit_for_bit(gpu_lib, oracle):
    models = [M.Model(c) for c in _cases()]
    st_seq, seq = _run(gpu_lib, models, fan_out=0)
    assert st_seq.fanned_out == 0
    for tuning in ({"fan_out": 1}, {"fan_out": 1, "element_threads": 320}, {"fan_out": 1, "element_threads": 224},
                   {"fan_out": 1, "element_threads": 160}, {"fan_out": 0, "element_threads": 160}):
        st_fan, fan = _run(gpu_lib, models, **tuning)
        assert (st_fan.fanned_out > 0) == (tuning["fan_out"] == 1)
        assert st_fan.global_newton_iterations == st_seq.global_newton_iterations
        assert st_fan.local_element_iterations == st_seq.local_element_iterations
        assert st_fan.section_evaluations == st_seq.section_evaluations
        for (d0, e0, i0), (d1, e1, i1) in zip(seq, fan):
            assert np.array_equal(i0, i1)
            assert np.array_equal(d0, d1)
            assert np.array_equal(e0, e1)
    for m, (gd, ge, gi) in zip(models, fan):
        worst_d, worst_e, n_diff, order = nearest_order(oracle, m, STEPS, gd, ge, gi, widths=(8,))[0]
        assert worst_d <= 1e-7 and worst_e <= 1e-7, (worst_d, worst_e, order)
        assert n_diff <= 0.01 * STEPS
