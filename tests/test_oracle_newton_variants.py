"""Newton variants on the oracle (transient_nonlinear.mojo:650-668, 2072-2085, 2236-2268,
2302-2335, 2421-2440): ModifiedNewton freezes the first iteration's tangent and the Rayleigh C
built from it for the step and factors once; ModifiedNewtonInitial does the same with K_init.

Known answer, after the reference's own check that Newton variants agree on an elastic case
(tests/unit/test_force_beam_column2d.py:160-205, abs and rel 1e-12): with elastic fibers the
tangent never changes, so all three give the same histories."""
import numpy as np
import pytest

from strut_b200 import model as M
from strut_b200 import workloads as W


def elastic_frame(steps, algorithm):
    case = W.rc_frame_case(stories=3, bays=2, steps=steps, seed=31, pga_g=0.3)
    for k, mat in enumerate(case["materials"]):
        E = 200.0e9 if mat["type"] in ("Steel02", "Steel01") else 30.0e9
        case["materials"][k] = {"id": mat["id"], "type": "Elastic", "params": {"E": E}}
    case["analysis"]["algorithm"] = algorithm
    return case


def rc_frame(steps, algorithm):
    case = W.rc_frame_case(stories=3, bays=2, steps=steps, seed=31, pga_g=0.3, max_iters=40)
    case["analysis"]["algorithm"] = algorithm
    return case


@pytest.mark.parametrize("algorithm", ["ModifiedNewton", "ModifiedNewtonInitial"])
def test_variants_match_newton_on_elastic_frame(oracle, algorithm):
    steps = 60
    ref_case, case = elastic_frame(steps, "Newton"), elastic_frame(steps, algorithm)
    rd, re, ri, rrc, _ = oracle.run_transient(M.Model(ref_case), steps)
    gd, ge, gi, grc, _ = oracle.run_transient(M.Model(case), steps)
    assert rrc == 0 and grc == 0
    np.testing.assert_allclose(gd, rd, rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(ge, re, rtol=1e-12, atol=1e-12 * np.abs(re).max())


@pytest.mark.parametrize("algorithm", ["ModifiedNewton", "ModifiedNewtonInitial"])
def test_variants_converge_to_the_same_response(oracle, algorithm):
    """On the RC frame the variants take more iterations (linear convergence) and stop within
    the same NormDispIncr tolerance of the same trajectory."""
    steps = 150
    rd, _re, ri, rrc, _ = oracle.run_transient(M.Model(rc_frame(steps, "Newton")), steps)
    gd, _ge, gi, grc, _ = oracle.run_transient(M.Model(rc_frame(steps, algorithm)), steps)
    assert rrc == 0 and grc == 0
    assert gi.mean() > ri.mean()
    assert np.max(np.abs(gd - rd)) <= 1e-6 * np.max(np.abs(rd))


def test_unknown_algorithm_is_rejected():
    case = rc_frame(10, "KrylovNewton")
    with pytest.raises(M.ModelError):
        M.Model(case)
