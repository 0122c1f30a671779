"""ModifiedNewton and ModifiedNewtonInitial on the GPU against the oracle running the same
variant: histories within 1e-7 of peak, Newton iteration counts equal on >= 99% of steps; the
variants agree with Newton on an elastic frame; one factorisation per step."""
import numpy as np
import pytest

from strut_b200 import _abi as A
from strut_b200 import model as M
from strut_b200 import workloads as W
from tests.helpers import rel_err_of_peak
from tests.test_oracle_newton_variants import elastic_frame, rc_frame

pytestmark = pytest.mark.gpu


def _parity(gpu_lib, oracle, cases, steps):
    models = [M.Model(c) for c in cases]
    with gpu_lib.Analysis(models) as an:
        st = an.run(steps)
        got = [an.history(i) for i in range(len(models))]
    for m, (gd, ge, gi) in zip(models, got):
        rd, re, ri, rc, failed = oracle.run_transient(m, steps)
        assert rc == 0, f"oracle failed at step {failed}"
        for j in range(rd.shape[1]):
            if np.max(np.abs(rd[:, j])) > 1e-9:
                assert rel_err_of_peak(gd[:, j], rd[:, j]) <= 1e-7, f"disp {j}"
        peak = np.max(np.abs(re))
        assert np.max(np.abs(ge - re)) <= 1e-7 * peak
        assert np.mean(gi == ri) >= 0.99
    return st, got


@pytest.mark.parametrize("algorithm", ["ModifiedNewton", "ModifiedNewtonInitial"])
def test_variant_parity(gpu_lib, oracle, algorithm):
    steps = 150
    st, got = _parity(gpu_lib, oracle, [rc_frame(steps, algorithm)], steps)
    assert st.factorizations == steps  # one per step
    assert st.global_newton_iterations > steps


def test_mixed_algorithms_in_one_batch(gpu_lib, oracle):
    steps = 100
    cases = [rc_frame(steps, "Newton"), rc_frame(steps, "ModifiedNewton"),
             W.rc_frame_case(stories=4, bays=3, steps=steps, seed=32, pga_g=0.25, max_iters=40)]
    cases[2]["analysis"]["algorithm"] = "ModifiedNewtonInitial"
    _parity(gpu_lib, oracle, cases, steps)


@pytest.mark.parametrize("algorithm", ["ModifiedNewton", "ModifiedNewtonInitial"])
def test_variants_match_newton_on_elastic_frame(gpu_lib, algorithm):
    steps = 60
    out = {}
    for alg in ("Newton", algorithm):
        with gpu_lib.Analysis([M.Model(elastic_frame(steps, alg))]) as an:
            an.run(steps)
            out[alg] = an.history(0)
    np.testing.assert_allclose(out[algorithm][0], out["Newton"][0], rtol=1e-12, atol=1e-12)
    peak = np.abs(out["Newton"][1]).max()
    np.testing.assert_allclose(out[algorithm][1], out["Newton"][1], rtol=1e-12, atol=1e-12 * peak)


def test_modified_newton_on_a_wide_band_is_unsupported(gpu_lib):
    case = W.rc_frame3d_case(stories=3, bays_x=3, bays_y=2, steps=5, element="forceBeamColumn3d",
                             seed=41, pga_g=0.4)
    case["analysis"]["algorithm"] = "ModifiedNewton"
    with pytest.raises(gpu_lib.StrutError) as ei:
        gpu_lib.Analysis([M.Model(case)])
    assert ei.value.code == A.STRUT_UNSUPPORTED


@pytest.mark.parametrize("algorithm", ["ModifiedNewton", "ModifiedNewtonInitial"])
def test_variant_on_3d_diaphragm_frame_with_slabs(gpu_lib, oracle, algorithm):
    """The variants through the 3D element kernel, the multi-point-constraint collapse and the
    slab shells' constant stiffness at once."""
    steps = 60
    case = W.rc_frame3d_case(stories=2, bays_x=2, bays_y=2, steps=steps, element="forceBeamColumn3d",
                             beam_element="dispBeamColumn3d", seed=71, pga_g=0.3, bidirectional=True,
                             diaphragm=True, record_elements=(1,), max_iters=40,
                             slabs={"E": 30.0e9, "nu": 0.2, "h": 0.2, "rho": 0.0})
    case["analysis"]["algorithm"] = algorithm
    st, _ = _parity(gpu_lib, oracle, [case], steps)
    assert st.factorizations == steps
