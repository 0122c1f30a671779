"""Failure detection on the GPU without a GPU fault: the cooperative wide-band factorisation's
grid barrier waits a bounded number of polls (strut_gpu_set_wait_limit).  With the limit at 0 a
waiting CTA gives up at once, every CTA of the launch returns, and the run reports
STRUT_CUDA_ERROR for the instance; the device stays usable, and a new handle on it runs the
same model to the oracle's answer."""
import numpy as np
import pytest

from strut_b200 import _abi as A
from strut_b200 import model as M
from strut_b200 import workloads as W
from tests.helpers import rel_err_of_peak

pytestmark = pytest.mark.gpu


def _wide_band_case(steps):
    return W.rc_frame3d_case(stories=5, bays_x=3, bays_y=3, steps=steps, element="forceBeamColumn3d",
                             beam_element="dispBeamColumn3d", diaphragm=True, seed=13, pga_g=0.35)


def test_barrier_gives_up_and_the_device_stays_usable(gpu_lib, oracle):
    steps = 6
    m = M.Model(_wide_band_case(steps))
    with gpu_lib.Analysis([m]) as an:
        _bw, rw = an.band_info(0)
        assert m.num_free * rw * 8 > 220 * 1024  # the cooperative global-memory path
        an.set_tuning(factor_ctas=4)
        assert an.tuning().factor_ctas == 4
        assert gpu_lib.lib().strut_gpu_set_wait_limit(an.h, 0) == A.STRUT_OK
        st = an.run(steps, check=False)
        assert st.status == A.STRUT_CUDA_ERROR
        assert an.instance_status()[0] == A.STRUT_CUDA_ERROR
        assert st.steps_done < steps
    # a new handle on the same device: normal run, checked against the oracle
    with gpu_lib.Analysis([m]) as an:
        st = an.run(steps)
        gd, _ge, gi = an.history(0)
    rd, _re, ri, rc, _f = oracle.run_transient(m, steps)
    assert rc == 0 and st.status == A.STRUT_OK
    for j in range(rd.shape[1]):
        if np.max(np.abs(rd[:, j])) > 1e-9:
            assert rel_err_of_peak(gd[:, j], rd[:, j]) <= 1e-7
    assert np.array_equal(gi, ri)
