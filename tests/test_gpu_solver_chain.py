"""The solver chain on the GPU (transient_nonlinear.mojo:1925-1942): a chain [Newton with one
iteration, Newton with 20] restores each failed step to its start, so the GPU's displacement and
element-force histories equal the plain Newton run's on the GPU bit for bit, with the retried
steps' counts one higher; and both match the oracle's (1e-7 of peak, identical counts).  A batch
mixes instances with and without a chain; ModifiedNewton gets Strut's automatic Newton fallback
as in the oracle."""
import copy

import numpy as np
import pytest

from strut_b200 import model as M
from strut_b200 import workloads as W
from tests.test_gpu_records import compare_histories
from tests.test_oracle_solver_chain import _chain_case

pytestmark = pytest.mark.gpu


def test_chain_on_the_gpu(gpu_lib, oracle):
    steps = 150
    plain, chain = _chain_case(steps)
    models = [M.Model(plain), M.Model(chain)]
    with gpu_lib.Analysis(models) as an:
        an.run(steps)
        (d0, e0, i0), (d1, e1, i1) = an.history(0), an.history(1)
    assert np.array_equal(d0, d1) and np.array_equal(e0, e1)
    retried = i1 != i0
    assert retried.sum() > steps // 2 and np.all(i1[retried] == i0[retried] + 1)
    rd, re, ri, rc, _f = oracle.run_transient(models[1], steps)
    assert rc == 0
    worst_d, worst_e, n_diff = compare_histories(d1, e1, i1, rd, re, ri)
    assert worst_d <= 1e-7 and worst_e <= 1e-7 and n_diff == 0


def test_modified_newton_fallback_on_the_gpu(gpu_lib, oracle):
    steps = 120
    case = W.rc_frame_case(stories=3, bays=2, steps=steps, seed=34, pga_g=0.5)
    case["analysis"]["algorithm"] = "ModifiedNewton"
    case["analysis"]["max_iters"] = 3
    m = M.Model(case)
    with gpu_lib.Analysis([m]) as an:
        st = an.run(steps)
        gd, ge, gi = an.history(0)
    assert st.steps_done == steps
    rd, re, ri, rc, _f = oracle.run_transient(m, steps)
    assert rc == 0
    worst_d, worst_e, n_diff = compare_histories(gd, ge, gi, rd, re, ri)
    assert worst_d <= 1e-7 and worst_e <= 1e-7 and n_diff == 0
    assert gi.max() > 3
