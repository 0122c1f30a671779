"""The solver chain of the transient step (transient_nonlinear.mojo:758-830, 1925-1942) in the
oracle.  A chain [Newton with one iteration, Newton with 20] restores u, the elements' basic state
and the fibers' trial state before its second attempt, so every step ends exactly where the plain
Newton run's does: the displacement histories are equal bit for bit, and each step's iteration
count is the plain count, plus one where the first attempt failed.  Without a chain,
ModifiedNewton gets Strut's automatic Newton fallback."""
import copy

import numpy as np

from strut_b200 import model as M
from strut_b200 import workloads as W


def _chain_case(steps):
    case = W.rc_frame_case(stories=3, bays=2, steps=steps, seed=33, pga_g=0.45)
    chain = copy.deepcopy(case)
    chain["analysis"]["solver_chain"] = [
        {"algorithm": "Newton", "test_type": "NormDispIncr", "max_iters": 1, "tol": 1e-8},
        {"algorithm": "Newton", "test_type": "NormDispIncr", "max_iters": 20, "tol": 1e-8},
    ]
    return case, chain


def test_chain_restores_the_step(oracle):
    steps = 150
    plain, chain = _chain_case(steps)
    d0, e0, i0, rc0, _ = oracle.run_transient(M.Model(plain), steps)
    d1, e1, i1, rc1, _ = oracle.run_transient(M.Model(chain), steps)
    assert rc0 == 0 and rc1 == 0
    assert np.array_equal(d0, d1)
    assert np.array_equal(e0, e1)
    retried = i1 != i0
    assert retried.sum() > steps // 2
    assert np.all(i1[retried] == i0[retried] + 1)
    assert np.all(i0[~retried] == 1)


def test_modified_newton_falls_back_to_newton(oracle):
    """ModifiedNewton with a 3-iteration limit fails some steps on its own; Strut's chain retries
    them with Newton, so the run completes."""
    steps = 120
    case = W.rc_frame_case(stories=3, bays=2, steps=steps, seed=34, pga_g=0.5)
    case["analysis"]["algorithm"] = "ModifiedNewton"
    case["analysis"]["max_iters"] = 3
    d, e, it, rc, failed = oracle.run_transient(M.Model(case), steps)
    assert rc == 0, f"failed at step {failed}"
    only = copy.deepcopy(case)
    only["analysis"]["solver_chain"] = [{"algorithm": "ModifiedNewton", "test_type": "NormDispIncr",
                                          "max_iters": 3, "tol": 1e-8}]
    _d, _e, _it, rc2, failed2 = oracle.run_transient(M.Model(only), steps)
    assert rc2 == 1 and failed2 >= 0  # the same settings with no fallback stop
    assert it.max() > 3  # some step needed the Newton attempt
