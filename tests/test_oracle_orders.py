"""The reference's own summation orders on the plain single-instance record.

Strut sums fiber families in SIMD-width chunks (solver/simd_contiguous.mojo:6, 197-225), so the
same model gives slightly different rounding on hosts of different vector width.  On the
3-story 3-bay RC frame's full 2000-step record the oracle at widths 1, 8 and 16, and at width 8
with contracted multiply-adds, agrees to rounding level (1e-10 of peak) with identical Newton
iteration counts on every step: this record has no rounding-level divergence, which is why the
GPU is held to identical counts on it (tests/test_gpu_records.py)."""
import numpy as np

from strut_b200 import model as M
from strut_b200 import workloads as W
from tests.helpers import rel_err_of_peak
from tests.test_gpu_records import record_everything


def test_config0_orders_agree(oracle):
    steps = 2000
    m = M.Model(record_everything(W.rc_frame_case(steps=steps)))
    runs = {}
    try:
        for w, fma in ((1, False), (8, False), (16, False), (8, True)):
            oracle.use_fma(fma)
            oracle.set_simd_width(w)
            d, e, it, rc, failed = oracle.run_transient(m, steps)
            assert rc == 0, f"width {w} failed at step {failed}"
            runs[(w, fma)] = (d, e, it)
    finally:
        oracle.use_fma(False)
        oracle.set_simd_width(8)
    d8, e8, i8 = runs[(8, False)]
    for w in ((1, False), (16, False), (8, True)):
        d, e, it = runs[w]
        assert np.array_equal(it, i8), f"width {w}: iteration counts differ"
        for j in range(d8.shape[1]):
            if np.max(np.abs(d8[:, j])) > 0.0:
                assert rel_err_of_peak(d[:, j], d8[:, j]) <= 1e-10
        for j in range(e8.shape[1]):
            for c in range(e8.shape[2]):
                if np.max(np.abs(e8[:, j, c])) > 0.0:
                    assert rel_err_of_peak(e[:, j, c], e8[:, j, c]) <= 1e-10
