"""strut_gpu_band_solve_noalloc: the band factor-solve on a caller's device buffers, for callers
that may not allocate device memory themselves or have the library do it (for instance a host
that reserves all device memory up front, or that must not trigger the device-wide
synchronisation a cudaMalloc / cudaFree can cause between Newton iterations).  Its scratch is a
static device array.  Checked against strut_gpu_factor_solve on the same effective matrix, two
calls in a row.  This file is collected last, so a run that stops at the first failure has run
every other test before it."""
import ctypes as C

import numpy as np
import pytest

from strut_b200 import _abi as A
from strut_b200 import model as M
from strut_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def _solve_noalloc(gpu_lib, band, n, bw, system, rhs):
    """Two calls in a row on the same device buffers; returns [(status, x), (status, x)]."""
    import torch

    band_d = torch.tensor(np.ascontiguousarray(band).reshape(-1), dtype=torch.float64, device="cuda")
    rhs_d = torch.tensor(rhs, dtype=torch.float64, device="cuda")
    x_d = torch.zeros(n, dtype=torch.float64, device="cuda")
    st = torch.full((1,), -1, dtype=torch.int32, device="cuda")
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    out = []
    for _ in range(2):
        x_d.zero_()
        st.fill_(-1)
        rc = gpu_lib.lib().strut_gpu_band_solve_noalloc(_ptr(band_d), n, bw, system, _ptr(rhs_d), _ptr(x_d),
                                                        _ptr(st), stream)
        assert rc == A.STRUT_OK, gpu_lib.lib().strut_gpu_last_error()
        torch.cuda.synchronize()
        out.append((int(st.item()), x_d.cpu().numpy().copy()))
    return out


def _small_units(case):
    # kN / m units keep K symmetric to BandSPD's 1e-10 check (linear_solver_backend.mojo:266-271)
    for m in case["materials"]:
        for k in list(m["params"]):
            if k in ("fpc", "fpcu", "ft", "Ets", "Fy", "E0"):
                m["params"][k] = m["params"][k] * 1e-6
    for ms in case["masses"]:
        ms["value"] *= 1e-6
    case["rayleigh"] = {"alphaM": 0.5, "betaKInit": 0.0}
    return case


@pytest.mark.parametrize("system", ["BandGeneral", "BandSPD"])
def test_noalloc_matches_factor_solve(gpu_lib, system):
    case = W.rc_frame_case(stories=3, bays=3, steps=10, seed=11, system=system)
    if system == "BandSPD":
        case = _small_units(case)
    model = M.Model(case)
    rng = np.random.default_rng(3)
    n = model.num_free
    u = rng.standard_normal(n) * 1e-4
    rhs = rng.standard_normal(n)
    with gpu_lib.Analysis([model]) as an:
        [(_f, band)] = an.state_determination([u])
        [du_ref] = an.factor_solve([rhs])
        bw, _rw = an.band_info(0)
    code = A.SYSTEM_BAND_SPD if system == "BandSPD" else A.SYSTEM_BAND_GENERAL
    scale = np.abs(du_ref).max()
    for st, x in _solve_noalloc(gpu_lib, band, n, bw, code, rhs):
        assert st == 0
        assert np.abs(x - du_ref).max() <= 1e-12 * scale


def test_noalloc_dense_fallback(gpu_lib):
    """A sub-diagonal entry larger than its pivot sends BandGeneral to the dense partial-pivot LU,
    which works in the static scratch; checked against numpy's LU solve."""
    rng = np.random.default_rng(8)
    n, bw = 40, 3
    K = np.zeros((n, n))
    for i in range(n):
        for j in range(max(0, i - bw), min(n, i + bw + 1)):
            K[i, j] = rng.standard_normal()
        K[i, i] += 4.0
    K[5, 4] = 50.0  # |a_54| > |a_44| at step 4
    band = np.zeros((n, 2 * bw + 1))
    for i in range(n):
        for j in range(max(0, i - bw), min(n, i + bw + 1)):
            band[i, j - i + bw] = K[i, j]
    rhs = rng.standard_normal(n)
    ref = np.linalg.solve(K, rhs)
    for st, x in _solve_noalloc(gpu_lib, band, n, bw, A.SYSTEM_BAND_GENERAL, rhs):
        assert st == 0
        assert np.abs(x - ref).max() <= 1e-10 * np.abs(ref).max()


def test_noalloc_rejects_sizes_beyond_scratch(gpu_lib):
    rc = gpu_lib.lib().strut_gpu_band_solve_noalloc(None, 100000, 2, A.SYSTEM_BAND_GENERAL, None, None, None,
                                                    None)
    assert rc == A.STRUT_BAD_ARG
    assert b"static scratch" in gpu_lib.lib().strut_gpu_last_error()


def test_noalloc_dense_fallback_at_the_largest_order(gpu_lib):
    """n = 512, the largest order the static scratch holds, through the dense fallback."""
    rng = np.random.default_rng(21)
    n, bw = 512, 3
    band = np.zeros((n, 2 * bw + 1))
    K = np.zeros((n, n))
    for i in range(n):
        for j in range(max(0, i - bw), min(n, i + bw + 1)):
            K[i, j] = rng.standard_normal() + (5.0 if i == j else 0.0)
    K[300, 299] = 80.0  # sends the factorisation to the dense partial-pivot LU
    for i in range(n):
        for j in range(max(0, i - bw), min(n, i + bw + 1)):
            band[i, j - i + bw] = K[i, j]
    rhs = rng.standard_normal(n)
    ref = np.linalg.solve(K, rhs)
    for st, x in _solve_noalloc(gpu_lib, band, n, bw, A.SYSTEM_BAND_GENERAL, rhs):
        assert st == 0
        assert np.abs(x - ref).max() <= 1e-10 * np.abs(ref).max()


def test_noalloc_reports_singular_and_not_positive_definite(gpu_lib):
    """Status 2 on the device: a BandGeneral system with a zero column (singular in the band LU
    and in its dense fallback) and a BandSPD system with a negative diagonal."""
    n, bw = 30, 2
    gen = np.zeros((n, 2 * bw + 1))
    spd = np.zeros((n, bw + 1))
    for i in range(n):
        gen[i, bw] = 4.0
        spd[i, 0] = 4.0
        for o in range(1, bw + 1):
            if i - o >= 0:
                gen[i, bw - o] = -1.0
                spd[i, o] = -1.0
            if i + o < n:
                gen[i, bw + o] = -1.0
    for i in range(n):  # column 7 of the general matrix is zero
        if abs(7 - i) <= bw:
            gen[i, 7 - i + bw] = 0.0
    spd[11, 0] = -4.0
    rhs = np.ones(n)
    for st, _x in _solve_noalloc(gpu_lib, gen, n, bw, A.SYSTEM_BAND_GENERAL, rhs):
        assert st == A.STRUT_SINGULAR
    for st, _x in _solve_noalloc(gpu_lib, spd, n, bw, A.SYSTEM_BAND_SPD, rhs):
        assert st == A.STRUT_SINGULAR
