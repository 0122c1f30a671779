"""GPU parity: the sm_100a kernels (through the C ABI) against the CPU oracle.

Tolerances: the GPU sums sections and band rows in its own (warp-tree) order and contracts
multiply-adds into FMAs, and CUDA's pow differs from glibc's in the last bits, so results
agree to rounding, not bit for bit:
  * material / section responses: rtol 1e-9 (absolute floor 1e-9 of the largest value)
  * one state determination (F_int, effective band): rtol 1e-9 of the largest entry
  * transient histories: every displacement and element-force history within 1e-7 of its
    peak (the north-star criterion), Newton iteration counts equal on >= 99% of steps
"""
import numpy as np
import pytest

from strut_b200 import _abi as A
from strut_b200 import model as M
from strut_b200 import workloads as W
from tests.helpers import (ALTERNATING, lcg_strains, mixed_section_case, path_array,
                           rel_err_of_peak)

pytestmark = pytest.mark.gpu

MATS = [
    {"id": 1, "type": "Steel02", "params": dict(W.STEEL)},
    {"id": 2, "type": "Concrete02", "params": dict(W.CORE)},
    {"id": 3, "type": "Concrete02", "params": dict(W.COVER)},
    {"id": 4, "type": "Steel01", "params": {"Fy": 350.0e6, "E0": 200.0e9, "b": 0.01}},
    {"id": 5, "type": "Elastic", "params": {"E": 30.0e9}},
    {"id": 6, "type": "Concrete01", "params": {"fpc": -30.0e6, "epsc0": -0.002, "fpcu": -6.0e6,
                                                "epscu": -0.006}},
]


@pytest.mark.parametrize("mat", MATS, ids=[m["type"] + str(m["id"]) for m in MATS])
def test_material_path(gpu_lib, oracle, mat):
    strains = lcg_strains(mat["id"] * 11 + 3, 600, 0.004, "cyclic")
    m = M.uniaxial_material(mat)
    ref = oracle.material_path(m, strains)
    got = gpu_lib.material_path(m, strains)
    scale = np.max(np.abs(ref), axis=0)
    np.testing.assert_allclose(got, ref, rtol=1e-9, atol=1e-9 * float(scale.max()))


def test_section_path_mixed(gpu_lib, oracle):
    case = mixed_section_case(ALTERNATING)
    mats, nm, fibs, nf = M.section_fibers(case["section"], case["materials"])
    ref = oracle.section_path(mats, nm, fibs, nf, path_array(case))
    got = gpu_lib.section_path(mats, nm, fibs, nf, path_array(case))
    np.testing.assert_allclose(got, ref, rtol=1e-9, atol=1e-9 * np.abs(ref).max())


def test_section_path_rc_long_history(gpu_lib, oracle):
    """The 148-fiber RC column section through a 300-point cyclic (eps0, kappa) path."""
    case = {"materials": [
        {"id": 1, "type": "Concrete02", "params": dict(W.CORE)},
        {"id": 2, "type": "Concrete02", "params": dict(W.COVER)},
        {"id": 3, "type": "Steel02", "params": dict(W.STEEL)}],
        "section": W.rc_section(1, 0.5, 0.5)}
    mats, nm, fibs, nf = M.section_fibers(case["section"], case["materials"])
    k = lcg_strains(5, 300, 0.004, "cyclic")
    e = -0.0005 + 0.3 * lcg_strains(6, 300, 0.001, "walk")
    ek = np.stack([e, k], axis=1)
    ref = oracle.section_path(mats, nm, fibs, nf, ek)
    got = gpu_lib.section_path(mats, nm, fibs, nf, ek)
    scale = np.abs(ref).max(axis=0)
    assert np.all(np.abs(got - ref) <= 1e-9 * scale + 1e-12)


@pytest.mark.parametrize("which", ["rc", "mixed"])
def test_section_batch_matches_oracle(gpu_lib, oracle, which):
    """257 histories of one section through the streaming kernel against the oracle: the 148-fiber
    RC column section, and a section with every family (Steel02, Concrete02, Steel01, Concrete01,
    elastic fibers with their own k12).  Before every committing call the same point is evaluated
    without commit: it returns the same response and leaves the histories where they were."""
    import torch

    if which == "rc":
        case = {"materials": [
            {"id": 1, "type": "Concrete02", "params": dict(W.CORE)},
            {"id": 2, "type": "Concrete02", "params": dict(W.COVER)},
            {"id": 3, "type": "Steel02", "params": dict(W.STEEL)}],
            "section": W.rc_section(1, 0.4, 0.6)}
    else:
        case = mixed_section_case(ALTERNATING)
    mats, nm, fibs, nf = M.section_fibers(case["section"], case["materials"])
    n_inst, npts = 257, 40
    rng = np.random.default_rng(0)
    ek = np.zeros((npts, n_inst, 2))
    ek[:, :, 0] = np.cumsum(rng.normal(0, 2e-4, (npts, n_inst)), axis=0)
    ek[:, :, 1] = np.cumsum(rng.normal(0, 2e-3, (npts, n_inst)), axis=0)
    ref = oracle.section_batch_path(mats, nm, fibs, nf, ek)
    d_ek = torch.empty((n_inst, 2), dtype=torch.float64, device="cuda")
    d_r = torch.empty((n_inst, 5), dtype=torch.float64, device="cuda")
    b = gpu_lib.SectionBatch(mats, nm, fibs, nf, n_inst)
    got = np.zeros_like(ref)
    for p in range(npts):
        d_ek.copy_(torch.from_numpy(ek[p]))
        b.eval(d_ek.data_ptr(), d_r.data_ptr(), commit=False)
        trial = d_r.cpu().numpy()
        b.eval(d_ek.data_ptr(), d_r.data_ptr(), commit=True)
        got[p] = d_r.cpu().numpy()
        assert np.array_equal(trial, got[p])
    b.close()
    scale = np.abs(ref).max(axis=(0, 1))
    assert np.all(np.abs(got - ref) <= 1e-9 * scale + 1e-12)


def _random_u(m, seed, scale=0.02):
    rng = np.random.default_rng(seed)
    u = rng.normal(0.0, scale, m.num_free)
    u[2::3] *= 0.05  # rotations smaller
    return u


@pytest.mark.parametrize("element,geom", [("forceBeamColumn2d", "Linear"),
                                          ("dispBeamColumn2d", "Linear"),
                                          ("forceBeamColumn2d", "PDelta"),
                                          ("dispBeamColumn2d", "PDelta")])
def test_state_determination(gpu_lib, oracle, element, geom):
    case = W.rc_frame_case(steps=10, element=element, geom=geom)
    m = M.Model(case)
    u = _random_u(m, 1, 0.01)
    f_ref, band_ref, bw = oracle.state_determination(m, u)
    with gpu_lib.Analysis([m]) as an:
        (f_got, band_got), = an.state_determination([u])
        assert an.band_info(0)[0] == bw
    assert np.max(np.abs(f_got - f_ref)) <= 1e-9 * np.max(np.abs(f_ref))
    assert np.max(np.abs(band_got - band_ref)) <= 1e-9 * np.max(np.abs(band_ref))


def test_factor_solve(gpu_lib, oracle):
    case = W.rc_frame_case(steps=10)
    m = M.Model(case)
    u = _random_u(m, 2, 0.005)
    with gpu_lib.Analysis([m]) as an:
        (_f, band), = an.state_determination([u])
        bw, rw = an.band_info(0)
        n = m.num_free
        K = np.zeros((n, n))
        for i in range(n):
            for o in range(rw):
                j = i + o - bw
                if 0 <= j < n:
                    K[i, j] = band[i, o]
        rhs = np.random.default_rng(3).normal(size=n)
        du, = an.factor_solve([rhs])
    ref = np.linalg.solve(K, rhs)
    np.testing.assert_allclose(du, ref, rtol=1e-8, atol=1e-12 * np.abs(ref).max())


def _transient_parity(gpu_lib, oracle, cases, steps, iters_frac=0.99):
    models = [M.Model(c) for c in cases]
    with gpu_lib.Analysis(models) as an:
        an.run(steps)
        got = [an.history(i) for i in range(len(models))]
    for m, (gd, ge, gi) in zip(models, got):
        rd, re, ri, rc, failed = oracle.run_transient(m, steps)
        assert rc == 0, f"oracle failed at step {failed}"
        for j in range(rd.shape[1]):
            assert rel_err_of_peak(gd[:, j], rd[:, j]) <= 1e-7, f"disp dof {j}"
        for j in range(re.shape[1]):
            for c in range(6):
                assert rel_err_of_peak(ge[:, j, c], re[:, j, c]) <= 1e-7, f"eforce {j},{c}"
        assert np.mean(gi == ri) >= iters_frac
    return got


def test_transient_config0_short(gpu_lib, oracle):
    """The 3-story 3-bay RC frame of the single-instance plain workload, 300 steps."""
    case = W.rc_frame_case(steps=300)
    _transient_parity(gpu_lib, oracle, [case], 300)


def test_transient_disp_beam_pdelta(gpu_lib, oracle):
    case = W.rc_frame_case(stories=2, bays=2, steps=200, element="dispBeamColumn2d",
                           geom="PDelta", seed=11, pga_g=0.4)
    _transient_parity(gpu_lib, oracle, [case], 200)


def test_transient_batched_uneven(gpu_lib, oracle):
    """Six frames of different sizes and records in one handle (per-instance masks)."""
    params = W.batched_frame_params(6, base_seed=2000)
    cases = [W.rc_frame_case(stories=min(p["stories"], 6), bays=p["bays"], wg=p["wg"],
                             pga_g=p["pga_g"], seed=p["seed"], steps=150) for p in params]
    _transient_parity(gpu_lib, oracle, cases, 150)


def test_transient_band_spd_small_units(gpu_lib, oracle):
    """BandSPD needs a K symmetric to 1e-10 (linear_solver_backend.mojo:266-271): a frame in
    kN / m units with an elastic-dominated response keeps it."""
    case = W.rc_frame_case(stories=2, bays=1, steps=80, system="BandSPD", seed=5, pga_g=0.05)
    for m in case["materials"]:
        for k in list(m["params"]):
            if k in ("fpc", "fpcu", "ft", "Ets", "Fy", "E0"):
                m["params"][k] = m["params"][k] * 1e-6
    for ms in case["masses"]:
        ms["value"] *= 1e-6
    case["rayleigh"] = {"alphaM": 0.5, "betaKInit": 0.0}
    models = [M.Model(case)]
    rd, re, ri, rc, failed = oracle.run_transient(models[0], 80)
    with gpu_lib.Analysis(models) as an:
        st = an.run(80, check=False)
        if rc != 0:
            # both sides must reject the same model at the same step
            assert an.last_status == rc
            return
        gd, ge, gi = an.history(0)
    for j in range(rd.shape[1]):
        assert rel_err_of_peak(gd[:, j], rd[:, j]) <= 1e-7


def test_nonconvergence_reported(gpu_lib):
    case = W.rc_frame_case(stories=2, bays=1, steps=10, seed=3, pga_g=0.5, tol=1e-30, max_iters=2)
    with gpu_lib.Analysis([M.Model(case)]) as an:
        st = an.run(10, check=False)
        assert an.last_status == A.STRUT_NONCONVERGED
        assert st.failed_instance == 0 and st.failed_step == 0


def test_run_split_equals_single_run(gpu_lib):
    """Running 40 + 60 steps gives the same history as 100 steps in one call."""
    case = W.rc_frame_case(stories=2, bays=2, steps=100, seed=21)
    m1, m2 = M.Model(case), M.Model(case)
    with gpu_lib.Analysis([m1]) as a:
        a.run(100)
        d1, e1, i1 = a.history(0)
    with gpu_lib.Analysis([m2]) as b:
        b.run(40)
        b.run(60)
        d2, e2, i2 = b.history(0)
    assert np.array_equal(d1, d2) and np.array_equal(e1, e2) and np.array_equal(i1, i2)


def test_transient_frame_with_pivoting_fallback(gpu_lib, oracle):
    """Frame 21 of the 256-frame batch (4 stories, 3 bays, PGA 0.6 g): around step 71 a
    sub-diagonal entry of the effective matrix ties with its pivot, so either side may switch
    to the dense partial-pivot LU of linear_solver_backend.mojo:175-240; the histories agree
    to the parity tolerance whichever factorization each side takes."""
    p = W.batched_frame_params(256)[21]
    case = W.rc_frame_case(stories=p["stories"], bays=p["bays"], wg=p["wg"], pga_g=p["pga_g"],
                           seed=p["seed"], steps=120)
    _transient_parity(gpu_lib, oracle, [case], 120)


def test_failed_instance_is_masked_and_others_continue(gpu_lib):
    """One record of a batch that cannot converge (tol 1e-30) is masked out at its failing
    step; the other record runs every step and matches its solo run bit for bit."""
    ok = W.rc_frame_case(stories=2, bays=2, steps=60, seed=31)
    bad = W.rc_frame_case(stories=2, bays=1, steps=60, seed=32, tol=1e-30, max_iters=3)
    with gpu_lib.Analysis([M.Model(bad), M.Model(ok)]) as an:
        st = an.run(60, check=False)
        assert an.last_status == A.STRUT_NONCONVERGED
        assert st.failed_instance == 0 and st.failed_step == 0 and st.steps_done == 60
        assert list(an.instance_status()) == [A.STRUT_NONCONVERGED, A.STRUT_OK]
        d_batch, e_batch, i_batch = an.history(1)
    with gpu_lib.Analysis([M.Model(ok)]) as solo:
        solo.run(60)
        d_solo, e_solo, i_solo = solo.history(0)
    assert np.array_equal(d_batch, d_solo) and np.array_equal(i_batch, i_solo)


def test_graph_loop_equals_host_loop(gpu_lib):
    """The CUDA-graph step loop (conditional WHILE nodes) and the host-driven loop used while
    profiling launch the same kernels in the same order: identical histories, bit for bit."""
    cases = [W.rc_frame_case(stories=s, bays=b, steps=50, seed=40 + s) for s, b in ((2, 1), (3, 2))]
    out = []
    for prof in (0, 1):
        models = [M.Model(c) for c in cases]
        with gpu_lib.Analysis(models) as an:
            gpu_lib.lib().strut_gpu_set_profiling(an.h, prof)
            an.run(20)
            an.run(30)
            out.append([an.history(i) for i in range(2)])
    for (d0, e0, i0), (d1, e1, i1) in zip(out[0], out[1]):
        assert np.array_equal(d0, d1) and np.array_equal(e0, e1) and np.array_equal(i0, i1)


def _concrete01_frame(element, steps, seed):
    """The RC frame with its cover concrete as Concrete01 (fpc -30 MPa, epsc0 -0.002, fpcu 0,
    epscu -0.004)."""
    case = W.rc_frame_case(stories=2, bays=2, steps=steps, element=element, seed=seed, pga_g=0.4)
    for m in case["materials"]:
        if m["id"] == 2:
            m["type"] = "Concrete01"
            m["params"] = {"fpc": -30.0e6, "epsc0": -0.002, "fpcu": 0.0, "epscu": -0.004}
    return case


@pytest.mark.parametrize("element", ["forceBeamColumn2d", "dispBeamColumn2d"])
def test_transient_concrete01_cover(gpu_lib, oracle, element):
    _transient_parity(gpu_lib, oracle, [_concrete01_frame(element, 150, 31)], 150)
