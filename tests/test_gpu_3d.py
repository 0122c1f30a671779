"""GPU parity of the 3D path (forceBeamColumn3d / dispBeamColumn3d with FiberSection3d)
through the C ABI against the CPU oracle.

Tolerances as for the 2D path: one state determination within 1e-9 of the largest entry;
transient histories within 1e-7 of peak with Newton iteration counts equal on >= 99% of steps.
"""
import numpy as np
import pytest

from strut_b200 import model as M
from strut_b200 import workloads as W
from tests.helpers import planar_frame_3d, rel_err_of_peak

pytestmark = pytest.mark.gpu


def _random_u(m, seed, scale):
    rng = np.random.default_rng(seed)
    u = rng.normal(0.0, scale, m.num_free)
    rot = np.zeros(m.num_dofs, dtype=bool)
    for node in range(m.num_nodes):
        rot[node * 6 + 3:node * 6 + 6] = True
    free_rot = np.array([rot[d] for d in range(m.num_dofs) if m.free_index[d] >= 0])
    u[free_rot] *= 0.05
    return u


@pytest.mark.parametrize("element,geom", [("forceBeamColumn3d", "Linear"),
                                          ("dispBeamColumn3d", "Linear"),
                                          ("forceBeamColumn3d", "PDelta"),
                                          ("dispBeamColumn3d", "Corotational"),
                                          ("forceBeamColumn3d", "Corotational")])
def test_state_determination_3d(gpu_lib, oracle, element, geom):
    case = W.rc_frame3d_case(stories=2, bays_x=1, bays_y=1, steps=10, element=element, geom=geom)
    m = M.Model(case)
    u = _random_u(m, 3, 0.004)
    f_ref, band_ref, bw = oracle.state_determination(m, u)
    with gpu_lib.Analysis([m]) as an:
        (f_got, band_got), = an.state_determination([u])
        assert an.band_info(0)[0] == bw
    assert np.max(np.abs(f_got - f_ref)) <= 1e-9 * np.max(np.abs(f_ref))
    assert np.max(np.abs(band_got - band_ref)) <= 1e-9 * np.max(np.abs(band_ref))


def _parity_3d(gpu_lib, oracle, cases, steps, iters_frac=0.99):
    models = [M.Model(c) for c in cases]
    with gpu_lib.Analysis(models) as an:
        an.run(steps)
        got = [an.history(i) for i in range(len(models))]
    for m, (gd, ge, gi) in zip(models, got):
        rd, re, ri, rc, failed = oracle.run_transient(m, steps)
        assert rc == 0, f"oracle failed at step {failed}"
        for j in range(rd.shape[1]):
            if np.max(np.abs(rd[:, j])) > 1e-9:
                assert rel_err_of_peak(gd[:, j], rd[:, j]) <= 1e-7, f"disp {j}"
        for j in range(re.shape[1]):
            peak = np.max(np.abs(re[:, j, :]))
            assert np.max(np.abs(ge[:, j, :] - re[:, j, :])) <= 1e-7 * peak, f"eforce {j}"
        assert np.mean(gi == ri) >= iters_frac
    return got


@pytest.mark.parametrize("element", ["forceBeamColumn3d", "dispBeamColumn3d"])
def test_transient_3d_frame(gpu_lib, oracle, element):
    case = W.rc_frame3d_case(stories=2, bays_x=2, bays_y=1, steps=150, element=element, seed=21,
                             pga_g=0.4, record_elements=(1, 4))
    _parity_3d(gpu_lib, oracle, [case], 150)


def test_transient_3d_bidirectional_pdelta(gpu_lib, oracle):
    case = W.rc_frame3d_case(stories=2, bays_x=1, bays_y=1, steps=120, element="forceBeamColumn3d",
                             geom="PDelta", seed=8, pga_g=0.45, bidirectional=True,
                             record_elements=(1, 2, 1))
    _parity_3d(gpu_lib, oracle, [case], 120)


def test_transient_3d_batched_uneven(gpu_lib, oracle):
    cases = [W.rc_frame3d_case(stories=s, bays_x=bx, bays_y=1, steps=80, seed=300 + s, pga_g=0.35,
                               element=el)
             for s, bx, el in ((1, 1, "forceBeamColumn3d"), (2, 2, "dispBeamColumn3d"),
                               (3, 1, "forceBeamColumn3d"))]
    _parity_3d(gpu_lib, oracle, cases, 80)


@pytest.mark.parametrize("element", ["forceBeamColumn2d", "dispBeamColumn2d"])
def test_plane_frame_as_3d_model_matches_2d_on_gpu(gpu_lib, element):
    steps = 150
    c2 = W.rc_frame_case(stories=2, bays=2, steps=steps, element=element, seed=11, pga_g=0.4)
    c3 = planar_frame_3d(c2)
    with gpu_lib.Analysis([M.Model(c2)]) as an:
        an.run(steps)
        d2, _e2, i2 = an.history(0)
    with gpu_lib.Analysis([M.Model(c3)]) as an:
        an.run(steps)
        d3, _e3, i3 = an.history(0)
    assert np.array_equal(i2, i3)
    for j, sgn in enumerate((1.0, 1.0, -1.0)):
        assert rel_err_of_peak(sgn * d3[:, j], d2[:, j]) <= 1e-9


def test_mixed_2d_3d_batch_is_rejected(gpu_lib):
    m2 = M.Model(W.rc_frame_case(stories=1, bays=1, steps=5))
    m3 = M.Model(W.rc_frame3d_case(stories=1, bays_x=1, bays_y=1, steps=5))
    with pytest.raises(RuntimeError):
        gpu_lib.Analysis([m2, m3])


def test_section3d_path_rc_cyclic(gpu_lib, oracle):
    """The RC FiberSection3d along a biaxial cyclic path with commits (KAT driver form)."""
    from tests.helpers import lcg_strains

    mats = [{"id": 1, "type": "Concrete02", "params": dict(W.CORE)},
            {"id": 2, "type": "Concrete02", "params": dict(W.COVER)},
            {"id": 3, "type": "Steel02", "params": dict(W.STEEL)},
            {"id": 4, "type": "Elastic", "params": {"E": 30.0e9}}]
    sec = W.rc_section(1, 0.4, 0.6, three_d=True)
    sec["params"]["fibers"] = [{"y": 0.05, "z": 0.02, "area": 1e-3, "material": 4}]
    m, nm, f, nf = M.section_fibers(sec, mats)
    n = 400
    path = np.stack([lcg_strains(1, n, 2.0e-4, "walk") - 3.0e-4,
                     lcg_strains(2, n, 3.0e-3, "cyclic") * 0.01,
                     lcg_strains(3, n, 4.0e-3, "cyclic") * 0.01], 1)
    ref = oracle.section3d_path(m, nm, f, nf, path)
    got = gpu_lib.section3d_path(m, nm, f, nf, path)
    scale = np.maximum(np.abs(ref).max(0), 1e-30)
    assert np.all(np.abs(got - ref).max(0) <= 1e-9 * scale)


# ---- bands beyond shared memory (blocked LU in global memory) ---------------------------------

def _large_case(steps, seed=41, element="forceBeamColumn3d", bays_x=3, bays_y=2, stories=3):
    # 12 nodes per floor: n = 216, half band ~77 -> a 268 KB band, factored in global memory
    return W.rc_frame3d_case(stories=stories, bays_x=bays_x, bays_y=bays_y, steps=steps,
                             element=element, seed=seed, pga_g=0.4, record_elements=(1,))


def test_large_band_factor_solve(gpu_lib):
    m = M.Model(_large_case(10))
    u = _random_u(m, 5, 0.003)
    with gpu_lib.Analysis([m]) as an:
        bw, rw = an.band_info(0)
        assert m.num_free * rw * 8 > 220 * 1024
        (_f, band), = an.state_determination([u])
        n = m.num_free
        K = np.zeros((n, n))
        for i in range(n):
            for o in range(rw):
                j = i + o - bw
                if 0 <= j < n:
                    K[i, j] = band[i, o]
        rhs = np.random.default_rng(7).normal(size=n)
        du, = an.factor_solve([rhs])
    ref = np.linalg.solve(K, rhs)
    np.testing.assert_allclose(du, ref, rtol=1e-8, atol=1e-12 * np.abs(ref).max())


def test_large_band_state_determination(gpu_lib, oracle):
    m = M.Model(_large_case(10, element="dispBeamColumn3d"))
    u = _random_u(m, 6, 0.003)
    f_ref, band_ref, bw = oracle.state_determination(m, u)
    with gpu_lib.Analysis([m]) as an:
        (f_got, band_got), = an.state_determination([u])
    assert np.max(np.abs(f_got - f_ref)) <= 1e-9 * np.max(np.abs(f_ref))
    assert np.max(np.abs(band_got - band_ref)) <= 1e-9 * np.max(np.abs(band_ref))


def test_large_band_transient(gpu_lib, oracle):
    _parity_3d(gpu_lib, oracle, [_large_case(80)], 80)


def test_large_and_small_bands_in_one_batch(gpu_lib, oracle):
    cases = [_large_case(60, seed=51),
             W.rc_frame3d_case(stories=1, bays_x=1, bays_y=1, steps=60, seed=52, pga_g=0.4),
             _large_case(60, seed=53, element="dispBeamColumn3d", bays_x=2, bays_y=3)]
    _parity_3d(gpu_lib, oracle, cases, 60)
