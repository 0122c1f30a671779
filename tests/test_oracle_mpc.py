"""Multi-point constraints (Transformation handler) in the CPU oracle.

The collapse is checked against an explicit transformation: at the same displacements, the
constrained model's effective band equals T^T K T of the unconstrained model inside the half
width detected from the elements' free dofs, entries outside it are dropped (as Strut's band
load drops them), and its F_int equals T^T F_int.
"""
import copy

import numpy as np
import pytest

from strut_b200 import model as M
from strut_b200 import workloads as W
from tests.helpers import band_to_dense, equal_dof_floors_2d, transformation_matrix


def _unconstrained(case):
    c = copy.deepcopy(case)
    c.pop("mp_constraints", None)
    c["analysis"].pop("constraints", None)
    return c


@pytest.mark.parametrize("case_fn", [
    lambda: W.rc_frame3d_case(stories=2, bays_x=2, bays_y=1, steps=5, element="dispBeamColumn3d",
                              diaphragm=True, seed=5),
    lambda: W.rc_frame3d_case(stories=2, bays_x=2, bays_y=2, steps=5, element="forceBeamColumn3d",
                              beam_element="dispBeamColumn3d", diaphragm=True, seed=6),
    lambda: equal_dof_floors_2d(W.rc_frame_case(stories=2, bays=2, steps=5, seed=7)),
])
def test_collapse_matches_transformation(oracle, case_fn):
    case = case_fn()
    case["rayleigh"] = {"alphaM": 0.0, "betaKInit": 0.0}
    m = M.Model(case)
    mf = M.Model(_unconstrained(case))
    T = transformation_matrix(m, mf)
    u = np.random.default_rng(0).normal(0.0, 2e-3, m.num_free)
    f_red, band_red, bw = oracle.state_determination(m, u)
    f_full, band_full, bw_full = oracle.state_determination(mf, T @ u)
    Kr = T.T @ band_to_dense(band_full, mf.num_free, bw_full) @ T
    Kb = band_to_dense(band_red, m.num_free, bw)
    n = m.num_free
    inside = np.abs(np.subtract.outer(np.arange(n), np.arange(n))) <= bw
    scale = np.abs(Kr).max()
    assert np.abs((Kr - Kb)[inside]).max() <= 1e-13 * scale
    assert np.abs(Kb[~inside]).max() == 0.0
    assert np.abs(T.T @ f_full - f_red).max() <= 1e-13 * np.abs(f_red).max()


def test_diaphragm_truncates_master_coupling(oracle):
    """With diaphragms the retained dofs couple beyond the detected half width; those entries
    exist in T^T K T and are absent from the band (Strut's behaviour, kept)."""
    case = W.rc_frame3d_case(stories=2, bays_x=2, bays_y=1, steps=5, element="dispBeamColumn3d",
                             diaphragm=True, seed=5)
    case["rayleigh"] = {"alphaM": 0.0, "betaKInit": 0.0}
    m = M.Model(case)
    mf = M.Model(_unconstrained(case))
    T = transformation_matrix(m, mf)
    u = np.zeros(m.num_free)
    _f, band_full, bw_full = oracle.state_determination(mf, T @ u)
    _f2, _band, bw = oracle.state_determination(m, u)
    Kr = T.T @ band_to_dense(band_full, mf.num_free, bw_full) @ T
    n = m.num_free
    outside = np.abs(np.subtract.outer(np.arange(n), np.arange(n))) > bw
    assert np.abs(Kr[outside]).max() > 1e-6 * np.abs(Kr).max()


def test_diaphragm_transient_runs(oracle):
    case = W.rc_frame3d_case(stories=2, bays_x=2, bays_y=1, steps=60, element="forceBeamColumn3d",
                             diaphragm=True, seed=9, pga_g=0.4, bidirectional=True)
    d, e, it, rc, failed = oracle.run_transient(M.Model(case), 60)
    assert rc == 0, failed
    assert np.abs(d[:, 0]).max() > 1e-4 and np.abs(d[:, 1]).max() > 1e-4


def test_slave_mass_is_rejected(oracle):
    case = W.rc_frame3d_case(stories=1, bays_x=1, bays_y=1, steps=5, diaphragm=True, seed=1)
    slave = case["mp_constraints"][0]["constrained_node"]
    case["masses"].append({"node": slave, "dof": 1, "value": 1000.0})
    d, e, it, rc, failed = oracle.run_transient(M.Model(case), 5)
    assert rc == 6  # STRUT_UNSUPPORTED


def test_model_errors():
    case = W.rc_frame3d_case(stories=1, bays_x=1, bays_y=1, steps=5, diaphragm=True, seed=1)
    bad = copy.deepcopy(case)
    bad["analysis"].pop("constraints")
    with pytest.raises(M.ModelError):
        M.Model(bad)
    bad = copy.deepcopy(case)
    bad["mp_constraints"].append(dict(bad["mp_constraints"][0]))
    with pytest.raises(M.ModelError):
        M.Model(bad)
