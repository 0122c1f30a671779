"""Slab shells (ShellMITC4 on ElasticMembranePlateSection, elements/shell4.mojo:10-363) on the GPU
against the oracle: the device-computed shell stiffness enters the band exactly like the
oracle's (one state determination within 1e-9 of the largest entry), and frame + slab
transients agree within 1e-7 of peak with Newton iteration counts equal on >= 99% of steps."""
import numpy as np
import pytest

from strut_b200 import model as M
from strut_b200 import workloads as W
from tests.helpers import rel_err_of_peak

pytestmark = pytest.mark.gpu

SLABS = {"E": 30.0e9, "nu": 0.2, "h": 0.2, "rho": 2400.0}


def slab_frame(steps, diaphragm=False, seed=61, **kw):
    # with a rigid diaphragm the slab's in-plane dofs are slaves, which may carry no mass: its
    # mass then belongs to the diaphragm's retained node (rho 0 here)
    slabs = dict(SLABS, rho=0.0) if diaphragm else SLABS
    return W.rc_frame3d_case(stories=2, bays_x=2, bays_y=2, steps=steps, element="forceBeamColumn3d",
                             beam_element="dispBeamColumn3d", seed=seed, pga_g=0.3, slabs=slabs,
                             bidirectional=True, diaphragm=diaphragm, record_elements=(1,), **kw)


def test_slab_state_determination(gpu_lib, oracle):
    m = M.Model(slab_frame(5))
    u = np.random.default_rng(4).normal(0.0, 2e-4, m.num_free)
    f_ref, band_ref, bw = oracle.state_determination(m, u)
    with gpu_lib.Analysis([m]) as an:
        (f_got, band_got), = an.state_determination([u])
        assert an.band_info(0)[0] == bw
    assert np.max(np.abs(f_got - f_ref)) <= 1e-9 * np.max(np.abs(f_ref))
    assert np.max(np.abs(band_got - band_ref)) <= 1e-9 * np.max(np.abs(band_ref))


@pytest.mark.parametrize("diaphragm", [False, True])
def test_slab_frame_transient(gpu_lib, oracle, diaphragm):
    steps = 80
    m = M.Model(slab_frame(steps, diaphragm=diaphragm))
    with gpu_lib.Analysis([m]) as an:
        an.run(steps)
        gd, ge, gi = an.history(0)
    rd, re, ri, rc, failed = oracle.run_transient(m, steps)
    assert rc == 0, f"oracle failed at step {failed}"
    for j in range(rd.shape[1]):
        if np.max(np.abs(rd[:, j])) > 1e-9:
            assert rel_err_of_peak(gd[:, j], rd[:, j]) <= 1e-7, f"disp {j}"
    assert np.max(np.abs(ge - re)) <= 1e-7 * np.max(np.abs(re))
    assert np.mean(gi == ri) >= 0.99
