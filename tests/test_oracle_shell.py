"""ShellMITC4 on an ElasticMembranePlateSection (elements/shell4.mojo:10-363), oracle side:
properties every correct element stiffness has (symmetry, the six rigid-body modes in its null
space, an exact constant-strain membrane patch), and a slab-stiffened 3D frame transient."""
import numpy as np
import pytest

from strut_b200 import model as M
from strut_b200 import workloads as W

E, NU, H = 30.0e9, 0.2, 0.2


def _rigid_modes(P):
    c = P.mean(0)
    modes = []
    for k in range(3):  # translations
        r = np.zeros(24)
        r[k::6] = 1.0
        modes.append(r)
    for k in range(3):  # rotations about the centroid: u = w x (p - c), theta = w
        w = np.zeros(3)
        w[k] = 1.0
        r = np.zeros(24)
        for i in range(4):
            r[6 * i:6 * i + 3] = np.cross(w, P[i] - c)
            r[6 * i + 3:6 * i + 6] = w
        modes.append(r)
    return modes


@pytest.mark.parametrize("P", [
    np.array([[0, 0, 3.5], [7, 0, 3.5], [7, 7, 3.5], [0, 7, 3.5]], dtype=float),
    np.array([[0, 0, 0], [6, 0.5, 0], [6.5, 5, 0], [-0.3, 4.5, 0]], dtype=float),  # distorted, flat
    np.array([[1, 2, 3], [4, 2, 3], [4, 2, 6], [1, 2, 6]], dtype=float),          # vertical
])
def test_symmetric_with_rigid_body_null_space(oracle, P):
    K = oracle.shell4_stiffness(E, NU, H, P)
    scale = np.abs(K).max()
    assert np.max(np.abs(K - K.T)) <= 1e-12 * scale
    for r in _rigid_modes(P):
        assert np.max(np.abs(K @ r)) <= 1e-9 * scale * np.abs(r).max()
    # positive semi-definite with exactly six zero modes
    ev = np.linalg.eigvalsh(0.5 * (K + K.T))
    assert np.sum(ev < 1e-9 * ev.max()) == 6 and ev.min() > -1e-9 * ev.max()


def test_warped_shell_keeps_translations(oracle):
    """The reference projects a warped quadrilateral onto its g1-g2 plane without a warping
    correction, so only the rigid translations stay exact there."""
    P = np.array([[0, 0, 0], [6, 0.5, 0.3], [6.5, 5, 0.2], [-0.3, 4.5, -0.1]], dtype=float)
    K = oracle.shell4_stiffness(E, NU, H, P)
    scale = np.abs(K).max()
    assert np.max(np.abs(K - K.T)) <= 1e-12 * scale
    for r in _rigid_modes(P)[:3]:
        assert np.max(np.abs(K @ r)) <= 1e-9 * scale


def test_membrane_constant_strain_patch(oracle):
    """Uniform stretch eps_x with eps_y = 0 on a flat a x b rectangle: plane-stress sigma_x =
    E eps / (1 - nu^2), so each node of the edge x = a carries sigma_x h b / 2 and the edge
    x = 0 the opposite; sigma_y = nu sigma_x acts on the y edges."""
    a, b, eps = 6.0, 4.0, 1e-4
    P = np.array([[0, 0, 0], [a, 0, 0], [a, b, 0], [0, b, 0]], dtype=float)
    K = oracle.shell4_stiffness(E, NU, H, P)
    u = np.zeros(24)
    for i in range(4):
        u[6 * i] = eps * P[i, 0]
    f = K @ u
    sx = E * eps / (1 - NU * NU)
    fx = sx * H * b / 2.0
    fy = NU * sx * H * a / 2.0
    np.testing.assert_allclose(f[0::6], [-fx, fx, fx, -fx], rtol=1e-10)
    np.testing.assert_allclose(f[1::6], [-fy, -fy, fy, fy], rtol=1e-10)
    assert np.max(np.abs(f[2::6])) <= 1e-10 * fx


def test_slab_frame_transient_and_mass(oracle):
    slabs = {"E": E, "nu": NU, "h": H, "rho": 2400.0}
    case = W.rc_frame3d_case(stories=2, bays_x=2, bays_y=1, steps=30, element="forceBeamColumn3d", seed=61,
                             pga_g=0.3, slabs=slabs, bidirectional=True)
    m = M.Model(case)
    assert len(m.shells) == 4
    bare = M.Model(W.rc_frame3d_case(stories=2, bays_x=2, bays_y=1, steps=30, element="forceBeamColumn3d",
                                     seed=61, pga_g=0.3, bidirectional=True))
    # the slab's rho h area on each floor's translations (loader.mojo:2060-2100)
    extra = m.mass.reshape(-1, 6)[:, :3].sum() - bare.mass.reshape(-1, 6)[:, :3].sum()
    xs = [n["x"] for n in case["nodes"]]
    ys = [n["y"] for n in case["nodes"]]
    floor_area = (max(xs) - min(xs)) * (max(ys) - min(ys))
    assert extra == pytest.approx(3 * 2400.0 * H * floor_area * 2, rel=1e-12)
    d, e, it, rc, _ = oracle.run_transient(m, 30)
    assert rc == 0 and np.all(np.isfinite(d))
