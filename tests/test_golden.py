"""Golden fixtures (tests/golden, written by make_golden.py from the oracle): the oracle
reproduces them bit for bit; the GPU reproduces them within the parity tolerances."""
import json
from pathlib import Path

import numpy as np
import pytest

from strut_b200 import model as M
from tests.helpers import path_array, rel_err_of_peak

G = Path(__file__).resolve().parent / "golden"


def _load(name):
    return json.loads((G / name).read_text())


def test_oracle_material_paths_bitwise(oracle):
    for fx in _load("material_paths.json"):
        got = oracle.material_path(M.uniaxial_material(fx["material"]), np.array(fx["strains"]))
        assert np.array_equal(got, np.array(fx["stress_tangent"]))


def test_oracle_section_paths_bitwise(oracle):
    for fx in _load("section_paths.json"):
        case = fx["case"]
        mats, nm, fibs, nf = M.section_fibers(case["section"], case["materials"])
        got = oracle.section_path(mats, nm, fibs, nf, path_array(case))
        assert np.array_equal(got, np.array(fx["response"]))


def test_oracle_transient_bitwise(oracle):
    fx = _load("transient_2x1.json")
    m = M.Model(fx["case"])
    disp, ef, iters, rc, _ = oracle.run_transient(m, len(fx["iters"]))
    assert rc == 0
    assert np.array_equal(disp, np.array(fx["disp"]))
    assert np.array_equal(ef, np.array(fx["eforce"]))
    assert np.array_equal(iters, np.array(fx["iters"]))


@pytest.mark.gpu
def test_gpu_matches_golden(gpu_lib):
    for fx in _load("material_paths.json"):
        got = gpu_lib.material_path(M.uniaxial_material(fx["material"]), np.array(fx["strains"]))
        ref = np.array(fx["stress_tangent"])
        np.testing.assert_allclose(got, ref, rtol=1e-9, atol=1e-9 * np.abs(ref).max())
    for fx in _load("section_paths.json"):
        case = fx["case"]
        mats, nm, fibs, nf = M.section_fibers(case["section"], case["materials"])
        got = gpu_lib.section_path(mats, nm, fibs, nf, path_array(case))
        ref = np.array(fx["response"])
        assert np.all(np.abs(got - ref) <= 1e-9 * np.abs(ref).max(axis=0) + 1e-12)
    fx = _load("transient_2x1.json")
    m = M.Model(fx["case"])
    with gpu_lib.Analysis([m]) as an:
        an.run(len(fx["iters"]))
        disp, ef, iters = an.history(0)
    ref = np.array(fx["disp"])
    for j in range(ref.shape[1]):
        assert rel_err_of_peak(disp[:, j], ref[:, j]) <= 1e-7
    assert np.array_equal(iters, np.array(fx["iters"]))
