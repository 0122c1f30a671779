"""ctypes binding of the CPU oracle (liboracle.so) -- test infrastructure only.

Imported by tests/, by ``__graft_entry__.smoke()`` as the checker and by ``bench.py``'s CPU
baseline leg.  The product package never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

from strut_b200 import _abi as A

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle.so"
LIB_PATH_FMA = HERE / "liboracle_fma.so"  # the same oracle with contracted multiply-adds

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


def build(force: bool = False, fma: bool = False) -> Path:
    path = LIB_PATH_FMA if fma else LIB_PATH
    srcs = list(HERE.glob("*.c")) + list(HERE.glob("*.h")) + [HERE.parent / "include" / "strut_cuda.h"]
    if force or not path.exists() or any(p.stat().st_mtime > path.stat().st_mtime for p in srcs):
        subprocess.check_call(["make", "-s", "-C", str(HERE), path.name])
    return path


_lib = None
_fma = False


def use_fma(on: bool):
    """Selects the oracle build for the following calls: separately rounded multiplies and adds
    (the default) or contracted multiply-adds.  Together with the SIMD width this gives the
    reference's algorithm under several roundings."""
    global _lib, _fma
    if bool(on) != _fma:
        _fma = bool(on)
        _lib = None


def lib():
    global _lib
    if _lib is None:
        path = build(fma=_fma)  # rebuilt when a source is newer than the library
        L = C.CDLL(str(path))
        L.oracle_set_simd_width.argtypes = [C.c_int]
        L.oracle_subdivisions.restype = C.c_long
        L.oracle_dense_fallbacks.restype = C.c_long
        L.oracle_get_simd_width.restype = C.c_int
        L.oracle_material_path.argtypes = [C.POINTER(A.StrutUniMaterial), _dp, C.c_int, _dp]
        L.oracle_section_path.argtypes = [C.POINTER(A.StrutUniMaterial), C.c_int,
                                          C.POINTER(A.StrutFiber), C.c_int, _dp, C.c_int, _dp]
        L.oracle_section_batch_path.argtypes = [C.POINTER(A.StrutUniMaterial), C.c_int,
                                                C.POINTER(A.StrutFiber), C.c_int, C.c_int, _dp,
                                                C.c_int, _dp]
        L.oracle_section3d_path.argtypes = [C.POINTER(A.StrutUniMaterial), C.c_int,
                                            C.POINTER(A.StrutFiber), C.c_int, _dp, C.c_int, _dp]
        L.oracle_element_state.argtypes = [C.POINTER(A.StrutModelDesc), C.c_int, _dp, _dp, _dp]
        L.oracle_run_transient.argtypes = [C.POINTER(A.StrutModelDesc), C.c_int, _dp, _dp, _ip, _ip]
        L.oracle_run_transient_sections.argtypes = [C.POINTER(A.StrutModelDesc), C.c_int, _dp, _dp, _ip,
                                                    _ip, _dp]
        L.oracle_state_determination.argtypes = [C.POINTER(A.StrutModelDesc), _dp, _dp, _dp, _ip]
        L.oracle_run_transient_batch.argtypes = [C.POINTER(A.StrutModelDesc), C.c_int, C.c_int,
                                                 C.c_int, _ip, _ip, _ip, _ip]
        _lib = L
    return _lib


def _d(a):
    return a.ctypes.data_as(_dp)


def subdivisions() -> int:
    """forceBeamColumn2d subdivision passes in which every scheme failed, since load."""
    return int(lib().oracle_subdivisions())


def set_simd_width(w: int):
    lib().oracle_set_simd_width(int(w))


def material_path(mat: A.StrutUniMaterial, strains) -> np.ndarray:
    s = np.ascontiguousarray(strains, dtype=np.float64)
    out = np.zeros((len(s), 2))
    lib().oracle_material_path(C.byref(mat), _d(s), len(s), _d(out))
    return out


def section_path(mats, nmat, fibs, nfib, eps0_kappa) -> np.ndarray:
    ek = np.ascontiguousarray(eps0_kappa, dtype=np.float64).reshape(-1, 2)
    out = np.zeros((len(ek), 5))
    rc = lib().oracle_section_path(mats, nmat, fibs, nfib, _d(ek), len(ek), _d(out))
    if rc != 0:
        raise RuntimeError(f"oracle_section_path failed: {A.STATUS_NAMES.get(rc, rc)}")
    return out


def shell4_stiffness(E: float, nu: float, h: float, xyz) -> np.ndarray:
    """24 x 24 global stiffness of a ShellMITC4 on an ElasticMembranePlateSection; xyz (4, 3)."""
    L = lib()
    P = np.ascontiguousarray(xyz, dtype=np.float64).reshape(4, 3)
    x, y, z = (np.ascontiguousarray(P[:, k]) for k in range(3))
    K = np.zeros(576)
    dp = C.POINTER(C.c_double)
    fn = L.oracle_shell4_stiffness
    fn.restype = C.c_int
    fn.argtypes = [C.c_double, C.c_double, C.c_double, dp, dp, dp, dp]
    rc = fn(E, nu, h, x.ctypes.data_as(dp), y.ctypes.data_as(dp), z.ctypes.data_as(dp), K.ctypes.data_as(dp))
    if rc != 0:
        raise RuntimeError("oracle_shell4_stiffness failed")
    return K.reshape(24, 24)


def section3d_path(mats, nmat, fibs, nfib, path) -> np.ndarray:
    """path: (npts, 3) of (eps0, kappa_y, kappa_z) -> (npts, 9) of N, My, Mz, k11, k12, k13,
    k22, k23, k33."""
    p = np.ascontiguousarray(path, dtype=np.float64).reshape(-1, 3)
    out = np.zeros((len(p), 9))
    rc = lib().oracle_section3d_path(mats, nmat, fibs, nfib, _d(p), len(p), _d(out))
    if rc != 0:
        raise RuntimeError(f"oracle_section3d_path failed: {A.STATUS_NAMES.get(rc, rc)}")
    return out


def section_batch_path(mats, nmat, fibs, nfib, eps0_kappa) -> np.ndarray:
    """eps0_kappa: (npts, n_inst, 2) -> (npts, n_inst, 5)"""
    ek = np.ascontiguousarray(eps0_kappa, dtype=np.float64)
    npts, n_inst = ek.shape[0], ek.shape[1]
    out = np.zeros((npts, n_inst, 5))
    rc = lib().oracle_section_batch_path(mats, nmat, fibs, nfib, n_inst, _d(ek), npts, _d(out))
    if rc != 0:
        raise RuntimeError(f"oracle_section_batch_path failed: {A.STATUS_NAMES.get(rc, rc)}")
    return out


def run_transient(model, steps: int, sections: bool = False):
    """(disp (steps, nrec), eforce (steps, nrece, 2*ndf), iters (steps,), rc, failed_step), and
    with sections the section recorders' values (steps, nsec, 2 in 2D / 4 in 3D) appended."""
    d = model.desc()
    nrec = d.num_record_dofs
    nrece = d.num_record_elements
    disp = np.zeros((steps, max(nrec, 1)))
    ef = np.zeros((steps, max(nrece, 1), 2 * model.ndf))
    iters = np.zeros(steps, dtype=np.int32)
    failed = C.c_int(-1)
    if not sections:
        rc = lib().oracle_run_transient(C.byref(d), steps, _d(disp), _d(ef),
                                        iters.ctypes.data_as(_ip), C.byref(failed))
        return disp[:, :nrec], ef[:, :nrece], iters, rc, failed.value
    nsec = d.num_record_sections
    sec = np.zeros((steps, max(nsec, 1), 2 if model.ndf == 3 else 4))
    rc = lib().oracle_run_transient_sections(C.byref(d), steps, _d(disp), _d(ef),
                                             iters.ctypes.data_as(_ip), C.byref(failed), _d(sec))
    return disp[:, :nrec], ef[:, :nrece], iters, rc, failed.value, sec[:, :nsec]


def state_determination(model, u_free):
    d = model.desc()
    u = np.ascontiguousarray(u_free, dtype=np.float64)
    f = np.zeros(model.num_free)
    bw = C.c_int(0)
    # first call with band_out NULL to learn the band width
    rc = lib().oracle_state_determination(C.byref(d), _d(u), _d(f), None, C.byref(bw))
    if rc != 0:
        raise RuntimeError(f"oracle_state_determination failed: {A.STATUS_NAMES.get(rc, rc)}")
    rw = bw.value + 1 if model.system == A.SYSTEM_BAND_SPD else 2 * bw.value + 1
    band = np.zeros((model.num_free, rw))
    rc = lib().oracle_state_determination(C.byref(d), _d(u), _d(f), _d(band), C.byref(bw))
    return f, band, bw.value


def element_state(model, elem: int, u_elem):
    """(k (nd, nd), f (nd,)) of one element at element displacements u_elem."""
    nd = 2 * model.ndf
    d = model.desc()
    u = np.ascontiguousarray(u_elem, dtype=np.float64)
    k = np.zeros((nd, nd))
    f = np.zeros(nd)
    rc = lib().oracle_element_state(C.byref(d), int(elem), _d(u), _d(k), _d(f))
    if rc != 0:
        raise RuntimeError(f"oracle_element_state failed: {A.STATUS_NAMES.get(rc, rc)}")
    return k, f


def run_batch(models, steps: int, nthreads: int, detail: bool = False):
    """Runs every model for `steps` steps over `nthreads` host threads.  Returns
    (first failure status or 0, total Newton iterations, per-record status array), plus, with
    detail, the per-record failing step (-1: none) and Newton iteration arrays."""
    descs = (A.StrutModelDesc * len(models))()
    for i, m in enumerate(models):
        descs[i] = m.desc()
    tot = C.c_int(0)
    st = np.zeros(len(models), dtype=np.int32)
    fs = np.zeros(len(models), dtype=np.int32)
    it = np.zeros(len(models), dtype=np.int32)
    rc = lib().oracle_run_transient_batch(descs, len(models), steps, nthreads, C.byref(tot),
                                          st.ctypes.data_as(_ip), fs.ctypes.data_as(_ip),
                                          it.ctypes.data_as(_ip))
    if detail:
        return rc, tot.value, st, fs, it
    return rc, tot.value, st
