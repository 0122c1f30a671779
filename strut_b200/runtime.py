"""Python host binding of ``libstrut_cuda.so`` (the sm_100a hot path) through its C ABI.

The library is built in-tree (``python -m strut_b200.build``).  There is no CPU fallback:
if the library or a GPU is missing, every entry point raises.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from . import _abi as A

LIB_PATH = Path(__file__).resolve().parent / "libstrut_cuda.so"

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)

_lib = None


class StrutError(RuntimeError):
    def __init__(self, code: int, where: str, detail: str = ""):
        self.code = code
        name = A.STATUS_NAMES.get(code, str(code))
        super().__init__(f"{where}: {name}" + (f" ({detail})" if detail else ""))


def lib():
    """The loaded library (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(
                f"{LIB_PATH.name} is not built; run `python -m strut_b200.build` (nvcc, sm_100a)"
            )
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in A.EXPORTS.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _check(rc: int, where: str):
    if rc != A.STRUT_OK:
        detail = lib().strut_gpu_last_error().decode(errors="replace")
        raise StrutError(rc, where, detail)


def _d(a: np.ndarray):
    return a.ctypes.data_as(_dp)


class Analysis:
    """A batch of transient analyses on one GPU (one handle).

    tuned: start from the launch shapes the autotuner recorded for this batch's workload class
    (strut_b200/tuned_shapes.json), if it has an entry; the library's defaults otherwise.  Every
    launch shape gives the same results bit for bit; set_tuning overrides them."""

    def __init__(self, models, device: int = -1, tuned: bool = True):
        self.models = list(models)
        n = len(self.models)
        self._descs = (A.StrutModelDesc * n)()
        for i, m in enumerate(self.models):
            self._descs[i] = m.desc()
        h = C.c_void_p()
        _check(lib().strut_gpu_create(self._descs, n, device, C.byref(h)), "strut_gpu_create")
        self.h = h
        self.steps_done = 0
        self.tuned = None
        if tuned:
            from . import autotune

            self.tuned = autotune.apply(self)

    def close(self):
        if getattr(self, "h", None):
            lib().strut_gpu_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def run(self, n_steps: int, check: bool = True) -> A.StrutStepStats:
        st = A.StrutStepStats()
        rc = lib().strut_gpu_run_steps(self.h, int(n_steps), C.byref(st))
        self.steps_done += st.steps_done
        if check:
            _check(rc, "strut_gpu_run_steps")
        self.last_status = rc
        return st

    def set_tuning(self, fan_out=None, commit_team=None, factor_ctas=None, element_threads=None):
        """Launch-shape choices (strut_gpu_set_tuning); None keeps the current value.  Every
        choice gives the same results bit for bit."""
        t = self.tuning()
        for name, v in (("fan_out", fan_out), ("commit_team", commit_team), ("factor_ctas", factor_ctas),
                        ("element_threads", element_threads)):
            if v is not None:
                setattr(t, name, int(v))
        _check(lib().strut_gpu_set_tuning(self.h, C.byref(t)), "strut_gpu_set_tuning")

    def tuning(self) -> A.StrutTuning:
        t = A.StrutTuning()
        _check(lib().strut_gpu_get_tuning(self.h, C.byref(t)), "strut_gpu_get_tuning")
        return t

    def history(self, instance: int = 0):
        m = self.models[instance]
        S = self.steps_done
        disp = np.zeros((S, max(len(m.record_dofs), 1)))
        ef = np.zeros((S, max(len(m.record_elements), 1), 2 * m.ndf))
        it = np.zeros(S, dtype=np.int32)
        _check(
            lib().strut_gpu_get_history(self.h, instance, _d(disp), _d(ef), it.ctypes.data_as(_ip)),
            "strut_gpu_get_history",
        )
        return disp[:, : len(m.record_dofs)], ef[:, : len(m.record_elements)], it

    def section_history(self, instance: int = 0) -> np.ndarray:
        """Section recorder values of one instance: steps x num_record_sections x (2 in 2D, 4
        in 3D)."""
        m = self.models[instance]
        w = 2 if m.ndf == 3 else 4
        out = np.zeros((self.steps_done, max(m.num_record_sections, 1), w))
        _check(lib().strut_gpu_get_section_history(self.h, instance, _d(out)), "strut_gpu_get_section_history")
        return out[:, : m.num_record_sections]

    def history_all(self):
        S = self.steps_done
        nd = sum(len(m.record_dofs) for m in self.models)
        ne = sum(len(m.record_elements) * 2 * m.ndf for m in self.models)
        disp = np.zeros(max(S * nd, 1))
        ef = np.zeros(max(S * ne, 1))
        it = np.zeros(max(S * len(self.models), 1), dtype=np.int32)
        _check(
            lib().strut_gpu_get_history_all(self.h, _d(disp), _d(ef), it.ctypes.data_as(_ip)),
            "strut_gpu_get_history_all",
        )
        return disp, ef, it

    def instance_status(self):
        st = np.zeros(len(self.models), dtype=np.int32)
        _check(lib().strut_gpu_instance_status(self.h, st.ctypes.data_as(_ip)), "strut_gpu_instance_status")
        return st

    def state(self, instance: int = 0):
        n = self.models[instance].num_free
        u, v, a = np.zeros(n), np.zeros(n), np.zeros(n)
        _check(lib().strut_gpu_get_state(self.h, instance, _d(u), _d(v), _d(a)), "strut_gpu_get_state")
        return u, v, a

    def band_info(self, instance: int = 0):
        bw, rw = C.c_int32(), C.c_int32()
        _check(lib().strut_gpu_band_info(self.h, instance, C.byref(bw), C.byref(rw)), "strut_gpu_band_info")
        return bw.value, rw.value

    def state_determination(self, u_free_list):
        u = np.ascontiguousarray(np.concatenate([np.asarray(x, dtype=np.float64) for x in u_free_list]))
        f = np.zeros_like(u)
        sizes = []
        for i, m in enumerate(self.models):
            _bw, rw = self.band_info(i)
            sizes.append(m.num_free * rw)
        band = np.zeros(sum(sizes))
        _check(lib().strut_gpu_state_determination(self.h, _d(u), _d(f), _d(band)),
               "strut_gpu_state_determination")
        out = []
        fo, bo = 0, 0
        for i, m in enumerate(self.models):
            _bw, rw = self.band_info(i)
            n = m.num_free
            out.append((f[fo:fo + n].copy(), band[bo:bo + n * rw].reshape(n, rw).copy()))
            fo += n
            bo += n * rw
        return out

    def factor_solve(self, rhs_list):
        r = np.ascontiguousarray(np.concatenate([np.asarray(x, dtype=np.float64) for x in rhs_list]))
        du = np.zeros_like(r)
        _check(lib().strut_gpu_factor_solve(self.h, _d(r), _d(du)), "strut_gpu_factor_solve")
        out, o = [], 0
        for m in self.models:
            out.append(du[o:o + m.num_free].copy())
            o += m.num_free
        return out

    def commit(self):
        _check(lib().strut_gpu_commit(self.h), "strut_gpu_commit")


def material_path(mat: A.StrutUniMaterial, strains) -> np.ndarray:
    s = np.ascontiguousarray(strains, dtype=np.float64)
    out = np.zeros((len(s), 2))
    _check(lib().strut_gpu_material_path(C.byref(mat), _d(s), len(s), _d(out)), "strut_gpu_material_path")
    return out


def section_path(mats, nmat, fibs, nfib, eps0_kappa) -> np.ndarray:
    ek = np.ascontiguousarray(eps0_kappa, dtype=np.float64).reshape(-1, 2)
    out = np.zeros((len(ek), 5))
    _check(lib().strut_gpu_section_path(mats, nmat, fibs, nfib, _d(ek), len(ek), _d(out)),
           "strut_gpu_section_path")
    return out


def section3d_path(mats, nmat, fibs, nfib, path) -> np.ndarray:
    """FiberSection3d along (eps0, kappa_y, kappa_z) points -> (n, 9) responses."""
    p = np.ascontiguousarray(path, dtype=np.float64).reshape(-1, 3)
    out = np.zeros((len(p), 9))
    _check(lib().strut_gpu_section3d_path(mats, nmat, fibs, nfib, _d(p), len(p), _d(out)),
           "strut_gpu_section3d_path")
    return out


class SectionBatch:
    """n_inst independent histories of one FiberSection2d (device-resident)."""

    def __init__(self, mats, nmat, fibs, nfib, n_inst: int):
        b = C.c_void_p()
        _check(lib().strut_gpu_section_batch_create(mats, nmat, fibs, nfib, n_inst, C.byref(b)),
               "strut_gpu_section_batch_create")
        self.b = b
        self.n_inst = n_inst

    def eval(self, eps0_kappa_dev_ptr: int, resp_dev_ptr: int, commit: bool = True, stream: int = 0):
        _check(lib().strut_gpu_section_eval_batch(self.b, C.c_void_p(eps0_kappa_dev_ptr),
                                                  C.c_void_p(resp_dev_ptr), 1 if commit else 0,
                                                  C.c_void_p(stream)),
               "strut_gpu_section_eval_batch")

    def fiber_state(self, instance: int) -> np.ndarray:
        n = C.c_int32()
        _check(lib().strut_gpu_section_batch_state(self.b, instance, None, C.byref(n)), "state")
        out = np.zeros((n.value, 16))
        _check(lib().strut_gpu_section_batch_state(self.b, instance, _d(out), C.byref(n)), "state")
        return out

    def close(self):
        if getattr(self, "b", None):
            lib().strut_gpu_section_batch_destroy(self.b)
            self.b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_fp = C.POINTER(C.c_float)


class Mlp:
    """The learned predictor's per-node network on the GPU (strut_gpu_mlp_*)."""

    H = 128

    def __init__(self, n_in: int, n_out: int):
        m = C.c_void_p()
        _check(lib().strut_gpu_mlp_create(n_in, n_out, C.byref(m)), "strut_gpu_mlp_create")
        self.m = m
        self.n_in, self.n_out = n_in, n_out

    def n_params(self) -> int:
        return int(lib().strut_gpu_mlp_param_count(self.m))

    @staticmethod
    def pack(p: dict) -> np.ndarray:
        return np.concatenate([np.asarray(p[k], dtype=np.float32).reshape(-1)
                               for k in ("W1", "b1", "W2", "b2", "W3", "b3")])

    def unpack(self, flat: np.ndarray) -> dict:
        shapes = (("W1", (self.n_in, self.H)), ("b1", (self.H,)), ("W2", (self.H, self.H)), ("b2", (self.H,)),
                  ("W3", (self.H, self.n_out)), ("b3", (self.n_out,)))
        out, o = {}, 0
        for k, sh in shapes:
            n = int(np.prod(sh))
            out[k] = flat[o:o + n].reshape(sh).copy()
            o += n
        return out

    def set_params(self, p: dict):
        flat = np.ascontiguousarray(self.pack(p))
        assert flat.size == self.n_params()
        _check(lib().strut_gpu_mlp_set_params(self.m, flat.ctypes.data_as(_fp)), "strut_gpu_mlp_set_params")

    def get_params(self) -> dict:
        flat = np.zeros(self.n_params(), dtype=np.float32)
        _check(lib().strut_gpu_mlp_get_params(self.m, flat.ctypes.data_as(_fp)), "strut_gpu_mlp_get_params")
        return self.unpack(flat)

    def forward(self, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float32)
        y = np.zeros((x.shape[0], self.n_out), dtype=np.float32)
        _check(lib().strut_gpu_mlp_forward(self.m, x.ctypes.data_as(_fp), x.shape[0], y.ctypes.data_as(_fp)),
               "strut_gpu_mlp_forward")
        return y

    def loss_grad(self, x: np.ndarray, t: np.ndarray):
        x = np.ascontiguousarray(x, dtype=np.float32)
        t = np.ascontiguousarray(t, dtype=np.float32)
        loss = C.c_float()
        g = np.zeros(self.n_params(), dtype=np.float32)
        _check(lib().strut_gpu_mlp_loss_grad(self.m, x.ctypes.data_as(_fp), t.ctypes.data_as(_fp), x.shape[0],
                                             C.byref(loss), g.ctypes.data_as(_fp)), "strut_gpu_mlp_loss_grad")
        return float(loss.value), self.unpack(g)

    def train(self, x: np.ndarray, t: np.ndarray, epochs: int, batch: int = 4096, lr: float = 1e-3,
              seed: int = 0) -> float:
        x = np.ascontiguousarray(x, dtype=np.float32)
        t = np.ascontiguousarray(t, dtype=np.float32)
        loss = C.c_float()
        _check(lib().strut_gpu_mlp_train(self.m, x.ctypes.data_as(_fp), t.ctypes.data_as(_fp), x.shape[0], epochs,
                                          batch, lr, seed, C.byref(loss)), "strut_gpu_mlp_train")
        return float(loss.value)

    def close(self):
        if getattr(self, "m", None):
            lib().strut_gpu_mlp_destroy(self.m)
            self.m = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
