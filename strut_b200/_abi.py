"""ctypes mirror of ``include/strut_cuda.h`` (the C ABI of the sm_100a hot path).

The structures here are byte-for-byte the C structs; :mod:`strut_b200.model` fills them
from Strut's JSON schema and :mod:`strut_b200.runtime` hands them to ``libstrut_cuda.so``.
"""
from __future__ import annotations

import ctypes as C

MAX_INT_PTS = 10

STRUT_OK = 0
STRUT_NONCONVERGED = 1
STRUT_SINGULAR = 2
STRUT_NAN = 3
STRUT_BAD_ARG = 4
STRUT_CUDA_ERROR = 5
STRUT_UNSUPPORTED = 6
STRUT_ELEMENT_FAILED = 7

STATUS_NAMES = {
    STRUT_OK: "OK",
    STRUT_NONCONVERGED: "NONCONVERGED",
    STRUT_SINGULAR: "SINGULAR",
    STRUT_NAN: "NAN",
    STRUT_BAD_ARG: "BAD_ARG",
    STRUT_CUDA_ERROR: "CUDA_ERROR",
    STRUT_UNSUPPORTED: "UNSUPPORTED",
    STRUT_ELEMENT_FAILED: "ELEMENT_FAILED",
}

# UniMaterialTypeTag (tag_types.mojo:136-141)
MAT_ELASTIC = 0
MAT_STEEL01 = 1
MAT_CONCRETE01 = 2
MAT_STEEL02 = 3
MAT_CONCRETE02 = 4

# ElementTypeTag (tag_types.mojo:1-14)
ELEM_FORCE_BEAM_COLUMN_2D = 2
ELEM_DISP_BEAM_COLUMN_2D = 3
ELEM_FORCE_BEAM_COLUMN_3D = 11
ELEM_DISP_BEAM_COLUMN_3D = 12

GEOM_LINEAR = 0
GEOM_PDELTA = 1
GEOM_COROTATIONAL = 2

SYSTEM_BAND_GENERAL = 1
SYSTEM_BAND_SPD = 2

TEST_MAX_DISP_INCR = 0
TEST_NORM_DISP_INCR = 1
TEST_NORM_UNBALANCE = 2
TEST_ENERGY_INCR = 3
ALGORITHM_NEWTON, ALGORITHM_MODIFIED_NEWTON, ALGORITHM_MODIFIED_NEWTON_INITIAL = 0, 1, 2

_dp = C.POINTER(C.c_double)
_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int32)


class StrutUniMaterial(C.Structure):
    _fields_ = [("type", C.c_int32), ("reserved", C.c_int32), ("p", C.c_double * 11)]


class StrutFiber(C.Structure):
    _fields_ = [
        ("y", C.c_double),
        ("z", C.c_double),
        ("area", C.c_double),
        ("material", C.c_int32),
        ("reserved", C.c_int32),
    ]


class StrutFiberSection(C.Structure):
    _fields_ = [
        ("fiber_offset", C.c_int32),
        ("fiber_count", C.c_int32),
        ("dim", C.c_int32),
        ("reserved", C.c_int32),
        ("G", C.c_double),
        ("J", C.c_double),
    ]


class StrutBeamIntegration(C.Structure):
    _fields_ = [
        ("num_int_pts", C.c_int32),
        ("reserved", C.c_int32),
        ("xi", C.c_double * MAX_INT_PTS),
        ("w", C.c_double * MAX_INT_PTS),
    ]


class StrutFrameElement(C.Structure):
    _fields_ = [
        ("type", C.c_int32),
        ("node_i", C.c_int32),
        ("node_j", C.c_int32),
        ("section", C.c_int32),
        ("geom", C.c_int32),
        ("integration", C.c_int32),
        ("dof", C.c_int32 * 12),
        ("vecxz", C.c_double * 3),
        ("has_vecxz", C.c_int32),
        ("reserved", C.c_int32),
    ]


class StrutShellElement(C.Structure):
    _fields_ = [
        ("nodes", C.c_int32 * 4),
        ("dof", C.c_int32 * 24),
        ("E", C.c_double),
        ("nu", C.c_double),
        ("h", C.c_double),
    ]


class StrutExcitation(C.Structure):
    _fields_ = [
        ("direction", C.c_int32),
        ("count", C.c_int32),
        ("values", _dp),
        ("dt", C.c_double),
        ("factor", C.c_double),
        ("start_time", C.c_double),
        ("use_last", C.c_int32),
        ("reserved", C.c_int32),
    ]


MAX_ATTEMPTS = 4


class StrutSolverAttempt(C.Structure):
    _fields_ = [
        ("algorithm", C.c_int32),
        ("test_type", C.c_int32),
        ("max_iters", C.c_int32),
        ("reserved", C.c_int32),
        ("tol", C.c_double),
    ]


SECTION_FORCE = 0
SECTION_DEFORMATION = 1


class StrutSectionRecord(C.Structure):
    _fields_ = [("element", C.c_int32), ("section", C.c_int32), ("kind", C.c_int32), ("reserved", C.c_int32)]


class StrutModelDesc(C.Structure):
    _fields_ = [
        ("ndm", C.c_int32),
        ("ndf", C.c_int32),
        ("num_nodes", C.c_int32),
        ("num_dofs", C.c_int32),
        ("node_coords", _dp),
        ("num_materials", C.c_int32),
        ("num_fibers", C.c_int32),
        ("materials", C.POINTER(StrutUniMaterial)),
        ("fibers", C.POINTER(StrutFiber)),
        ("num_sections", C.c_int32),
        ("num_integrations", C.c_int32),
        ("sections", C.POINTER(StrutFiberSection)),
        ("integrations", C.POINTER(StrutBeamIntegration)),
        ("num_elements", C.c_int32),
        ("num_free", C.c_int32),
        ("elements", C.POINTER(StrutFrameElement)),
        ("free_index", _ip),
        ("mass", _dp),
        ("mass_rayleigh", _dp),
        ("f_const", _dp),
        ("alpha_m", C.c_double),
        ("beta_k", C.c_double),
        ("beta_k_init", C.c_double),
        ("beta_k_comm", C.c_double),
        ("dt", C.c_double),
        ("gamma", C.c_double),
        ("beta", C.c_double),
        ("tol", C.c_double),
        ("max_iters", C.c_int32),
        ("test_type", C.c_int32),
        ("system", C.c_int32),
        ("num_excitations", C.c_int32),
        ("excitation", StrutExcitation * 2),
        ("num_record_dofs", C.c_int32),
        ("num_record_elements", C.c_int32),
        ("record_dofs", _ip),
        ("record_elements", _ip),
        ("num_slaves", C.c_int32),
        ("algorithm", C.c_int32),
        ("slave_dof", _ip),
        ("slave_ptr", _ip),
        ("slave_master", _ip),
        ("slave_coef", _dp),
        ("num_shells", C.c_int32),
        ("reserved_shell", C.c_int32),
        ("shells", C.POINTER(StrutShellElement)),
        ("num_attempts", C.c_int32),
        ("reserved_attempts", C.c_int32),
        ("attempts", StrutSolverAttempt * MAX_ATTEMPTS),
        ("num_record_sections", C.c_int32),
        ("reserved_sections", C.c_int32),
        ("record_sections", C.POINTER(StrutSectionRecord)),
    ]


class StrutStepStats(C.Structure):
    _fields_ = [
        ("global_newton_iterations", C.c_int64),
        ("local_element_iterations", C.c_int64),
        ("section_evaluations", C.c_int64),
        ("fiber_updates", C.c_int64),
        ("factorizations", C.c_int64),
        ("steps_done", C.c_int32),
        ("failed_instance", C.c_int32),
        ("failed_step", C.c_int32),
        ("status", C.c_int32),
        ("fanned_out", C.c_int64),
    ]


class StrutTuning(C.Structure):
    _fields_ = [
        ("fan_out", C.c_int32),
        ("commit_team", C.c_int32),
        ("factor_ctas", C.c_int32),
        ("element_threads", C.c_int32),
        ("reserved", C.c_int32 * 4),
    ]


class StrutKernelProfile(C.Structure):
    _fields_ = [
        ("launches", C.c_int64 * 8),
        ("ms", C.c_double * 8),
        ("bytes", C.c_double * 8),
    ]


PROF_ELEMENT = 0
PROF_INSTANCE = 1
PROF_COMMIT = 2
PROF_PREDICTOR = 3
PROF_POST = 4
PROF_ELEMENT_CRITICAL = 5


# Every function the header declares, with its ctypes signature.  Used by the binding and by
# the test that checks the built library exports all of them.
EXPORTS = {
    "strut_gpu_abi_version": (C.c_int, []),
    "strut_gpu_get_section_history": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_double)]),
    "strut_gpu_last_error": (C.c_char_p, []),
    "strut_gpu_create": (
        C.c_int,
        [C.POINTER(StrutModelDesc), C.c_int32, C.c_int32, C.POINTER(C.c_void_p)],
    ),
    "strut_gpu_destroy": (C.c_int, [C.c_void_p]),
    "strut_gpu_num_instances": (C.c_int, [C.c_void_p]),
    "strut_gpu_run_steps": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(StrutStepStats)]),
    "strut_gpu_get_history": (C.c_int, [C.c_void_p, C.c_int32, _dp, _dp, _ip]),
    "strut_gpu_get_history_all": (C.c_int, [C.c_void_p, _dp, _dp, _ip]),
    "strut_gpu_get_state": (C.c_int, [C.c_void_p, C.c_int32, _dp, _dp, _dp]),
    "strut_gpu_instance_status": (C.c_int, [C.c_void_p, _ip]),
    "strut_gpu_set_profiling": (C.c_int, [C.c_void_p, C.c_int32]),
    "strut_gpu_get_profile": (C.c_int, [C.c_void_p, C.POINTER(StrutKernelProfile)]),
    "strut_gpu_stream": (C.c_void_p, [C.c_void_p]),
    "strut_gpu_set_tuning": (C.c_int, [C.c_void_p, C.c_void_p]),
    "strut_gpu_get_tuning": (C.c_int, [C.c_void_p, C.c_void_p]),
    "strut_gpu_set_wait_limit": (C.c_int, [C.c_void_p, C.c_int32]),
    "strut_gpu_state_determination": (C.c_int, [C.c_void_p, _dp, _dp, _dp]),
    "strut_gpu_band_info": (C.c_int, [C.c_void_p, C.c_int32, _ip, _ip]),
    "strut_gpu_factor_solve": (C.c_int, [C.c_void_p, _dp, _dp]),
    "strut_gpu_commit": (C.c_int, [C.c_void_p]),
    "strut_gpu_revert": (C.c_int, [C.c_void_p]),
    "strut_gpu_section_path": (
        C.c_int,
        [C.POINTER(StrutUniMaterial), C.c_int32, C.POINTER(StrutFiber), C.c_int32, _dp,
         C.c_int32, _dp],
    ),
    "strut_gpu_section3d_path": (
        C.c_int,
        [C.POINTER(StrutUniMaterial), C.c_int32, C.POINTER(StrutFiber), C.c_int32, _dp,
         C.c_int32, _dp],
    ),
    "strut_gpu_material_path": (
        C.c_int, [C.POINTER(StrutUniMaterial), _dp, C.c_int32, _dp]
    ),
    "strut_gpu_section_batch_create": (
        C.c_int,
        [C.POINTER(StrutUniMaterial), C.c_int32, C.POINTER(StrutFiber), C.c_int32, C.c_int32,
         C.POINTER(C.c_void_p)],
    ),
    "strut_gpu_section_batch_destroy": (C.c_int, [C.c_void_p]),
    "strut_gpu_section_eval_batch": (
        C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p]
    ),
    "strut_gpu_section_batch_state": (C.c_int, [C.c_void_p, C.c_int32, _dp, _ip]),
    "strut_gpu_mlp_create": (C.c_int, [C.c_int32, C.c_int32, C.POINTER(C.c_void_p)]),
    "strut_gpu_mlp_destroy": (C.c_int, [C.c_void_p]),
    "strut_gpu_mlp_param_count": (C.c_int32, [C.c_void_p]),
    "strut_gpu_mlp_set_params": (C.c_int, [C.c_void_p, _fp]),
    "strut_gpu_mlp_get_params": (C.c_int, [C.c_void_p, _fp]),
    "strut_gpu_mlp_forward": (C.c_int, [C.c_void_p, _fp, C.c_int32, _fp]),
    "strut_gpu_mlp_loss_grad": (C.c_int, [C.c_void_p, _fp, _fp, C.c_int32, _fp, _fp]),
    "strut_gpu_set_predictor": (C.c_int, [C.c_void_p, C.c_void_p, _fp, _fp, _fp]),
    "strut_gpu_predictor_nodes": (C.c_int32, [C.c_void_p]),
    "strut_gpu_predictor_stats": (C.c_int, [C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    "strut_gpu_predictor_features": (C.c_int, [C.c_void_p, _fp]),
    "strut_gpu_band_solve_noalloc": (
        C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    ),
    "strut_gpu_mlp_train": (
        C.c_int, [C.c_void_p, _fp, _fp, C.c_int32, C.c_int32, C.c_int32, C.c_float, C.c_uint64, _fp]
    ),
}
