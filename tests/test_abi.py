"""The C-ABI library builds, loads without a GPU and exports every function the header
declares (no compute calls here)."""
import ctypes as C
import re
from pathlib import Path

from strut_b200 import _abi as A

ROOT = Path(__file__).resolve().parents[1]


def header_functions():
    text = (ROOT / "include" / "strut_cuda.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(strut_gpu_\w+)\s*\(", text)))


def test_header_and_binding_agree():
    assert header_functions() == sorted(A.EXPORTS)


def test_library_exports_every_header_symbol(gpu_lib):
    lib = C.CDLL(str(gpu_lib.LIB_PATH))
    for name in header_functions():
        assert hasattr(lib, name), name


def test_abi_version_and_error_text_without_gpu(gpu_lib):
    lib = gpu_lib.lib()
    assert lib.strut_gpu_abi_version() == 3
    assert isinstance(lib.strut_gpu_last_error(), bytes)


def test_struct_sizes_match_c_layout():
    # sizes from the C compiler's view of include/strut_cuda.h (x86-64 / aarch64 LP64)
    assert C.sizeof(A.StrutUniMaterial) == 96
    assert C.sizeof(A.StrutFiber) == 32
    assert C.sizeof(A.StrutBeamIntegration) == 168
    assert C.sizeof(A.StrutFrameElement) == 104
    assert C.sizeof(A.StrutFiberSection) == 32
    assert C.sizeof(A.StrutExcitation) == 48
    assert C.sizeof(A.StrutModelDesc) == 320
    assert C.sizeof(A.StrutStepStats) == 56
