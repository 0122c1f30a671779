"""The C-ABI library builds, loads without a GPU and exports every function the header
declares (no compute calls here)."""
import ctypes as C

import pytest
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
    assert lib.strut_gpu_abi_version() == 7
    assert isinstance(lib.strut_gpu_last_error(), bytes)


def test_struct_sizes_match_c_layout(tmp_path):
    """ctypes layouts against the C compiler's view of include/strut_cuda.h."""
    import shutil
    import subprocess
    from pathlib import Path

    names = ["StrutUniMaterial", "StrutFiber", "StrutBeamIntegration", "StrutFrameElement",
             "StrutFiberSection", "StrutExcitation", "StrutModelDesc", "StrutStepStats",
             "StrutTuning", "StrutSolverAttempt", "StrutSectionRecord"]
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    inc = Path(__file__).resolve().parents[1] / "include"
    src = tmp_path / "sizes.c"
    src.write_text('#include <stdio.h>\n#include "strut_cuda.h"\nint main(void) {\n' +
                   "".join(f'printf("%zu\\n", sizeof({n}));\n' for n in names) + "return 0;\n}\n")
    exe = tmp_path / "sizes"
    subprocess.check_call([cc, "-I", str(inc), str(src), "-o", str(exe)])
    sizes = [int(x) for x in subprocess.check_output([str(exe)]).split()]
    for n, sz in zip(names, sizes):
        assert C.sizeof(getattr(A, n)) == sz, n
