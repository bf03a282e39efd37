"""CPU-side checks of the C ABI library: it loads, exports every entry point
include/*.h declares, and rejects bad arguments without a GPU."""
import ctypes
import glob
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        txt = open(h).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?\w+\*?\s+\**(pp_\w+)\s*\(", txt, flags=re.M):
            names.add(m.group(1))
    return sorted(names)


@pytest.fixture(scope="module")
def lib():
    from pittpack_b200 import build

    build.build()
    return ctypes.CDLL(build.LIB)


def test_header_declares_entry_points():
    names = _declared()
    for n in ("pp_create", "pp_assign_boundary", "pp_assign_rhs", "pp_solve", "pp_get_solution", "pp_destroy"):
        assert n in names


def test_library_exports_every_declared_symbol(lib):
    missing = [n for n in _declared() if not hasattr(lib, n)]
    assert not missing, missing


def test_status_strings_and_null_arguments(lib):
    from pittpack_b200 import _lib

    L = _lib.load()
    assert L.pp_result_string(0) == b"SUCCESS"
    assert b"INPUT_ARGS" in L.pp_result_string(19)
    # null handle / null pointers are rejected before any CUDA call
    assert L.pp_solve(None) == _lib.PP_INVALID_HANDLE
    assert L.pp_destroy(None) == _lib.PP_INVALID_HANDLE
    assert L.pp_create(8, 8, 8, None) == _lib.PP_INPUT_ARGS
    h = ctypes.c_void_p()
    assert L.pp_create(1, 8, 8, ctypes.byref(h)) == _lib.PP_INPUT_ARGS
    assert L.pp_create(8, 8, 2, ctypes.byref(h)) == _lib.PP_INPUT_ARGS
    o = _lib.Options()
    assert L.pp_default_options(ctypes.byref(o)) == 0
    assert o.compat_zero_mode == 1 and o.dirichlet_lift == 1 and o.precision == 0 and o.zero_mean == 0


def test_no_gpu_here_reports_init_failure(lib):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from pittpack_b200 import _lib

    h = ctypes.c_void_p()
    assert _lib.load().pp_create(8, 8, 8, ctypes.byref(h)) == 1  # GPU_INIT_FAILURE


@pytest.mark.skipif(not __import__("shutil").which("gcc"), reason="no C compiler")
def test_header_is_plain_c_and_links(tmp_path):
    """The ABI is C: a C99 translation unit that includes the header and
    takes the address of every declared entry point compiles, with no CUDA
    headers, and links against the library."""
    import subprocess

    names = _declared()
    src = tmp_path / "abi.c"
    src.write_text('#include "pittpack_b200.h"\n#include <stdio.h>\nint main(void) {\n'
                   "    const void* fns[] = {\n" + ",\n".join(f"        (const void*){n}" for n in names) + "\n    };\n"
                   '    printf("%d %s\\n", (int)(sizeof fns / sizeof fns[0]), pp_result_string(PP_INPUT_ARGS));\n'
                   "    return 0;\n}\n")
    libdir = os.path.join(ROOT, "pittpack_b200")
    exe = tmp_path / "abi"
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), str(src), "-L", libdir,
                    "-lpittpack_b200", f"-Wl,-rpath,{libdir}", "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split(maxsplit=1)
    assert int(out[0]) == len(names) and out[1].startswith("INPUT_ARGS")
