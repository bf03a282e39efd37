"""The reference-side binding (include/binding/poissonB200Binding.hpp: a
PoissonCPU subclass whose solveOnB200() hands P to the B200 library) compiled
against the reference's own headers, linked with its objects and
libpittpack_b200.so (oracle/Makefile target _ref/binding_check, driver
oracle/binding_driver.cpp) and run in the order of src/main.cpp:73-134.

The executable is built where the PittPack sources are (the build step) and
runs wherever the tree is copied.  Without a GPU the binding must come back
with the library's GPU_INIT_FAILURE status (no crash); on a GPU it must solve
and agree with the reference's own pittPack() on the same input to 1e-12
relative L2."""
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "oracle", "_ref", "binding_check")
LIB = os.path.join(ROOT, "pittpack_b200", "libpittpack_b200.so")


def _run():
    if not (os.path.exists(EXE) and os.path.exists(LIB)):
        pytest.skip("binding check not built (make -C oracle PITTPACK_SRC=<PittPack tree>)")
    r = subprocess.run([EXE], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    line = [s for s in r.stdout.splitlines() if s.startswith("BINDING")][-1]
    return int(re.search(r"rc=(-?\d+)", line).group(1)), float(re.search(r"rel=(\S+)", line).group(1)), line


def test_binding_without_gpu_returns_status():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present: test_binding_matches_reference_on_gpu covers this machine")
    rc, _, line = _run()
    assert rc == 1, line  # PP_GPU_INIT_FAILURE


@pytest.mark.gpu
def test_binding_matches_reference_on_gpu():
    rc, rel, line = _run()
    assert rc == 0, line
    assert rel <= 1e-12, line
