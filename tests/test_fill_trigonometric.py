"""fillTrigonometric (src/pencilDcmp.cpp:5685-5759): the reference's analytic
RHS, f = -4 pi^2 cos(2 pi z) at the cell centres of the box, which
src/main.cpp:115 passes to assignRhs.  The library's host function
(pp_fill_trigonometric_box, no GPU needed) is checked bit for bit against the
reference's own build (oracle/_ref/libppref.so) and against the formula; the
facade methods that have nothing to do at one rank (constructConnectivity,
graphCreate, readIn) and the writer IO (which needs a solved handle) are
checked too."""
import ctypes
import os

import numpy as np
import pytest

from pittpack_b200 import _lib
from pittpack_b200._lib import PittPackError
from pittpack_b200.poisson import PoissonGPU

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref", "libppref.so")
DP = ctypes.POINTER(ctypes.c_double)
CASES = [(8, 6, 5, (0, 1, 0, 1, 0, 1)), (12, 10, 9, (-1, 1, 0, 2, 0.5, 1.5)), (5, 4, 16, (0, 3, -2, 1, -1, 0.25))]


def _fill(nx, ny, nz, box):
    L = _lib.load()
    b = np.ascontiguousarray(box, dtype=np.float64)
    out = np.full(nx * ny * nz, np.nan)
    rc = L.pp_fill_trigonometric_box(nx, ny, nz, b.ctypes.data_as(DP), out.ctypes.data)
    assert rc == _lib.PP_SUCCESS
    return out.reshape(nz, ny, nx)


@pytest.mark.parametrize("nx,ny,nz,box", CASES)
def test_matches_the_formula(nx, ny, nz, box):
    f = _fill(nx, ny, nz, box)
    dz = (box[5] - box[4]) / nz
    z = box[4] + (np.arange(nz) + 0.5) * dz
    want = -4 * np.pi ** 2 * np.cos(2 * np.pi * z)
    assert np.allclose(f, want[:, None, None], rtol=1e-14, atol=1e-13)


@pytest.mark.skipif(not os.path.exists(REF), reason="reference build absent (make -C oracle)")
@pytest.mark.parametrize("nx,ny,nz,box", CASES)
def test_matches_the_reference_bit_for_bit(nx, ny, nz, box):
    L = ctypes.CDLL(REF)
    L.ppref_fill_trigonometric.argtypes = [ctypes.c_int] * 3 + [ctypes.c_char_p, DP, DP]
    L.ppref_fill_trigonometric.restype = ctypes.c_int
    b = np.ascontiguousarray(box, dtype=np.float64)
    ref = np.full(nx * ny * nz, np.nan)
    assert L.ppref_fill_trigonometric(nx, ny, nz, b"NNNNDD", b.ctypes.data_as(DP), ref.ctypes.data_as(DP)) == 0
    assert np.array_equal(_fill(nx, ny, nz, box).ravel(), ref)


def test_rejects_bad_arguments():
    L = _lib.load()
    out = np.zeros(8)
    good = np.array([0, 1, 0, 1, 0, 1.0])
    bad = np.array([0, 1, 1, 1, 0, 1.0])  # empty y extent
    assert L.pp_fill_trigonometric_box(2, 2, 2, bad.ctypes.data_as(DP), out.ctypes.data) == _lib.PP_INPUT_ARGS
    assert L.pp_fill_trigonometric_box(0, 2, 2, good.ctypes.data_as(DP), out.ctypes.data) == _lib.PP_INPUT_ARGS
    assert L.pp_fill_trigonometric_box(2, 2, 2, good.ctypes.data_as(DP), None) == _lib.PP_INPUT_ARGS
    assert L.pp_fill_trigonometric(None, out.ctypes.data) == _lib.PP_INVALID_HANDLE


def _solver(nx, ny, nz, box):
    M = PoissonGPU.__new__(PoissonGPU)
    M._L = _lib.load()
    M.nx, M.ny, M.nz = nx, ny, nz
    M._box = np.array(box, dtype=np.float64)
    M.bc = None
    M._h = None  # no device handle: this test runs without a GPU
    return M


def test_facade_follows_the_reference_driver():
    nx, ny, nz, box = CASES[1]
    M = _solver(nx, ny, nz, box)
    assert M.constructConnectivity() == _lib.PP_SUCCESS
    M.graphCreate()
    M.readIn()
    assert np.array_equal(M.fillTrigonometric(), _fill(nx, ny, nz, box))
    out = np.empty((nz, ny, nx))
    assert M.fillTrigonometric(out) is out
    with pytest.raises(PittPackError) as e:
        M.fillTrigonometric(np.empty(nx * ny * nz, dtype=np.float32))
    assert e.value.code == _lib.PP_INPUT_ARGS
    with pytest.raises(PittPackError) as e:
        M.IO(1, 2, 0)  # the writer needs a solved handle
    assert e.value.code == _lib.PP_INVALID_HANDLE
