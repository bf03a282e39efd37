"""Argument checks of the Python facade that run before any call reaches the
GPU: wrong sizes, dtypes and face numbers raise PittPackError with the
reference's INPUT_ARGS code (src/include/params.h:86-114), or ValueError for
the server's host buffers.  The objects are made without a device handle,
so these run on the CPU."""
import numpy as np
import pytest

from pittpack_b200 import _lib
from pittpack_b200._lib import PittPackError
from pittpack_b200.batch import Server
from pittpack_b200.poisson import PoissonGPU


def _solver(nx=6, ny=5, nz=4):
    M = PoissonGPU.__new__(PoissonGPU)
    M._L = _lib.load()
    M.nx, M.ny, M.nz = nx, ny, nz
    M._box = np.array([0.0, 1, 0, 1, 0, 1])
    M.bc = None
    return M


def _input_args(fn, *a):
    with pytest.raises(PittPackError) as e:
        fn(*a)
    assert e.value.code == _lib.PP_INPUT_ARGS


def test_boundary_and_box_sizes():
    M = _solver()
    _input_args(M.assignBoundary, "NNDD")
    _input_args(M.assignBoundary, "NNDDDDD")
    _input_args(M.setBox, [0, 1, 0, 1])


def test_face_values_shape_and_face_number():
    M = _solver(6, 5, 4)
    _input_args(M.setFaceValues, 6, np.zeros((5, 4)))
    _input_args(M.setFaceValues, -1, np.zeros((5, 4)))
    _input_args(M.setFaceValues, 0, np.zeros((4, 6)))   # x face: (nz, ny) = 20 values
    _input_args(M.setFaceValues, 2, np.zeros((4, 5)))   # y face: (nz, nx) = 24 values
    _input_args(M.setFaceValues, 4, np.zeros((4, 6)))   # z face: (ny, nx) = 30 values


def test_rhs_and_solution_buffers():
    M = _solver(6, 5, 4)
    n = 6 * 5 * 4
    _input_args(M.assignRhs, np.zeros(n - 1))
    _input_args(M.assignRhsComplex, np.zeros(n + 1, dtype=np.complex128))
    _input_args(M.assignRhsAsync, np.zeros(n, dtype=np.float32))
    _input_args(M.assignRhsAsync, np.zeros((2 * n,))[::2])
    _input_args(M.assignRhsAsync, [0.0] * n)
    _input_args(M.getSolution, np.zeros(n, dtype=np.float64))
    _input_args(M.getSolution, np.zeros(2 * n, dtype=np.complex128)[::2])
    _input_args(M.getSolutionAsync, np.zeros(n - 1, dtype=np.complex128))
    _input_args(M.getSolutionAsync, np.zeros(n, dtype=np.float64))


def test_server_submit_checks_host_buffers():
    S = Server.__new__(Server)
    S._L = None
    S._keep = {}
    n = 4 * 4 * 4
    with pytest.raises(ValueError):
        S.submit(4, 4, 4, "NNNNDD", np.zeros(n - 1), np.zeros(n, dtype=np.complex128))
    with pytest.raises(ValueError):
        S.submit(4, 4, 4, "NNNNDD", np.zeros(n), np.zeros(n, dtype=np.float32))  # complex128 or float64 only
    with pytest.raises(ValueError):
        S.submit(4, 4, 4, "NNNNDD", np.zeros(n), np.zeros(n - 1, dtype=np.float64))
    assert S._keep == {}


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    """No CPU fallback: without libpittpack_b200.so the first call raises
    ImportError naming the build command."""
    monkeypatch.setattr(_lib, "_lib", None)
    monkeypatch.setattr(_lib, "LIB_PATH", str(tmp_path / "libpittpack_b200.so"))
    with pytest.raises(ImportError, match="pittpack_b200.build"):
        PoissonGPU(8, 8, 8)
