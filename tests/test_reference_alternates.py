"""The reference's alternate z solvers (SOLUTIONMETHOD 1 = PCR, 2 = CR-P;
src/pencilDcmp.cpp:5239-5315 -> src/triDiag.cpp:1285-1542), built from its own
sources by oracle/Makefile, measured against its default Thomas path on the
same input.  They do not reproduce it -- the normalised PCR drops the
boundary-row modifications and CR-P only approximates the Dirichlet ends --
so parity of the z solve is pinned to the Thomas path (the golden files) and
the B200 z solve is an exact partition-method / PCR hybrid of that system.
These numbers are recorded here so that the claim stays checked.  The GPU's
parity modes PP_ZSOLVE_REF_PCR / PP_ZSOLVE_REF_CRP reproduce the two
alternates; their checker, the oracle's restatement (z_method 1 / 2), equals
these builds bit for bit."""
import ctypes
import os

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref")
LIBS = {m: os.path.join(REF, f) for m, f in (("thomas", "libppref.so"), ("pcr", "libppref_pcr.so"),
                                             ("crp", "libppref_crp.so"))}

pytestmark = pytest.mark.skipif(not all(os.path.exists(p) for p in LIBS.values()),
                                reason="reference builds absent (make -C oracle)")


def _ref_solve(lib, nx, ny, nz, bc, f):
    L = ctypes.CDLL(lib)
    dp = ctypes.POINTER(ctypes.c_double)
    L.ppref_solve.argtypes = [ctypes.c_int] * 3 + [ctypes.c_char_p, dp, dp, dp, dp, dp]
    L.ppref_solve.restype = ctypes.c_int
    box = np.array([0, 1, 0, 1, 0, 1], dtype=np.float64)
    fr = np.ascontiguousarray(f, dtype=np.float64)
    fi = np.zeros_like(fr)
    P = np.zeros(2 * f.size)
    sec = np.zeros(1)
    rc = L.ppref_solve(nx, ny, nz, bc.encode(), box.ctypes.data_as(dp), fr.ctypes.data_as(dp),
                       fi.ctypes.data_as(dp), P.ctypes.data_as(dp), sec.ctypes.data_as(dp))
    assert rc == 0
    return P.view(np.complex128).reshape(nz, ny, nx)


def _ref_solve_c(lib, nx, ny, nz, bc, f, fi=None):
    """As _ref_solve, with an optional imaginary part of the RHS; the
    reference's set-up messages kept off the test output."""
    L = ctypes.CDLL(lib)
    dp = ctypes.POINTER(ctypes.c_double)
    L.ppref_solve.argtypes = [ctypes.c_int] * 3 + [ctypes.c_char_p, dp, dp, dp, dp, dp]
    L.ppref_solve.restype = ctypes.c_int
    box = np.array([0, 1, 0, 1, 0, 1], dtype=np.float64)
    fr = np.ascontiguousarray(f, dtype=np.float64)
    fim = np.ascontiguousarray(fi if fi is not None else np.zeros_like(fr), dtype=np.float64)
    P = np.zeros(2 * f.size)
    sec = np.zeros(1)
    fd = os.dup(1)
    nul = os.open(os.devnull, os.O_WRONLY)
    os.dup2(nul, 1)
    try:
        rc = L.ppref_solve(nx, ny, nz, bc.encode(), box.ctypes.data_as(dp), fr.ctypes.data_as(dp),
                           fim.ctypes.data_as(dp), P.ctypes.data_as(dp), sec.ctypes.data_as(dp))
    finally:
        os.dup2(fd, 1)
        os.close(fd)
        os.close(nul)
    assert rc == 0
    return P.view(np.complex128).reshape(nz, ny, nx)


def _rel(a, b):
    return np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel())


def test_reference_alternates_do_not_reproduce_its_thomas_solution():
    nx, ny, nz, bc = 16, 8, 31, "DDDDDD"  # CR-P needs Dirichlet z and nz = 2^L - 1
    f = np.random.default_rng(0).standard_normal((nz, ny, nx))
    T = _ref_solve(LIBS["thomas"], nx, ny, nz, bc, f)
    pcr = _rel(_ref_solve(LIBS["pcr"], nx, ny, nz, bc, f).real, T.real)
    crp = _rel(_ref_solve(LIBS["crp"], nx, ny, nz, bc, f).real, T.real)
    assert pcr > 0.5, pcr
    assert crp > 0.02, crp


def test_reference_thomas_build_matches_the_oracle():
    from oracle import oracle as O

    nx, ny, nz, bc = 16, 8, 31, "DDDDDD"
    f = np.random.default_rng(0).standard_normal((nz, ny, nx))
    T = _ref_solve(LIBS["thomas"], nx, ny, nz, bc, f)
    assert _rel(O.solve(O.problem(nx, ny, nz, bc), f), T) <= 1e-13


ORACLE_CASES = [(1, 16, 8, 31, "DDDDDD"), (1, 12, 10, 100, "NNDDNN"), (1, 8, 6, 255, "NNNNDN"), (1, 10, 12, 7, "DDNNND"),
                (1, 9, 7, 50, "NNNNNN"), (1, 12, 8, 33, "PPPPDD"), (1, 10, 6, 20, "NNDDND"),
                (2, 16, 8, 31, "DDDDDD"), (2, 12, 10, 127, "NNDDDD"), (2, 8, 6, 255, "NNNNDD"), (2, 10, 12, 7, "DDNNDD"),
                (2, 6, 6, 3, "NNNNDD"), (2, 12, 8, 15, "PPPPDD")]


@pytest.mark.parametrize("method,nx,ny,nz,bc", ORACLE_CASES)
def test_oracle_reproduces_the_reference_alternates_bit_for_bit(method, nx, ny, nz, bc):
    """The oracle's restatement of SOLUTIONMETHOD 1 (PCR) and 2 (CR-P), the
    checker of the GPU parity modes, gives the reference build's own output
    bit for bit (its FFT in the shim is the oracle's exactly rounded DFT)."""
    from oracle import oracle as O

    f = np.random.default_rng(nz * nx).standard_normal((nz, ny, nx))
    fi = np.random.default_rng(nz * nx + 1).standard_normal((nz, ny, nx)) if bc[0] == "P" else None
    R = _ref_solve_c(LIBS["pcr" if method == 1 else "crp"], nx, ny, nz, bc, f, fi)
    Q = O.solve(O.problem(nx, ny, nz, bc, z_method=method), f, fi)
    assert np.array_equal(R, Q)


def test_reference_pcr_is_constant_along_z():
    """The CPU build of the reference's PCR updates every row of a 256-row
    block with the neighbours of the block's last row: its solution does not
    vary along z (so it does not solve the system; the parity mode reproduces
    exactly this)."""
    nx, ny, nz, bc = 16, 8, 31, "DDDDNN"
    f = np.random.default_rng(0).standard_normal((nz, ny, nx))
    P = _ref_solve(LIBS["pcr"], nx, ny, nz, bc, f).real
    assert np.array_equal(P, np.broadcast_to(P[0:1], P.shape))
