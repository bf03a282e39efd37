"""The CPU oracle against the reference's golden outputs and against the
mathematics (7-point residual, manufactured-solution convergence)."""
import glob
import os

import numpy as np
import pytest

from oracle import oracle as O

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))
# recorded from the reference built with ZERO_MEAN on (tests/golden/make_golden.py)
GOLDEN_ZM = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "zero_mean", "*.npz")))


def _load(path):
    z = np.load(path)
    bc = str(z["bc"])
    fi = z["f_im"] if z["f_im"].size else None
    return int(z["nx"]), int(z["ny"]), int(z["nz"]), bc, tuple(z["box"]), z["f_re"], fi, z["P"]


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_oracle_matches_reference_golden(path):
    nx, ny, nz, bc, box, fr, fi, P = _load(path)
    Q = O.solve(O.problem(nx, ny, nz, bc, box), fr, fi)
    # the oracle restates the reference's arithmetic step by step; the only
    # foreign piece (the DFT) is the same exactly rounded DFT in both
    assert O.rel_l2(Q, P) <= 1e-15
    assert np.max(np.abs(Q - P)) <= 1e-15 * max(1.0, np.max(np.abs(P)))


VALID = ["DDDDDD", "NNNNDD", "PPPPDD", "NNDDNN", "DDPPPP", "NDDNDD", "DNPPND", "PPPPPP",
         "NNNNNN", "DDNNDN", "NDNDNN", "PPPPND"]


def _singular(bc):
    return bc[4] in "NP" and bc[5] in "NP" and bc[0:2] in ("NN", "PP") and bc[2:4] in ("NN", "PP")


@pytest.mark.parametrize("bc", VALID)
@pytest.mark.parametrize("shape", [(12, 10, 9), (7, 9, 5), (16, 8, 4)])
def test_exact_mode_solves_the_7_point_system(bc, shape):
    nx, ny, nz = shape
    rng = np.random.default_rng(hash((bc, shape)) % 2**32)
    pb = O.problem(nx, ny, nz, bc, compat_zero_mode=0)
    f = rng.standard_normal((nz, ny, nx))
    if _singular(bc):
        f -= f.mean()
    P = O.solve(pb, f)
    b = O.scaled_rhs(pb, f)
    r = O.residual(pb, P.real, b)
    assert np.linalg.norm(r) <= 1e-13 * np.linalg.norm(b)


def test_compat_zero_mode_differs_only_in_the_zero_mode():
    # NN-NN with Dirichlet z: the reference pins row 0 of the kx=ky=0 column
    nx, ny, nz = 8, 6, 7
    f = np.random.default_rng(5).standard_normal((nz, ny, nx))
    a = O.solve(O.problem(nx, ny, nz, "NNNNDD", compat_zero_mode=1), f)
    b = O.solve(O.problem(nx, ny, nz, "NNNNDD", compat_zero_mode=0), f)
    d = (a - b).real
    # the difference is constant over every z-plane (it lives in kx=ky=0 only)
    assert np.max(np.abs(d - d.mean(axis=(1, 2), keepdims=True))) < 1e-13
    assert np.max(np.abs(d)) > 1e-6


def test_dft_matches_numpy():
    rng = np.random.default_rng(0)
    for n in (2, 3, 5, 8, 12, 30, 97):
        x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
        assert np.allclose(O.dft(x), np.fft.fft(x), rtol=0, atol=1e-13)
        assert np.allclose(O.dft(x, +1), np.fft.ifft(x) * n, rtol=0, atol=1e-13)


@pytest.mark.parametrize("bc", ["NNNNDD", "DDDDDD", "PPPPDD", "DDNNDD"])
def test_manufactured_solution_converges_second_order(bc):
    errs = []
    for n in (8, 16, 32):
        pb = O.problem(n, n, n, bc)
        fr, fi, ur, ui = O.manufactured(pb)
        P = O.solve(pb, fr, fi if bc[0] == "P" else None)
        e = np.sqrt(np.mean(np.abs(P.real - ur) ** 2 + (np.abs(P.imag - ui) ** 2 if bc[0] == "P" else 0)))
        errs.append(e)
    rates = [np.log2(errs[i] / errs[i + 1]) for i in range(2)]
    assert min(rates) > 1.8, (errs, rates)


@pytest.mark.parametrize("case", [(8, 6, 5, "DDDDDD"), (8, 6, 5, "NNDDDN"), (6, 5, 7, "DNNDND"), (8, 8, 4, "NDDNDD")])
def test_oracle_face_values_give_the_exact_discrete_solution(case):
    # the construction of the GPU test: f and the face data from a smooth u
    # through the ghost-cell relations, so that u solves the discrete problem
    from test_gpu_face_values import _problem

    nx, ny, nz, bc = case
    box = (0.0, 1.0, -0.5, 1.0, 0.2, 1.0)
    u, f, faces = _problem(nx, ny, nz, bc, box)
    P = O.solve(O.problem(nx, ny, nz, bc, box=box, compat_zero_mode=0, faces=faces), f)
    assert np.linalg.norm(P.real - u) / np.linalg.norm(u) <= 1e-12


def test_oracle_zero_mean_subtracts_the_solution_mean():
    nx, ny, nz, bc = 8, 6, 5, "NNNNNN"
    f = np.random.default_rng(2).uniform(-1, 1, (nz, ny, nx))
    f -= f.mean()
    P0 = O.solve(O.problem(nx, ny, nz, bc, compat_zero_mode=0), f)
    P1 = O.solve(O.problem(nx, ny, nz, bc, compat_zero_mode=0, zero_mean=1), f)
    assert np.allclose(P1.real, P0.real - P0.real.mean(), rtol=0, atol=1e-14 * np.abs(P0.real).max())
    assert abs(P1.real.mean()) <= 1e-14 * np.abs(P0.real).max()


@pytest.mark.parametrize("path", GOLDEN_ZM, ids=[os.path.basename(p)[:-4] for p in GOLDEN_ZM])
def test_oracle_zero_mean_matches_reference_zero_mean_golden(path):
    # the reference's subtractMeanValue (src/pencilDcmp.cpp:5649-5683) after
    # its default solve, against the oracle's zero_mean step
    nx, ny, nz, bc, box, fr, fi, P = _load(path)
    Q = O.solve(O.problem(nx, ny, nz, bc, box, zero_mean=1), fr, fi)
    assert O.rel_l2(Q, P) <= 1e-14
    assert abs(P.real.mean()) <= 1e-15 * np.abs(P.real).max()
    assert abs(Q.real.mean()) <= 1e-15 * np.abs(Q.real).max()


REF_LIB = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref", "libppref.so")
SWEEP = [fx + fy + z for fx in ("PP", "NN", "DD") for fy in ("PP", "NN", "DD") for z in ("DD", "NN", "DN", "ND", "PP")]


@pytest.mark.skipif(not os.path.exists(REF_LIB), reason="reference build absent (make -C oracle)")
@pytest.mark.parametrize("bc", SWEEP)
def test_oracle_equals_the_reference_build_on_every_family(bc):
    """Live sweep against the reference's own CPU solve (oracle/_ref): every
    x/y family pair the reference has times every z end pair, two shapes
    (odd and even lengths), a non-unit box, RHS as given (no compatibility
    projection for the singular sets), complex data when x is periodic."""
    import ctypes

    L = ctypes.CDLL(REF_LIB)
    dp = ctypes.POINTER(ctypes.c_double)
    L.ppref_solve.argtypes = [ctypes.c_int] * 3 + [ctypes.c_char_p, dp, dp, dp, dp, dp]
    L.ppref_solve.restype = ctypes.c_int
    box = np.array([0, 1, 0, 2, -1, 1.0])
    for k, (nx, ny, nz) in enumerate([(8, 6, 5), (10, 12, 9)]):
        rng = np.random.default_rng(SWEEP.index(bc) * 2 + k)
        fr = rng.uniform(-1, 1, (nz, ny, nx))
        fi = rng.uniform(-1, 1, (nz, ny, nx)) if bc[0] == "P" else None
        out = np.zeros(2 * nx * ny * nz)
        sec = ctypes.c_double()
        rc = L.ppref_solve(nx, ny, nz, bc.encode(), box.ctypes.data_as(dp), fr.ctypes.data_as(dp),
                           None if fi is None else fi.ctypes.data_as(dp), out.ctypes.data_as(dp), ctypes.byref(sec))
        assert rc == 0
        Q = O.solve(O.problem(nx, ny, nz, bc, tuple(box)), fr, fi)
        # identical bits on this image; the bound allows another libm
        assert O.rel_l2(Q, out.view(np.complex128).reshape(nz, ny, nx)) <= 1e-15, (bc, (nx, ny, nz))


@pytest.mark.skipif(not os.path.exists(REF_LIB), reason="reference build absent (make -C oracle)")
@pytest.mark.parametrize("shape", [(14, 13, 5), (7, 22, 6), (11, 17, 4), (26, 9, 7)])
@pytest.mark.parametrize("bc", ["PPPPDD", "NNNNDD", "DDDDNN", "NNDDPP"])
def test_oracle_equals_the_reference_build_on_lengths_with_large_prime_factors(bc, shape):
    """Lengths with prime factors above 5 (7, 11, 13, 17): the reference
    hands them to FFTW like any other; the oracle's DFT takes every length."""
    import ctypes

    L = ctypes.CDLL(REF_LIB)
    dp = ctypes.POINTER(ctypes.c_double)
    L.ppref_solve.argtypes = [ctypes.c_int] * 3 + [ctypes.c_char_p, dp, dp, dp, dp, dp]
    nx, ny, nz = shape
    rng = np.random.default_rng(nx * ny + nz)
    fr = rng.uniform(-1, 1, (nz, ny, nx))
    fi = rng.uniform(-1, 1, (nz, ny, nx)) if bc[0] == "P" else None
    out = np.zeros(2 * nx * ny * nz)
    box = np.array([0, 1, 0, 1, 0, 1.0])
    sec = ctypes.c_double()
    L.ppref_solve(nx, ny, nz, bc.encode(), box.ctypes.data_as(dp), fr.ctypes.data_as(dp),
                  None if fi is None else fi.ctypes.data_as(dp), out.ctypes.data_as(dp), ctypes.byref(sec))
    Q = O.solve(O.problem(nx, ny, nz, bc), fr, fi)
    assert O.rel_l2(Q, out.view(np.complex128).reshape(nz, ny, nx)) <= 1e-15, (bc, shape)
