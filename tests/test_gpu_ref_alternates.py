"""The parity modes PP_ZSOLVE_REF_PCR and PP_ZSOLVE_REF_CRP: the reference's
alternate z solvers (SOLUTIONMETHOD 1 and 2, src/pencilDcmp.cpp:6102-6148) as
its CPU build computes them, on the GPU, against the oracle's restatement
(equal to those builds bit for bit, tests/test_reference_alternates.py) and
against the builds themselves where they are present.  Tolerance: relative L2
<= 1e-12 (the transforms differ in rounding; the z step is the reference's
operation order).  Sizes outside what each alternate is defined for return
UNSUPPORTED."""
import os

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PCR = 2
CRP = 3


def gpu_solve(nx, ny, nz, bc, f, z_solver):
    import pittpack_b200 as pp

    with pp.make_Poisson(nx, ny, nz) as M:
        M.assignBoundary(bc)
        M.setOptions(z_solver=z_solver)
        if np.iscomplexobj(f):
            M.assignRhsComplex(f)
        else:
            M.assignRhs(f)
        M.pittPack()
        return M.getSolution()


CASES = [(PCR, 16, 8, 31, "DDDDDD"), (PCR, 12, 10, 100, "NNDDNN"), (PCR, 8, 6, 255, "NNNNDN"),
         (PCR, 64, 24, 50, "PPPPDD"), (PCR, 48, 20, 20, "NDNDND"), (PCR, 40, 30, 7, "PPNNDN"),
         (CRP, 16, 8, 31, "DDDDDD"), (CRP, 12, 10, 127, "NNDDDD"), (CRP, 8, 6, 255, "NNNNDD"),
         (CRP, 64, 32, 63, "PPPPDD"), (CRP, 48, 20, 15, "DNDNDD"), (CRP, 128, 64, 1023, "NNNNDD")]


@pytest.mark.parametrize("z_solver,nx,ny,nz,bc", CASES)
def test_parity_modes_match_the_oracle(z_solver, nx, ny, nz, bc):
    rng = np.random.default_rng(nx * nz)
    f = rng.standard_normal((nz, ny, nx))
    if bc[0] == "P":
        f = f + 1j * rng.standard_normal((nz, ny, nx))
    fr, fi = (f.real.copy(), f.imag.copy()) if np.iscomplexobj(f) else (f, None)
    Q = O.solve(O.problem(nx, ny, nz, bc, z_method=z_solver - 1), fr, fi)
    P = gpu_solve(nx, ny, nz, bc, f, z_solver)
    assert O.rel_l2(P, Q) <= 1e-12
    if z_solver == PCR:
        # the reference's PCR leaves the solution constant along z
        assert np.allclose(P, P[0:1], rtol=0, atol=1e-12 * np.abs(P).max())


@pytest.mark.parametrize("z_solver,nx,ny,nz,bc", [(PCR, 16, 8, 31, "NNDDDD"), (CRP, 16, 8, 31, "DDDDDD")])
def test_parity_modes_match_the_reference_build(z_solver, nx, ny, nz, bc):
    lib = os.path.join(ROOT, "oracle", "_ref", "libppref_pcr.so" if z_solver == PCR else "libppref_crp.so")
    if not os.path.exists(lib):
        pytest.skip("reference alternate builds absent (make -C oracle alternates)")
    import sys

    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    from test_reference_alternates import _ref_solve_c

    f = np.random.default_rng(9).standard_normal((nz, ny, nx))
    R = _ref_solve_c(lib, nx, ny, nz, bc, f)
    assert O.rel_l2(gpu_solve(nx, ny, nz, bc, f, z_solver), R) <= 1e-12


@pytest.mark.parametrize("z_solver,nz,bc", [(PCR, 32, "NNDDDD"), (PCR, 300, "NNDDDD"), (PCR, 30, "NNDDPP"),
                                             (CRP, 30, "NNDDDD"), (CRP, 31, "NNDDDN")])
def test_parity_modes_reject_sizes_they_are_not_defined_for(z_solver, nz, bc):
    """PCR: nz a power of two or past 256 (the reference reads out of bounds
    there), periodic z; CR-P: nz not 2^L - 1, or a Neumann end."""
    import pittpack_b200 as pp

    with pp.make_Poisson(8, 8, nz) as M:
        M.assignBoundary(bc)
        M.setOptions(z_solver=z_solver)
        M.assignRhs(np.ones((nz, 8, 8)))
        with pytest.raises(pp.PittPackError) as e:
            M.pittPack()
        assert e.value.code == 27
