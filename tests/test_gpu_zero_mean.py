"""The zero-mean option (the reference's ZERO_MEAN switch, subtractMeanValue,
src/pencilDcmp.cpp:5649-5683): after the solve the mean of the solution's
real part over the grid is subtracted from it.  Checked against the plain
solve minus its own mean, for a pure-Neumann (singular, zero-mean RHS) and a
Dirichlet problem, in FP64 and in the refined mode.  The mean, and the
refined mode's plane sums, are summed in a fixed order, so repeated solves
give the same bits in both precisions.  The golden files under
tests/golden/zero_mean/ pin it to the reference's own ZERO_MEAN build."""
import glob
import os

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

GOLDEN_ZM = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "zero_mean", "*.npz")))


@pytest.mark.parametrize("path", GOLDEN_ZM, ids=[os.path.basename(p)[:-4] for p in GOLDEN_ZM])
def test_zero_mean_matches_reference_zero_mean_golden(path):
    """Default options (the reference's zero-mode row replacement) plus
    zero_mean, against the reference built with ZERO_MEAN on: relative L2
    <= 1e-12, the plain path's bar."""
    import pittpack_b200 as pp

    z = np.load(path)
    nx, ny, nz = int(z["nx"]), int(z["ny"]), int(z["nz"])
    f = z["f_re"] + 1j * z["f_im"] if z["f_im"].size else z["f_re"]
    with pp.make_Poisson(nx, ny, nz) as M:
        M.assignBoundary(str(z["bc"]))
        M.setBox(tuple(z["box"]))
        M.setOptions(zero_mean=1)
        M.assignRhs(f)
        M.pittPack()
        P = M.getSolution()
    assert O.rel_l2(P, z["P"]) <= 1e-12


@pytest.mark.parametrize("bc", ["NNNNNN", "DDNNDD", "PPPPNN"])
@pytest.mark.parametrize("precision", [0, 1])
def test_zero_mean_subtracts_the_solution_mean(bc, precision):
    import pittpack_b200 as pp

    nx, ny, nz = 32, 24, 20
    f = np.random.default_rng(len(bc) + precision).uniform(-1, 1, (nz, ny, nx))
    f -= f.mean()
    with pp.make_Poisson(nx, ny, nz) as M:
        M.assignBoundary(bc)
        M.setOptions(compat_zero_mode=0, precision=precision)
        M.assignRhs(f)
        M.pittPack()
        P0 = M.getSolution().copy()
        M.setOptions(zero_mean=1)
        M.pittPack()
        P1 = M.getSolution().copy()
        M.pittPack()
        P2 = M.getSolution()
    ref = P0.real - P0.real.mean()
    scale = np.abs(P0.real).max()
    assert abs(P1.real.mean()) <= 1e-13 * scale
    assert np.abs(P1.real - ref).max() <= 1e-12 * scale
    assert np.array_equal(P1.imag, P0.imag)
    assert np.array_equal(P1, P2)


def test_zero_mean_option_is_validated():
    import pittpack_b200 as pp

    with pp.make_Poisson(16, 16, 8) as M:
        with pytest.raises(pp.PittPackError):
            M.setOptions(zero_mean=2)
        assert M.options().zero_mean == 0
