"""The zero-mean option (the reference's ZERO_MEAN switch, subtractMeanValue,
src/pencilDcmp.cpp:5649-5683): after the solve the mean of the solution's
real part over the grid is subtracted from it.  Checked against the plain
solve minus its own mean, for a pure-Neumann (singular, zero-mean RHS) and a
Dirichlet problem, in FP64 and in the refined mode.  The mean is summed in
a fixed order, so repeated FP64 solves give the same bits; the refined mode's
plane sums are accumulated with one atomic per CTA, so its repeats agree to
round-off."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


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
    if precision == 0:
        assert np.array_equal(P1, P2)
    else:
        assert np.abs(P1 - P2).max() <= 1e-14 * scale


def test_zero_mean_option_is_validated():
    import pittpack_b200 as pp

    with pp.make_Poisson(16, 16, 8) as M:
        with pytest.raises(pp.PittPackError):
            M.setOptions(zero_mean=2)
        assert M.options().zero_mean == 0
