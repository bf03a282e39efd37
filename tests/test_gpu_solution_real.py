"""The real-part solution download (pp_get_solution_real / _async): exactly
the real part of the chunkedArray P that pp_get_solution returns, for the
plain and the refined solve, real RHS in every x/y family, through the C ABI."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("bc", ["PPPPDD", "NNNNDD", "NDNDDD", "DDDDDD", "PPNNNN"])
@pytest.mark.parametrize("precision", [0, 1])
def test_real_part_equals_complex_solution(bc, precision):
    import pittpack_b200 as pp
    from pittpack_b200.poisson import pinned_empty

    nx, ny, nz = 64, 48, 40
    f = np.random.default_rng(3).uniform(-1, 1, (nz, ny, nx))
    if bc[0:2] in ("NN", "PP") and bc[2:4] in ("NN", "PP") and bc[4] != "D":
        f -= f.mean()
    with pp.make_Poisson(nx, ny, nz) as M:
        M.assignBoundary(bc)
        M.setOptions(precision=precision, compat_zero_mode=0 if precision else 1)
        M.assignRhs(f)
        M.pittPack()
        P = M.getSolution()
        u = M.getSolutionReal()
        assert np.array_equal(u, P.real)
        assert np.max(np.abs(P.imag)) == 0.0  # a real RHS gives a real solution
        w = pinned_empty((nz, ny, nx), np.float64)
        M.pittPack()
        M.getSolutionRealAsync(w)
        M.synchronize()
        assert np.array_equal(np.asarray(w), P.real)


def test_real_part_rejects_wrong_buffers():
    import pittpack_b200 as pp

    with pp.make_Poisson(16, 16, 8) as M:
        M.assignBoundary("NNNNDD")
        M.assignRhs(np.ones((8, 16, 16)))
        M.pittPack()
        with pytest.raises(pp.PittPackError):
            M.getSolutionReal(np.empty((8, 16, 16), dtype=np.float32))
