"""The multigrid alternate z solver (the reference's MultiGrid, src/multiGrid.cpp:
1105-1515, reached through PencilDcmp::solveMG, src/pencilDcmp.cpp:4047-4135)
solves the same z systems as the direct path, its V-cycles down to the FP64
rounding floor.  Tolerance: relative L2 <= 1e-10 against the CPU oracle
(oracle/pp_oracle.c, the reference's Thomas solve restated) and against the
direct path, with no system left at the cycle bound."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-10


def _solve(nx, ny, nz, bc, f, **opts):
    import pittpack_b200 as pp

    with pp.make_Poisson(nx, ny, nz) as M:
        M.assignBoundary(bc)
        M.setOptions(**opts)
        M.assignRhs(f)
        M.pittPack()
        stats = M.zsolveStats()
        return M.getSolution(), stats


def _rel(a, b):
    return np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel())


CASES = ["PPPPDD", "NNNNDD", "NDNDDD", "DDDDDD", "NNDDNN", "DNPPND", "PPPPPP", "NNNNNN", "DDNNPP", "PPPPDN"]


@pytest.mark.parametrize("bc", CASES)
@pytest.mark.parametrize("shape", [(32, 16, 64), (24, 20, 96), (16, 16, 37), (20, 12, 100), (16, 32, 8)])
@pytest.mark.parametrize("compat", [1, 0])
def test_multigrid_matches_direct(bc, shape, compat):
    nx, ny, nz = shape
    rng = np.random.default_rng(nz * 7 + len(bc))
    f = rng.standard_normal((nz, ny, nx))
    if all(bc[k:k + 2] in ("PP", "NN") for k in (0, 2, 4)):
        f -= f.mean()
    Q, _ = _solve(nx, ny, nz, bc, f, compat_zero_mode=compat)
    P, (cycles, stuck) = _solve(nx, ny, nz, bc, f, compat_zero_mode=compat, z_solver=1)
    assert _rel(P, Q) <= TOL
    assert stuck == 0
    assert cycles <= 40


@pytest.mark.parametrize("bc", CASES)
@pytest.mark.parametrize("shape", [(32, 16, 64), (20, 12, 100)])
@pytest.mark.parametrize("compat", [1, 0])
def test_multigrid_matches_oracle(bc, shape, compat):
    from oracle import oracle as O

    nx, ny, nz = shape
    rng = np.random.default_rng(nz * 11 + len(bc))
    f = rng.standard_normal((nz, ny, nx))
    if all(bc[k:k + 2] in ("PP", "NN") for k in (0, 2, 4)):
        f -= f.mean()
    Q = O.solve(O.problem(nx, ny, nz, bc, compat_zero_mode=compat), f)
    P, (cycles, stuck) = _solve(nx, ny, nz, bc, f, compat_zero_mode=compat, z_solver=1)
    assert _rel(P, Q) <= TOL
    assert stuck == 0


def test_multigrid_larger_grid():
    nx, ny, nz, bc = 128, 96, 256, "NNNNDD"
    f = np.random.default_rng(3).standard_normal((nz, ny, nx))
    Q, _ = _solve(nx, ny, nz, bc, f)
    P, (cycles, stuck) = _solve(nx, ny, nz, bc, f, z_solver=1)
    assert _rel(P, Q) <= TOL
    assert stuck == 0 and 0 < cycles <= 40


def test_multigrid_option_rules():
    import pittpack_b200 as pp

    with pp.make_Poisson(16, 16, 16) as M:
        M.assignBoundary("DDDDDD")
        with pytest.raises(pp.PittPackError) as e:
            M.setOptions(z_solver=4)  # 0..3: direct, multigrid, the two reference parity modes
        assert e.value.code == 19
        # the refined mixed-precision solve uses the direct z solve only
        M.setOptions(z_solver=1, precision=1)
        M.assignRhs(np.ones((16, 16, 16)))
        with pytest.raises(pp.PittPackError) as e:
            M.pittPack()
        assert e.value.code == 27
