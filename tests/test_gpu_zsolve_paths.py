"""The z solve's register paths on grids of at least 256^2 z systems, where
the rows stay in registers, against the CPU oracle: two half blocks per lane
(exactly 16 or 32 rows a lane) and uneven row counts, with the tile moved by
bulk copies in the z-tiled layout (complex spectra on the uneven path too),
in FP64 (relative L2 <= 1e-12) and in the refined mode on FP32 spectra
(<= 1e-10 against the oracle's exact zero mode).  Periodic z with a zero
mode reads row nz - 1 from the last lane's chunk.

Which path each grid takes follows from the lane rule of the z solve: about
32 rows a lane for real spectra, 16 for complex ones, the fewest lanes that
leave at most that many; exactly 16 or 32 rows give the split solve."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = [pytest.mark.gpu, pytest.mark.timeout(600)]


def _singular(bc):
    return bc[0:2] in ("NN", "PP") and bc[2:4] in ("NN", "PP") and bc[4] in "NP" and bc[5] in "NP"


def _solve(nx, ny, nz, bc, f, zsolve_tile=0, **opts):
    import pittpack_b200 as pp

    with pp.make_Poisson(nx, ny, nz) as M:
        M.assignBoundary(bc)
        M.setOptions(**opts)
        if zsolve_tile:
            # a z tile other than the y pass's lines per tile: the usual
            # [k][ky][kx] spectrum, tiles copied element by element
            M.setTuning(zsolve_tile=zsolve_tile)
        M.assignRhs(f)
        M.pittPack()
        P = M.getSolution()
        assert M.kernelTimeouts() == 0
        return P


def _rhs(nx, ny, nz, bc, seed):
    f = np.random.default_rng(seed).uniform(-1, 1, (nz, ny, nx))
    if _singular(bc):
        f -= f.mean()
    return f


FP64_CASES = [
    (256, 256, 32, "NNNNDD"),   # real, 1 lane x 32 rows: split, bulk tiles
    (256, 256, 64, "NNNNPP"),   # real, 2 lanes x 32 rows, periodic z with the zero mode
    (256, 256, 64, "DDDDPP"),   # real, split, periodic z without a zero mode
    (256, 256, 48, "NDNDDD"),   # real, 2 lanes x 24 rows: split
    (256, 256, 40, "NDNDDD"),   # real, 2 lanes x 20 rows: split
    (256, 256, 36, "NNNNDD"),   # real, 2 lanes x 18 rows: uneven register rows
    (256, 256, 1024, "NNNNDD"), # real, 32 lanes x 32 rows: split, 256-thread CTAs, chunks near the tile's size
    (512, 256, 32, "PPPPDD"),   # complex half spectra, 2 lanes x 16 rows: split, bulk tiles
    (512, 256, 32, "PPPPPP"),   # complex, split, periodic z with the zero mode
    (512, 256, 24, "PPPPPP"),   # complex, 2 lanes x 12 rows: split, bulk tiles, zero mode
    (512, 256, 40, "PPPPNN"),   # complex, 4 lanes x 10 rows: split, bulk tiles
    (512, 256, 36, "PPPPNN"),   # complex, 4 lanes x 9 rows: uneven rows, bulk tiles
]


@pytest.mark.parametrize("nx,ny,nz,bc", FP64_CASES)
def test_fp64_register_paths_vs_oracle(nx, ny, nz, bc):
    f = _rhs(nx, ny, nz, bc, nx + ny + nz)
    Q = O.solve(O.problem(nx, ny, nz, bc), f)
    P = _solve(nx, ny, nz, bc, f)
    assert O.rel_l2(P, Q) <= 1e-12


@pytest.mark.parametrize("nx,ny,nz,bc", [(256, 256, 48, "NDNDDD"), (256, 256, 64, "NNNNPP"), (256, 256, 40, "DDDDNN"),
                                         (512, 256, 24, "PPPPPP"), (512, 256, 32, "PPPPDD"), (512, 256, 40, "PPPPDD")])
def test_fp64_register_paths_untiled_vs_oracle(nx, ny, nz, bc):
    """The same register paths on the usual spectrum layout (a z tile of one
    system, which the z-tiled layout never has): rows read from and written to
    the skewed shared column."""
    f = _rhs(nx, ny, nz, bc, nx + ny + nz + 1)
    Q = O.solve(O.problem(nx, ny, nz, bc), f)
    P = _solve(nx, ny, nz, bc, f, zsolve_tile=1)
    assert O.rel_l2(P, Q) <= 1e-12


REFINED_CASES = [
    (256, 256, 64, "NNNNDD"),   # FP32 real spectra, split (no register cap)
    (512, 256, 32, "PPPPDD"),   # FP32 complex spectra, split (128 registers)
    (512, 256, 24, "PPPPPP"),   # FP32 complex spectra, uneven rows, zero mode
]


@pytest.mark.parametrize("nx,ny,nz,bc", REFINED_CASES)
def test_refined_register_paths_vs_oracle(nx, ny, nz, bc):
    f = _rhs(nx, ny, nz, bc, 3 * nz + 1)
    Q = O.solve(O.problem(nx, ny, nz, bc, compat_zero_mode=0), f)
    P = _solve(nx, ny, nz, bc, f, precision=1, max_sweeps=3)
    assert O.rel_l2(P.real, Q.real) <= 1e-10
