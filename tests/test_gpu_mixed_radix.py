"""Parity of the register-resident transform pass for the lengths m 2^k,
m = 3, 5, 9, 15 (48 .. 1536): its power-of-two factor runs as register
passes, the odd factor as one shared-memory pass (radix 3 or 5, or a
Cooley-Tukey DFT-9 = 3 x 3 or DFT-15 = 5 x 3).  Every such length in x
(contiguous pass) and in y (strided pass, z-tiled spectrum), for the real,
periodic and quarter-wave families, against the CPU oracle at the plain
path's bar (relative L2 <= 1e-12)."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-12
LENGTHS = [48, 80, 96, 144, 160, 192, 240, 288, 320, 384, 480, 576, 640, 768, 960, 1152, 1280, 1536]
FAMS = ["NNNNDD", "DDDDDD", "PPPPDD", "NDNDNN", "DNDNPP", "NNDDDN"]


def _solve(nx, ny, nz, bc, f):
    import pittpack_b200 as pp

    with pp.make_Poisson(nx, ny, nz) as M:
        M.assignBoundary(bc)
        M.assignRhs(f)
        M.pittPack()
        return M.getSolution()


@pytest.mark.parametrize("n", LENGTHS)
@pytest.mark.parametrize("axis", ["x", "y"])
@pytest.mark.parametrize("bc", FAMS)
def test_mixed_radix_lengths_vs_oracle(n, axis, bc):
    nx, ny, nz = (n, 16, 5) if axis == "x" else (16, n, 5)
    rng = np.random.default_rng(n * 7 + len(bc))
    f = rng.uniform(-1, 1, (nz, ny, nx))
    Q = O.solve(O.problem(nx, ny, nz, bc), f)
    P = _solve(nx, ny, nz, bc, f)
    assert O.rel_l2(P, Q) <= TOL, (n, axis, bc, O.rel_l2(P, Q))


def test_mixed_radix_cube_with_lift():
    # a grid where both transform directions take the new kernel and the
    # Dirichlet faces carry the manufactured lift
    nx, ny, nz, bc = 96, 80, 12, "DDDDDD"
    f = np.random.default_rng(3).uniform(-1, 1, (nz, ny, nx))
    Q = O.solve(O.problem(nx, ny, nz, bc), f)
    P = _solve(nx, ny, nz, bc, f)
    assert O.rel_l2(P, Q) <= TOL
