"""The refined mixed-precision solve (FP32 transforms + FP64 residual
refinement of the true 7-point system) against the FP64 oracle in exact
zero-mode semantics.  Tolerance: relative L2 <= 1e-10, the bar of the refined
solve, reached within 3 refinement sweeps."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-10


def mixed_solve(nx, ny, nz, bc, f, sweeps, box=(0, 1, 0, 1, 0, 1)):
    import pittpack_b200 as pp

    with pp.make_Poisson(nx, ny, nz) as M:
        M.assignBoundary(bc)
        M.setBox(box)
        M.setOptions(precision=1, max_sweeps=sweeps)
        M.assignRhs(f)
        M.pittPack()
        return M.getSolution()


def _singular(bc):
    return bc[0:2] in ("NN", "PP") and bc[2:4] in ("NN", "PP") and bc[4] in "NP" and bc[5] in "NP"


CASES = ["PPPPDD", "NNNNDD", "NDNDDD", "DDDDDD", "NNDDNN", "DNPPND", "PPPPPP", "NNNNNN", "DDNNPP", "PPNNDN"]


@pytest.mark.parametrize("bc", CASES)
# power-of-two lengths (register-resident FP32 kernel) and 2/3/5-smooth ones
# (shared-memory FP32 kernel), mixed within one grid too
@pytest.mark.parametrize("shape", [(32, 64, 24), (64, 16, 7), (48, 40, 30), (24, 20, 18), (60, 36, 9), (32, 30, 16),
                                   # the residual kernel's edge cases: fewer rows than its 8-row tile,
                                   # odd nx (8-byte copies), partial x / y tiles, nz below its z chunk
                                   (16, 4, 10), (45, 12, 10), (96, 100, 40), (128, 12, 3),
                                   # prime lengths past 72: the chirp z-transform in FP32, x and y
                                   (131, 24, 10), (24, 131, 10)])
def test_refined_vs_exact_oracle(bc, shape):
    nx, ny, nz = shape
    if bc[0:2] == "PP" and bc[2:4] != "PP":
        bc = "PPPP" + bc[4:]
    rng = np.random.default_rng(abs(hash((bc, shape))) % 2**32)
    f = rng.uniform(-1, 1, (nz, ny, nx))
    if _singular(bc):
        f -= f.mean()
    Q = O.solve(O.problem(nx, ny, nz, bc, compat_zero_mode=0), f)
    errs = [O.rel_l2(mixed_solve(nx, ny, nz, bc, f, k).real, Q.real) for k in range(4)]
    # every sweep reduces the error, and 3 sweeps reach the refined-solve bar
    assert errs[0] < 1e-4, errs
    assert errs[3] <= TOL, errs
    assert errs[1] < errs[0], errs


@pytest.mark.parametrize("bc", ["NNNNNN", "PPPPDD", "DDDDDD", "NDNDDD"])
@pytest.mark.parametrize("shape", [(64, 48, 40), (60, 36, 20)])
def test_refined_solves_are_bitwise_reproducible(bc, shape):
    """The plane sums of the kx = ky = 0 column come from per-CTA partials
    added in a fixed order: two refined solves of one RHS give the same bits
    (with the residual in the transform's load, and from the residual kernel
    for lengths of the generic transform kernel)."""
    import pittpack_b200 as pp

    nx, ny, nz = shape
    f = np.random.default_rng(8).uniform(-1, 1, (nz, ny, nx))
    if _singular(bc):
        f -= f.mean()
    with pp.make_Poisson(nx, ny, nz) as M:
        M.assignBoundary(bc)
        M.setOptions(precision=1, max_sweeps=2)
        M.assignRhs(f)
        M.pittPack()
        a = M.getSolution().copy()
        M.pittPack()
        b = M.getSolution()
    assert np.array_equal(a, b)


def test_refined_full_size_residual():
    """512^3: the refined solution satisfies the 7-point system to ~FP64 accuracy."""
    n = 512
    bc = "NNNNDD"
    f = np.random.default_rng(4).uniform(-1, 1, (n, n, n))
    P = mixed_solve(n, n, n, bc, f, 2)
    pb = O.problem(n, n, n, bc, compat_zero_mode=0)
    b = O.scaled_rhs(pb, f)
    r = O.residual(pb, np.ascontiguousarray(P.real), b)
    assert np.linalg.norm(r) <= 1e-10 * np.linalg.norm(b)


def test_refined_rejects_unsupported_inputs():
    import pittpack_b200 as pp

    with pp.make_Poisson(24, 16, 8) as M:  # the refined solve takes a real RHS only
        M.assignBoundary("NNNNDD")
        M.setOptions(precision=1, max_sweeps=1)
        M.assignRhsComplex(np.zeros((8, 16, 24), dtype=np.complex128))
        with pytest.raises(pp.PittPackError) as e:
            M.pittPack()
        assert e.value.code == 27
