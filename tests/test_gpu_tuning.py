"""Launch-shape tuning, the autotuner, zero-copy device buffers and the
asynchronous copies: every variant gives the default solve's result (plain
FP64, relative L2 <= 1e-12)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _rel(a, b):
    return np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel())


def _default(nx, ny, nz, bc, f):
    import pittpack_b200 as pp

    with pp.make_Poisson(nx, ny, nz) as M:
        M.assignBoundary(bc)
        M.assignRhs(f)
        M.pittPack()
        return M.getSolution()


SHAPES = [(32, 16, 64, "PPPPDD"), (48, 40, 30, "NNDDNN"), (24, 20, 100, "DDNNPP"), (64, 64, 9, "NDNDDD")]


@pytest.mark.parametrize("shape", SHAPES)
def test_every_launch_shape_gives_the_same_solution(shape):
    import pittpack_b200 as pp

    nx, ny, nz, bc = shape
    f = np.random.default_rng(nz).standard_normal((nz, ny, nx))
    Q = _default(nx, ny, nz, bc, f)
    with pp.make_Poisson(nx, ny, nz) as M:
        M.assignBoundary(bc)
        M.assignRhs(f)
        lanes = [P for P in (1, 2, 4, 8, 16, 32) if P == 1 or P <= nz // 2]
        for P in lanes:
            for L, T in ((0, 0), (1, 2), (4, 8), (8, 1), (0, 32)):
                M.setTuning(zsolve_lanes=P, line_tile=L, zsolve_tile=T)
                assert M.tuning() == {"zsolve_lanes": P, "line_tile": L, "zsolve_tile": T}
                M.pittPack()
                assert _rel(M.getSolution(), Q) <= TOL, (P, L, T)


def test_autotune_keeps_a_valid_shape_and_the_result():
    import pittpack_b200 as pp

    nx, ny, nz, bc = 40, 36, 48, "NNNNDD"
    f = np.random.default_rng(5).standard_normal((nz, ny, nx))
    Q = _default(nx, ny, nz, bc, f)
    with pp.make_Poisson(nx, ny, nz) as M:
        M.assignBoundary(bc)
        M.assignRhs(f)
        shape, ms = M.autotune(reps=2)
        assert ms > 0
        assert shape == M.tuning()
        M.pittPack()
        assert _rel(M.getSolution(), Q) <= TOL


def test_invalid_tuning_is_rejected():
    import pittpack_b200 as pp

    with pp.make_Poisson(16, 16, 8) as M:
        for bad in ({"zsolve_lanes": 3}, {"zsolve_lanes": 8}, {"zsolve_lanes": 64}, {"line_tile": 33},
                    {"zsolve_tile": 3}, {"zsolve_tile": 64}):
            with pytest.raises(pp.PittPackError) as e:
                M.setTuning(**bad)
            assert e.value.code == 19


@pytest.mark.parametrize("cplx", [False, True])
def test_bound_device_buffers_zero_copy(cplx):
    import torch

    import pittpack_b200 as pp

    nx, ny, nz, bc = 32, 24, 20, "PPPPNN" if cplx else "DDNNDD"
    rng = np.random.default_rng(11)
    f = rng.standard_normal((nz, ny, nx))
    if cplx:
        f = f + 1j * rng.standard_normal((nz, ny, nx))
        f -= f.mean()
    Q = _default(nx, ny, nz, bc, f)
    d_rhs = torch.from_numpy(np.ascontiguousarray(f).view(np.float64).ravel().copy()).cuda()
    d_P = torch.zeros(2 * f.size, dtype=torch.float64, device="cuda")
    with pp.make_Poisson(nx, ny, nz) as M:
        M.assignBoundary(bc)
        M.setStream(torch.cuda.current_stream().cuda_stream)
        M.bindDeviceBuffers(d_rhs.data_ptr(), cplx, d_P.data_ptr())
        for _ in range(2):
            d_P.zero_()
            M.pittPack()
            torch.cuda.synchronize()
            P = d_P.cpu().numpy().view(np.complex128).reshape(nz, ny, nx)
            assert _rel(P, Q) <= TOL
            assert M.solutionDevicePtr() == d_P.data_ptr()
            assert _rel(M.getSolution(), Q) <= TOL
        # a host RHS unbinds d_rhs; the solution still goes to d_P
        M.assignRhs(f)
        M.pittPack()
        torch.cuda.synchronize()
        assert _rel(d_P.cpu().numpy().view(np.complex128).reshape(nz, ny, nx), Q) <= TOL


def test_async_copies():
    import pittpack_b200 as pp
    from pittpack_b200.poisson import pinned_empty

    nx, ny, nz, bc = 64, 32, 17, "NNDDDD"
    f = np.random.default_rng(2).standard_normal((nz, ny, nx))
    Q = _default(nx, ny, nz, bc, f)
    rhs = pinned_empty((nz, ny, nx), np.float64)
    rhs[...] = f
    out = pinned_empty((nz, ny, nx), np.complex128)
    with pp.make_Poisson(nx, ny, nz) as M:
        M.assignBoundary(bc)
        M.assignRhsAsync(rhs)
        M.pittPack()
        M.getSolutionAsync(out)
        M.synchronize()
        assert _rel(np.asarray(out), Q) <= TOL
