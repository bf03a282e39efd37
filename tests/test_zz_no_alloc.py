"""pp_solve_noalloc: the allocation-free solve for callers that cannot call
cudaMalloc (services whose device memory belongs to their own pool
allocator, plugins that must not grow their host process's device heap).  It
is checked through the C ABI against the handle-based entry point (pp_create
/ pp_solve) and against the CPU oracle, within the 1e-12 relative L2 the
plain FP64 path is held to, on calls in a row that reuse the same fixed
scratch array: shapes one after the other, then the first shape again after
a different one.  It must also return without waiting for earlier work on
its stream (its tables are built on the device; nothing is copied from the
host).  This file is collected last so that a run that stops at the first
failure has already run every other test."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _lib():
    from pittpack_b200 import _lib

    L = _lib.load()
    fn = L.pp_solve_noalloc
    fn.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_char_p, ctypes.POINTER(ctypes.c_double),
                   ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    fn.restype = ctypes.c_int
    return L


def _handle_solve(nx, ny, nz, bc, box, f):
    import pittpack_b200 as pp

    with pp.make_Poisson(nx, ny, nz) as M:
        M.assignBoundary(bc)
        M.setBox(box)
        M.assignRhs(f)
        M.pittPack()
        return M.getSolution()


def _noalloc_solve(L, nx, ny, nz, bc, box, f):
    import torch

    d_rhs = torch.from_numpy(np.ascontiguousarray(f, dtype=np.float64).ravel()).cuda()
    d_P = torch.empty(2 * nx * ny * nz, dtype=torch.float64, device="cuda")
    b = np.ascontiguousarray(box, dtype=np.float64)
    stream = torch.cuda.current_stream()
    rc = L.pp_solve_noalloc(nx, ny, nz, bc.encode(), b.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                            d_rhs.data_ptr(), d_P.data_ptr(), stream.cuda_stream)
    torch.cuda.synchronize()
    return rc, d_P.cpu().numpy().view(np.complex128).reshape(nz, ny, nx)


def test_noalloc_matches_handle_path_and_oracle_on_calls_in_a_row():
    from oracle import oracle as O

    L = _lib()
    rng = np.random.default_rng(21)
    cases = [
        (64, 48, 40, "NNDDDD", (0, 1, 0, 1, 0, 1)),      # 3 2^k y: register passes + radix-3 pass
        (60, 36, 20, "DDNNDD", (0, 1, 0, 1, 0, 1)),      # lengths of the generic transform kernel
        (128, 64, 32, "PPPPDN", (0, 2, 0, 1, 0.5, 1.5)),  # power-of-two lengths, periodic x/y
        (256, 256, 16, "NNNNDD", (0, 1, 0, 1, 0, 1)),     # >= 256^2 z systems, 16 rows per lane
        (256, 256, 20, "DDNNDD", (0, 1, 0, 1, 0, 1)),     # >= 256^2 z systems, uneven register rows
        (45, 21, 12, "NDDNDD", (0, 1, 0, 1, 0, 1)),      # odd quarter-wave lengths: 2n-point FFTs
    ]
    inputs = [rng.uniform(-1, 1, (nz, ny, nx)) for nx, ny, nz, _, _ in cases]
    first = None
    for (nx, ny, nz, bc, box), f in zip(cases, inputs):
        rc, P = _noalloc_solve(L, nx, ny, nz, bc, box, f)
        assert rc == 0, L.pp_result_string(rc)
        Q = _handle_solve(nx, ny, nz, bc, box, f)
        err = np.linalg.norm((P - Q).ravel()) / np.linalg.norm(Q.ravel())
        assert err <= TOL, (bc, err)
        R = O.solve(O.problem(nx, ny, nz, bc, box), f)
        assert O.rel_l2(P, R) <= TOL, bc
        if first is None:
            first = P
    # the first shape again, after the others have left their contents in the array
    nx, ny, nz, bc, box = cases[0]
    rc, P = _noalloc_solve(L, nx, ny, nz, bc, box, inputs[0])
    assert rc == 0
    assert np.array_equal(P, first)


def test_noalloc_returns_without_waiting_for_the_stream():
    """Enqueued behind a long spin kernel on the same stream, the call comes
    back before the spin has finished (a call that copied tables from pageable
    host memory would wait for it)."""
    import time

    import torch

    L = _lib()
    nx, ny, nz, bc, box = 64, 48, 40, "NNDDDD", (0, 1, 0, 1, 0, 1)
    f = np.random.default_rng(5).uniform(-1, 1, (nz, ny, nx))
    _, P0 = _noalloc_solve(L, nx, ny, nz, bc, box, f)  # first call: device set-up
    d_rhs = torch.from_numpy(f.ravel().copy()).cuda()
    d_P = torch.empty(2 * nx * ny * nz, dtype=torch.float64, device="cuda")
    b = np.ascontiguousarray(box, dtype=np.float64)
    stream = torch.cuda.current_stream()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    torch.cuda._sleep(int(2e9))  # about one second of spinning at B200 clocks
    rc = L.pp_solve_noalloc(nx, ny, nz, bc.encode(), b.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                            d_rhs.data_ptr(), d_P.data_ptr(), stream.cuda_stream)
    t_call = time.perf_counter() - t0
    torch.cuda.synchronize()
    t_all = time.perf_counter() - t0
    assert rc == 0
    assert t_call < 0.25 * t_all, (t_call, t_all)
    assert np.array_equal(d_P.cpu().numpy().view(np.complex128).reshape(nz, ny, nx), P0)


def test_noalloc_rejects_grids_beyond_its_scratch():
    import torch

    L = _lib()
    n = 256  # 16.7 M points: far beyond the 32 MiB scratch
    d = torch.empty(1, dtype=torch.float64, device="cuda")
    box = np.array([0, 1, 0, 1, 0, 1.0])
    rc = L.pp_solve_noalloc(n, n, n, b"NNNNDD", box.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                            d.data_ptr(), d.data_ptr(), None)
    assert rc == 28
    assert b"NOALLOC_TOO_LARGE" in L.pp_result_string(rc)
