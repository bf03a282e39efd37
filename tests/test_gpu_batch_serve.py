"""Batched solves (one CUDA-graph replay for many uneven grids) and the request
server: every grid's result equals its stand-alone solve, within the tolerance
of its precision (plain FP64: 1e-12; refined mixed: 1e-10 against the FP64
solve of the same system with the exact zero mode)."""
import numpy as np
import pytest

pytestmark = [pytest.mark.gpu, pytest.mark.timeout(300)]

FAMS = ["PPPP", "NNNN", "NDND", "DDDD"]


def _grids(seed, n):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        nx = int(rng.choice([16, 32, 48, 64, 96]))
        ny = int(rng.choice([16, 32, 40, 64]))
        nz = int(rng.integers(8, 70))
        bc = FAMS[int(rng.integers(0, 4))] + ["DD", "NN"][int(rng.integers(0, 2))]
        f = rng.standard_normal((nz, ny, nx))
        if bc[0:2] in ("PP", "NN") and bc[2:4] in ("PP", "NN") and bc[4:] == "NN":
            f -= f.mean()
        out.append((nx, ny, nz, bc, f))
    return out


def _alone(nx, ny, nz, bc, f, **opts):
    import pittpack_b200 as pp

    with pp.make_Poisson(nx, ny, nz) as M:
        M.assignBoundary(bc)
        if opts:
            M.setOptions(**opts)
        M.assignRhs(f)
        M.pittPack()
        return M.getSolution()


def _rel(a, b):
    return np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel())


def _check(P, grid, precision):
    nx, ny, nz, bc, f = grid
    if precision == 1:
        Q = _alone(nx, ny, nz, bc, f, compat_zero_mode=0)
        assert _rel(np.asarray(P).real, Q.real) <= 1e-10, (nx, ny, nz, bc)
    else:
        Q = _alone(nx, ny, nz, bc, f)
        assert _rel(np.asarray(P), Q) <= 1e-12, (nx, ny, nz, bc)


@pytest.mark.parametrize("precision", [0, 1])
def test_batch_graph_matches_single_solves(precision):
    import torch

    from pittpack_b200.batch import Batch

    grids = _grids(7, 14)
    items, outs = [], []
    for nx, ny, nz, bc, f in grids:
        d_rhs = torch.from_numpy(f.ravel().copy()).cuda()
        d_P = torch.empty(2 * f.size, dtype=torch.float64, device="cuda")
        items.append(dict(nx=nx, ny=ny, nz=nz, bc=bc, d_rhs=d_rhs.data_ptr(), d_P=d_P.data_ptr()))
        outs.append((d_rhs, d_P))
    B = Batch(items, precision=precision, sweeps=2, branches=4, autotune=True)
    for _ in range(2):  # two replays of the same graph
        for _, d_P in outs:
            d_P.zero_()
        torch.cuda.synchronize()
        B.run(torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        for grid, (_, d_P) in zip(grids, outs):
            nx, ny, nz = grid[:3]
            _check(d_P.cpu().numpy().view(np.complex128).reshape(nz, ny, nx), grid, precision)
    n, nodes = B.info()
    assert n == len(grids) and nodes >= 5 * len(grids)
    B.close()


def test_server_results_same_alone_and_in_the_mix():
    from pittpack_b200.batch import Server
    from pittpack_b200.poisson import pinned_empty

    grids = _grids(11, 24)
    S = Server(streams=6, hbm_fraction=0.3)
    tickets = []
    for k, (nx, ny, nz, bc, f) in enumerate(grids):
        rhs = pinned_empty(f.shape, np.float64)
        rhs[...] = f
        P = pinned_empty(f.shape, np.complex128)
        prec = k % 2  # FP64 and refined requests in the same stream of work
        tickets.append((S.submit(nx, ny, nz, bc, rhs, P, precision=prec, sweeps=2), P, prec))
    for (t, P, prec), grid in zip(tickets, grids):
        st, ms, used = S.wait(t)
        assert st == 0
        assert used == prec
        assert ms > 0
        _check(P, grid, prec)
    stats = S.stats()
    assert stats["completed"] == len(grids)
    assert stats["max_inflight"] >= 2  # requests overlapped on the device
    S.close()


def test_server_real_part_output_in_the_mix():
    """Requests asking for the solution's real part alone (half the copy)
    mixed with requests for the complex P: each real-part result is exactly the
    real part of the same request's complex result."""
    from pittpack_b200.batch import Server
    from pittpack_b200.poisson import pinned_empty

    grids = _grids(13, 12)
    S = Server(streams=4, hbm_fraction=0.3)
    pairs = []
    for k, (nx, ny, nz, bc, f) in enumerate(grids):
        rhs = pinned_empty(f.shape, np.float64)
        rhs[...] = f
        Pc = pinned_empty(f.shape, np.complex128)
        Pr = pinned_empty(f.shape, np.float64)
        prec = k % 2
        pairs.append((S.submit(nx, ny, nz, bc, rhs, Pc, precision=prec, sweeps=2),
                      S.submit(nx, ny, nz, bc, rhs, Pr, precision=prec, sweeps=2), Pc, Pr, rhs))
    for tc, tr, Pc, Pr, _ in pairs:
        assert S.wait(tc)[0] == 0 and S.wait(tr)[0] == 0
        assert np.array_equal(np.asarray(Pr), np.asarray(Pc).real)
    st = S.stats()
    assert st["handles_created"] >= 1 and st["handles_evicted"] >= 0
    S.close()


def test_server_rejects_a_request_that_never_fits():
    from pittpack_b200.batch import Server
    from pittpack_b200.poisson import pinned_empty

    S = Server(streams=2, hbm_fraction=1e-6)  # a budget of a few KB
    rhs = pinned_empty((16, 16, 16), np.float64)
    rhs[...] = 1.0
    P = pinned_empty((16, 16, 16), np.complex128)
    st, _, _ = S.wait(S.submit(16, 16, 16, "DDDDDD", rhs, P))
    assert st == 15  # ALLOCATION_FAIL
    S.close()


def test_batch_with_chirp_and_long_line_grids():
    """Grids whose x length takes the chirp z-transform (131) or the
    four-step path (8192, 7500) in one graph with an ordinary grid: their
    scratch is set up by the first solve, outside the capture."""
    import torch

    from pittpack_b200.batch import Batch

    rng = np.random.default_rng(17)
    shapes = [(131, 16, 8, "NNDDDD"), (8192, 4, 3, "DDDDDD"), (7500, 4, 3, "NNNNDD"), (40, 40, 20, "DDDDNN")]
    grids, items, outs = [], [], []
    for nx, ny, nz, bc in shapes:
        f = rng.standard_normal((nz, ny, nx))
        grids.append((nx, ny, nz, bc, f))
        d_rhs = torch.from_numpy(f.ravel().copy()).cuda()
        d_P = torch.empty(2 * f.size, dtype=torch.float64, device="cuda")
        items.append(dict(nx=nx, ny=ny, nz=nz, bc=bc, d_rhs=d_rhs.data_ptr(), d_P=d_P.data_ptr()))
        outs.append((d_rhs, d_P))
    for precision in (0, 1):
        B = Batch(items, precision=precision, sweeps=2, branches=4, autotune=False)
        B.run(torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        for grid, (_, d_P) in zip(grids, outs):
            nx, ny, nz = grid[:3]
            _check(d_P.cpu().numpy().view(np.complex128).reshape(nz, ny, nx), grid, precision)
        B.close()
