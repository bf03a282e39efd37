"""One grid solved as z slabs over several ranks (pittpack_b200/distributed.py,
the staged C ABI pp_set_slab / pp_stage_*) against the oracle's whole-grid
solve, relative L2 <= 1e-12.

There is one GPU here, so the ranks are processes sharing it with gloo
exchanges staged through host memory: no kernel of one rank waits on another
(each rank's launches finish before its exchange), which is what lets them
share a GPU.  Over several GPUs the same code runs its exchanges over NCCL."""
import multiprocessing as mp
import os
import socket

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = [pytest.mark.gpu, pytest.mark.timeout(600)]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rhs(nx, ny, nz, bc):
    rng = np.random.default_rng(nx * ny + nz)
    f = rng.standard_normal((nz, ny, nx))
    if bc[0] == "P":
        f = f + 1j * rng.standard_normal((nz, ny, nx))
    return f


def _rank(rank, world, port, nx, ny, nz, bc, box, q):
    import torch
    import torch.distributed as dist

    from pittpack_b200.distributed import SlabPoisson

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        f = _rhs(nx, ny, nz, bc)
        with SlabPoisson(nx, ny, nz, bc, box) as S:
            P = S.solve(f[S.k0:S.k0 + S.nzl])
            P2 = S.solve(f[S.k0:S.k0 + S.nzl])  # a second solve on the same slab
            q.put((rank, S.k0, P, bool(np.array_equal(P, P2))))
    except Exception as e:  # reported to the parent
        q.put((rank, -1, repr(e), False))
    finally:
        dist.destroy_process_group()


def _run(target, world, *args):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=target, args=(r, world, port) + args + (q,)) for r in range(world)]
    for p in ps:
        p.start()
    res = sorted((q.get(timeout=300) for _ in ps), key=lambda r: r[0])
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    return res


CASES = [(2, 16, 12, 10, "NNNNDD", (0, 1, 0, 1, 0, 1)),        # Dirichlet z: each end face on one slab
         (2, 32, 20, 9, "PPPPDD", (0, 1, 0, 2, -1, 1)),        # half spectra, complex y / z, uneven slabs
         (2, 12, 10, 8, "DDNNPP", (0, 1, 0, 1, 0, 1)),         # periodic z (Sherman-Morrison on whole columns)
         (3, 24, 18, 15, "NDDNNN", (0, 2, 0, 1, 0, 1)),        # three ranks, quarter-wave x
         (3, 20, 10, 12, "NNNNNN", (0, 1, 0, 1, 0, 1))]        # the singular zero-mode column on one rank


@pytest.mark.parametrize("world,nx,ny,nz,bc,box", CASES)
def test_slab_solve_matches_the_whole_grid(world, nx, ny, nz, bc, box):
    res = _run(_rank, world, nx, ny, nz, bc, box)
    for rank, k0, P, same in res:
        assert k0 >= 0, P
        assert same
    P = np.concatenate([r[2] for r in res], axis=0)
    f = _rhs(nx, ny, nz, bc)
    fr, fi = (f.real.copy(), f.imag.copy()) if np.iscomplexobj(f) else (f, None)
    Q = O.solve(O.problem(nx, ny, nz, bc, box=box), fr, fi)
    assert O.rel_l2(P, Q) <= 1e-12


def test_slab_handle_refuses_the_whole_solve_and_other_modes():
    import pittpack_b200 as pp
    from pittpack_b200 import _lib

    L = _lib.load()
    with pp.make_Poisson(8, 8, 6) as M:
        M.assignBoundary("NNNNDD")
        M.assignRhs(np.ones((6, 8, 8)))
        _lib.check(L.pp_set_slab(M._h, 1, 0), "pp_set_slab")
        with pytest.raises(pp.PittPackError) as e:
            M.pittPack()  # a slab solves through the staged entry points
        assert e.value.code == 27
        M.setOptions(precision=1)
        assert L.pp_stage_forward(M._h) == 27  # the staged solve is the plain FP64 one


def _bench_rank(rank, world, port, q):
    import types

    import torch
    import torch.distributed as dist

    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        res = bench.run_slab_leg(types.SimpleNamespace(warmup=1, steps=3), torch, dist, 24, 20, 16, "NNNNDD")
        q.put((rank, res))
    except Exception as e:
        q.put((rank, repr(e)))
    finally:
        dist.destroy_process_group()


def test_bench_slab_leg_runs_and_agrees_with_one_gpu():
    """bench.py's slab leg (run on N > 1 GPUs over NCCL) through the same
    code with two gloo ranks: its line and its parity figure."""
    for rank, r in _run(_bench_rank, 2):
        assert isinstance(r, dict), r
        assert r["value"] > 0 and r["scaling"] == "strong"
        assert r["rel_l2_vs_single_gpu"] <= 1e-12
