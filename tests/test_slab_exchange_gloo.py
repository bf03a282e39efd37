"""The host logic of the slab-decomposed solve (pittpack_b200/distributed.py)
on CPU tensors with two and three gloo ranks: the forward exchange gives each
rank every slab's planes of its spectrum rows in grid order, [k][row][col],
and the reverse exchange puts them back where they came from.  No GPU."""
import multiprocessing as mp
import os
import socket

import numpy as np
import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, nz, ny, cols, q):
    import torch
    import torch.distributed as dist

    from pittpack_b200.distributed import exchange, pack_rows, split, unpack_rows

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        zs, z0 = split(nz, world)
        ys, y0 = split(ny, world)
        # the whole grid's "spectrum": value = 1e6 k + 1e3 row + col
        k = np.arange(nz)[:, None, None]
        j = np.arange(ny)[None, :, None]
        c = np.arange(cols)[None, None, :]
        G = torch.from_numpy((1e6 * k + 1e3 * j + c).astype(np.float64))
        S = G[z0[rank]:z0[rank] + zs[rank]].clone()
        in_sizes = [zs[rank] * ys[s] * cols for s in range(world)]
        out_sizes = [zs[r] * ys[rank] * cols for r in range(world)]
        send = pack_rows(S, ys, y0)
        recv = torch.empty(sum(out_sizes), dtype=torch.float64)
        exchange(recv, send, out_sizes, in_sizes)
        ok_fwd = torch.equal(recv.view(nz, ys[rank], cols), G[:, y0[rank]:y0[rank] + ys[rank]])
        # the "z solve": columns times 2, then back
        recv *= 2
        back = torch.empty_like(send)
        exchange(back, recv, in_sizes, out_sizes)
        S2 = torch.zeros_like(S)
        unpack_rows(S2, back, ys, y0)
        ok_back = torch.equal(S2, 2 * S)
        q.put((rank, bool(ok_fwd), bool(ok_back)))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,nz,ny,cols", [(2, 8, 6, 5), (2, 7, 5, 3), (3, 10, 7, 4)])
def test_exchanges_regroup_and_restore_the_spectrum(world, nz, ny, cols):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank, args=(r, world, port, nz, ny, cols, q)) for r in range(world)]
    for p in ps:
        p.start()
    res = [q.get(timeout=120) for _ in ps]
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert all(f and b for _, f, b in res), res


def test_split_is_even_first_ranks_take_one_more():
    from pittpack_b200.distributed import split

    assert split(10, 3) == ([4, 3, 3], [0, 4, 7])
    assert split(8, 2) == ([4, 4], [0, 4])
