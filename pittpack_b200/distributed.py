"""One grid solved over several GPUs: z slabs and two all-to-all exchanges.

The reference decomposes the grid into pencils over MPI ranks and moves data
between them with host-staged exchanges (src/pencilDcmp.cpp:851-1825).  Here
rank r of a torch.distributed group holds the z planes k0 .. k0 + nz_r - 1 of
the grid and a handle for that slab (pp_set_slab), and one solve is

    pp_stage_forward      x and y transforms of the slab (local)
    all-to-all            rank s receives, from every slab, the spectrum rows
                          ky = j0_s .. j0_s + rows_s - 1: in rank order the
                          blocks form [k][ky - j0_s][col] over the whole grid
    pp_stage_zsolve       the z solve of those columns (local)
    all-to-all            the columns go back to their slabs
    pp_stage_inverse      inverse y and x transforms (local)

so that each z system is solved whole on one GPU.  The exchanges use
all_to_all_single on device tensors over NCCL; over gloo (CPU tests) they
are staged through host memory.  Uneven splits are allowed: nz and ny are
divided as evenly as possible, the first ranks taking one more.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import check
from .poisson import make_Poisson


def split(n: int, parts: int):
    """Sizes and first indices of n items over parts ranks."""
    sizes = [n // parts + (1 if r < n % parts else 0) for r in range(parts)]
    starts = [sum(sizes[:r]) for r in range(parts)]
    return sizes, starts


def pack_rows(S, ys, y0):
    """The send buffer of the forward exchange: for each destination s, the
    slab's spectrum rows y0[s] .. y0[s] + ys[s] - 1, [k][row][col] each."""
    import torch

    return torch.cat([S[:, y0[s]:y0[s] + ys[s], :].reshape(-1) for s in range(len(ys))])


def unpack_rows(S, back, ys, y0):
    """The reverse exchange's buffer (blocks in rank order, [k][row][col]
    each) written back into the slab's spectrum rows."""
    off = 0
    nzl, cols = S.shape[0], S.shape[2]
    for s in range(len(ys)):
        n = nzl * ys[s] * cols
        S[:, y0[s]:y0[s] + ys[s], :] = back[off:off + n].view(nzl, ys[s], cols)
        off += n


def exchange(out, inp, out_sizes, in_sizes, group=None):
    """all_to_all_single; over a backend without device tensors (gloo) the
    buffers go through host memory."""
    import torch.distributed as dist

    if out.is_cuda and dist.get_backend(group) != "nccl":
        o = out.new_empty(out.shape, device="cpu")
        dist.all_to_all_single(o, inp.cpu(), out_sizes, in_sizes, group=group)
        out.copy_(o)
    else:
        dist.all_to_all_single(out, inp, out_sizes, in_sizes, group=group)


class _DevArray:
    """A device pointer presented to torch.as_tensor."""

    def __init__(self, ptr: int, count: int):
        self.__cuda_array_interface__ = {"shape": (count,), "typestr": "<f8", "data": (ptr, False), "version": 3}


class SlabPoisson:
    """The plain FP64 solve of an nx x ny x nz grid whose z planes are split
    over the ranks of a torch.distributed group (one GPU each).  solve() takes
    the rank's planes of the RHS, (nz_r, ny, nx) real or complex, and returns
    the same planes of the chunkedArray solution P (complex)."""

    def __init__(self, nx: int, ny: int, nz: int, bc: str, box=(0, 1, 0, 1, 0, 1), group=None):
        import torch.distributed as dist

        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.nx, self.ny, self.nz = nx, ny, nz
        self.zs, self.z0 = split(nz, self.world)
        self.ys, self.y0 = split(ny, self.world)
        if min(self.zs) < 1 or min(self.ys) < 1:
            raise ValueError("every rank needs at least one z plane and one y row")
        self.nzl, self.k0 = self.zs[self.rank], self.z0[self.rank]
        dz = (box[5] - box[4]) / nz
        self.M = make_Poisson(nx, ny, self.nzl)
        self.M.assignBoundary(bc)
        # the slab's own z extent, so that its cell size is the grid's
        self.M.setBox([box[0], box[1], box[2], box[3], box[4] + self.k0 * dz, box[4] + (self.k0 + self.nzl) * dz])
        self._L = _lib.load()
        check(self._L.pp_set_slab(self.M._h, int(self.rank == 0), int(self.rank == self.world - 1)), "pp_set_slab")

    def close(self):
        self.M.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def solve(self, f_local, to_host: bool = True):
        """Solve with this rank's planes of the RHS: a host array, or a CUDA
        tensor (copied on the device).  Returns this rank's planes of P as a
        host array, or (to_host False) None, P staying in the handle's device
        buffer (solution_device())."""
        import torch

        L, h = self._L, self.M._h
        if isinstance(f_local, torch.Tensor):
            f = f_local.contiguous()
            self.M.assignRhsDevice(f.data_ptr(), f.is_complex())
        elif np.iscomplexobj(f_local):
            self.M.assignRhsComplex(f_local)
        else:
            self.M.assignRhs(f_local)
        check(L.pp_stage_forward(h), "pp_stage_forward")
        ptr = ctypes.c_void_p()
        ncol, parts = ctypes.c_int(), ctypes.c_int()
        check(L.pp_stage_spectrum(h, ctypes.byref(ptr), ctypes.byref(ncol), ctypes.byref(parts)), "pp_stage_spectrum")
        cols = ncol.value * parts.value
        self.M.synchronize()
        S = torch.as_tensor(_DevArray(ptr.value, self.nzl * self.ny * cols), device="cuda").view(self.nzl, self.ny, cols)
        in_sizes = [self.nzl * self.ys[s] * cols for s in range(self.world)]
        out_sizes = [self.zs[r] * self.ys[self.rank] * cols for r in range(self.world)]
        send = pack_rows(S, self.ys, self.y0)
        recv = torch.empty(sum(out_sizes), dtype=torch.float64, device="cuda")
        exchange(recv, send, out_sizes, in_sizes, self.group)
        torch.cuda.synchronize()
        check(L.pp_stage_zsolve(h, recv.data_ptr(), self.nz, self.ys[self.rank], self.y0[self.rank]), "pp_stage_zsolve")
        self.M.synchronize()
        back = torch.empty_like(send)
        exchange(back, recv, in_sizes, out_sizes, self.group)
        unpack_rows(S, back, self.ys, self.y0)
        torch.cuda.synchronize()
        check(L.pp_stage_inverse(h), "pp_stage_inverse")
        if not to_host:
            return None
        return self.M.getSolution()

    def solution_device(self):
        """This rank's planes of P on the device, a complex128 tensor view
        (nz_r, ny, nx) of the handle's buffer (valid until the next solve)."""
        import torch

        self.M.synchronize()
        n = 2 * self.nzl * self.ny * self.nx
        t = torch.as_tensor(_DevArray(self.M.solutionDevicePtr(), n), device="cuda")
        return t.view(torch.complex128).view(self.nzl, self.ny, self.nx)
