"""Batched solves and the request server (C ABI: pp_batch_*, pp_server_*).

    B = Batch(items, precision=1, sweeps=1, branches=8, autotune=True)
    B.run(stream)                      # one CUDA-graph launch for all grids

    S = Server(streams=8, hbm_fraction=0.5)
    t = S.submit(nx, ny, nz, bc, rhs_host, P_host, precision=1, sweeps=1)
    status, latency_ms, precision_used = S.wait(t)

Neither exists in the reference, which solves one grid per PencilDcmp object
and per process run (src/main.cpp:73-134).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import Options, check


class BatchItem(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
        ("bc", ctypes.c_char * 6),
        ("box", ctypes.c_double * 6),
        ("d_rhs", ctypes.c_void_p),
        ("d_P", ctypes.c_void_p),
    ]


class Request(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
        ("bc", ctypes.c_char * 6),
        ("box", ctypes.c_double * 6),
        ("precision", ctypes.c_int),
        ("sweeps", ctypes.c_int),
        ("rhs", ctypes.c_void_p),
        ("P", ctypes.c_void_p),
        ("output_real", ctypes.c_int),
    ]


def _bind(L):
    if getattr(L, "_pp_batch_bound", False):
        return L
    H = ctypes.c_void_p
    i = ctypes.c_int
    L.pp_batch_create.argtypes = [ctypes.POINTER(BatchItem), i, ctypes.POINTER(Options), i, i, ctypes.POINTER(H)]
    L.pp_batch_run.argtypes = [H, ctypes.c_void_p]
    L.pp_batch_info.argtypes = [H, ctypes.POINTER(i), ctypes.POINTER(i)]
    L.pp_batch_destroy.argtypes = [H]
    L.pp_server_create.argtypes = [i, ctypes.c_double, ctypes.POINTER(H)]
    L.pp_server_submit.argtypes = [H, ctypes.POINTER(Request), ctypes.POINTER(ctypes.c_ulonglong)]
    L.pp_server_wait.argtypes = [H, ctypes.c_ulonglong, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(i)]
    L.pp_server_stats.argtypes = [H, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(i),
                                  ctypes.POINTER(ctypes.c_size_t)]
    L.pp_server_pool_stats.argtypes = [H, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_longlong)]
    L.pp_server_destroy.argtypes = [H]
    for n in ("pp_batch_create", "pp_batch_run", "pp_batch_info", "pp_batch_destroy", "pp_server_create",
              "pp_server_submit", "pp_server_wait", "pp_server_stats", "pp_server_pool_stats", "pp_server_destroy"):
        getattr(L, n).restype = i
    L._pp_batch_bound = True
    return L


def _box(b):
    arr = (ctypes.c_double * 6)()
    for k in range(6):
        arr[k] = float(b[k])
    return arr


class Batch:
    """Many grids (dicts with nx, ny, nz, bc, optional box, and device
    pointers d_rhs, d_P) solved by one graph replay."""

    def __init__(self, items, precision=0, sweeps=1, compat_zero_mode=None, branches=8, autotune=True):
        L = _bind(_lib.load())
        self._L = L
        arr = (BatchItem * len(items))()
        for k, it in enumerate(items):
            arr[k].nx, arr[k].ny, arr[k].nz = it["nx"], it["ny"], it["nz"]
            arr[k].bc = it["bc"].encode()
            arr[k].box = _box(it.get("box", (0, 1, 0, 1, 0, 1)))
            arr[k].d_rhs = it["d_rhs"]
            arr[k].d_P = it["d_P"]
        o = Options()
        L.pp_default_options(ctypes.byref(o))
        o.precision = int(precision)
        o.max_sweeps = int(sweeps)
        o.compat_zero_mode = int(compat_zero_mode if compat_zero_mode is not None else (precision == 0))
        h = ctypes.c_void_p()
        check(L.pp_batch_create(arr, len(items), ctypes.byref(o), int(branches), int(bool(autotune)),
                                ctypes.byref(h)), "pp_batch_create")
        self._h = h

    def run(self, stream: int = 0) -> None:
        check(self._L.pp_batch_run(self._h, ctypes.c_void_p(stream)), "pp_batch_run")

    def info(self):
        g, nodes = ctypes.c_int(), ctypes.c_int()
        check(self._L.pp_batch_info(self._h, ctypes.byref(g), ctypes.byref(nodes)), "pp_batch_info")
        return g.value, nodes.value

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self._L.pp_batch_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Continuous batching of single solves on the current GPU."""

    def __init__(self, streams=8, hbm_fraction=0.5):
        L = _bind(_lib.load())
        self._L = L
        h = ctypes.c_void_p()
        check(L.pp_server_create(int(streams), float(hbm_fraction), ctypes.byref(h)), "pp_server_create")
        self._h = h
        self._keep = {}

    def submit(self, nx, ny, nz, bc, rhs: np.ndarray, P: np.ndarray, precision=0, sweeps=1,
               box=(0, 1, 0, 1, 0, 1)) -> int:
        """Queue one solve; P is complex128 (the chunkedArray P) or float64 (the
        solution's real part alone, half the copy), nx*ny*nz values."""
        if not (rhs.dtype == np.float64 and rhs.size == nx * ny * nz and rhs.flags.c_contiguous):
            raise ValueError("rhs must be contiguous float64 with nx*ny*nz values")
        if not (P.dtype in (np.complex128, np.float64) and P.size == nx * ny * nz and P.flags.c_contiguous):
            raise ValueError("P must be contiguous complex128 (or float64: real part) with nx*ny*nz values")
        r = Request()
        r.nx, r.ny, r.nz = nx, ny, nz
        r.bc = bc.encode()
        r.box = _box(box)
        r.precision = int(precision)
        r.sweeps = int(sweeps)
        r.rhs = rhs.ctypes.data
        r.P = P.ctypes.data
        r.output_real = 1 if P.dtype == np.float64 else 0
        t = ctypes.c_ulonglong()
        check(self._L.pp_server_submit(self._h, ctypes.byref(r), ctypes.byref(t)), "pp_server_submit")
        self._keep[t.value] = (rhs, P)  # the buffers stay alive until wait()
        return t.value

    def wait(self, ticket: int):
        """(status, latency in ms, precision the request ran in)."""
        lat = ctypes.c_double()
        prec = ctypes.c_int()
        st = self._L.pp_server_wait(self._h, ctypes.c_ulonglong(ticket), ctypes.byref(lat), ctypes.byref(prec))
        self._keep.pop(ticket, None)
        return st, lat.value, prec.value

    def stats(self):
        c, m, b = ctypes.c_longlong(), ctypes.c_int(), ctypes.c_size_t()
        check(self._L.pp_server_stats(self._h, ctypes.byref(c), ctypes.byref(m), ctypes.byref(b)), "pp_server_stats")
        cr, ev = ctypes.c_longlong(), ctypes.c_longlong()
        check(self._L.pp_server_pool_stats(self._h, ctypes.byref(cr), ctypes.byref(ev)), "pp_server_pool_stats")
        return {"completed": c.value, "max_inflight": m.value, "pool_bytes": b.value,
                "handles_created": cr.value, "handles_evicted": ev.value}

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self._L.pp_server_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
