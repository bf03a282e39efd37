"""CPU oracle for the PittPack Poisson solve -- TEST INFRASTRUCTURE ONLY.

This module is the checker used by ``tests/``, ``__graft_entry__.smoke()`` and
the CPU-baseline leg of ``bench.py``.  The product package ``pittpack_b200``
never imports it.

It wraps ``pp_oracle.c`` (a plain-C restatement of the reference's single-rank
solve, every step cited there against the PittPack sources) through ctypes and
adds a few numpy helpers.  Parity status: pinned against outputs of the
reference's own CPU path built from its unmodified sources
(``oracle/ref_probe.cpp`` + ``oracle/Makefile``; fixtures in ``tests/golden``).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libpp_oracle.so")
_lib = None

DST2, DCT2, FFT, DCT4, DST4 = 0, 1, 2, 3, 4


class Problem(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int),
        ("ny", ctypes.c_int),
        ("nz", ctypes.c_int),
        ("bc", ctypes.c_char * 6),
        ("box", ctypes.c_double * 6),
        ("compat_zero_mode", ctypes.c_int),
        ("dirichlet_lift", ctypes.c_int),
        ("face", ctypes.c_void_p * 6),
        ("zero_mean", ctypes.c_int),
        ("z_method", ctypes.c_int),
    ]


def build(force: bool = False) -> str:
    """Compile pp_oracle.c into libpp_oracle.so next to this file."""
    src = os.path.join(_HERE, "pp_oracle.c")
    if force or not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        subprocess.check_call(
            ["gcc", "-O2", "-fPIC", "-shared", "-o", _LIB_PATH, src, "-lm"], cwd=_HERE
        )
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_LIB_PATH)
        dp = ctypes.POINTER(ctypes.c_double)
        pp = ctypes.POINTER(Problem)
        L.ppo_solve.argtypes = [pp, dp, dp, dp]
        L.ppo_solve.restype = ctypes.c_int
        L.ppo_check.argtypes = [pp]
        L.ppo_eigenvalue.argtypes = [pp, ctypes.c_int, ctypes.c_int]
        L.ppo_eigenvalue.restype = ctypes.c_double
        L.ppo_dft.argtypes = [ctypes.c_int, ctypes.c_int, dp, dp]
        L.ppo_dirichlet_lift.argtypes = [pp, dp]
        L.ppo_manufactured.argtypes = [pp, dp, dp, dp, dp]
        L.ppo_residual.argtypes = [pp, dp, dp, dp]
        L.ppo_kind_from_bc.argtypes = [ctypes.c_char, ctypes.c_char]
        _lib = L
    return _lib


def _dp(a):
    if a is None:
        return None
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def problem(nx, ny, nz, bc, box=(0, 1, 0, 1, 0, 1), compat_zero_mode=1, dirichlet_lift=1, faces=None,
            zero_mean=0, z_method=0) -> Problem:
    """faces: {face 0..5: array} of boundary data (Dirichlet values / Neumann
    outward derivatives, shaped (nz, ny), (nz, nx) or (ny, nx) for x, y, z
    faces); zero_mean: subtract the solution's mean (ZERO_MEAN)."""
    p = Problem()
    p.nx, p.ny, p.nz = nx, ny, nz
    p.bc = bc.encode() if isinstance(bc, str) else bytes(bc)
    for i in range(6):
        p.box[i] = float(box[i])
    p.compat_zero_mode = int(compat_zero_mode)
    p.dirichlet_lift = int(dirichlet_lift)
    p.zero_mean = int(zero_mean)
    p.z_method = int(z_method)
    keep = []
    for f, g in (faces or {}).items():
        a = np.ascontiguousarray(g, dtype=np.float64).ravel()
        keep.append(a)
        p.face[int(f)] = a.ctypes.data
    p._keep = keep  # the face arrays live as long as the problem
    return p


def solve(pb: Problem, f_re: np.ndarray, f_im: np.ndarray | None = None) -> np.ndarray:
    """Return P (complex128, shape (nz, ny, nx)) as the reference leaves it."""
    n = pb.nx * pb.ny * pb.nz
    f_re = np.ascontiguousarray(f_re, dtype=np.float64).reshape(-1)
    assert f_re.size == n
    if f_im is not None:
        f_im = np.ascontiguousarray(f_im, dtype=np.float64).reshape(-1)
    out = np.zeros(2 * n, dtype=np.float64)
    rc = lib().ppo_solve(ctypes.byref(pb), _dp(f_re), _dp(f_im), _dp(out))
    if rc != 0:
        raise ValueError(f"oracle rejected the problem (code {rc})")
    return out.view(np.complex128).reshape(pb.nz, pb.ny, pb.nx)


def eigenvalue(pb: Problem, kx: int, ky: int) -> float:
    return lib().ppo_eigenvalue(ctypes.byref(pb), kx, ky)


def dft(x: np.ndarray, sign: int = -1) -> np.ndarray:
    x = np.asarray(x, dtype=np.complex128)
    re = np.ascontiguousarray(x.real)
    im = np.ascontiguousarray(x.imag)
    lib().ppo_dft(x.size, sign, _dp(re), _dp(im))
    return re + 1j * im


def manufactured(pb: Problem):
    """(f_re, f_im, u_re, u_im) of the reference's manufactured solution."""
    n = pb.nx * pb.ny * pb.nz
    arrs = [np.zeros(n) for _ in range(4)]
    lib().ppo_manufactured(ctypes.byref(pb), *[_dp(a) for a in arrs])
    return [a.reshape(pb.nz, pb.ny, pb.nx) for a in arrs]


def dirichlet_lift(pb: Problem) -> np.ndarray:
    n = pb.nx * pb.ny * pb.nz
    out = np.zeros(n)
    lib().ppo_dirichlet_lift(ctypes.byref(pb), _dp(out))
    return out.reshape(pb.nz, pb.ny, pb.nx)


def residual(pb: Problem, u: np.ndarray, b: np.ndarray) -> np.ndarray:
    """b - A u for the dz^2-scaled 7-point operator with ghost-cell BCs."""
    u = np.ascontiguousarray(u, dtype=np.float64).reshape(-1)
    b = np.ascontiguousarray(b, dtype=np.float64).reshape(-1)
    r = np.zeros_like(u)
    lib().ppo_residual(ctypes.byref(pb), _dp(u), _dp(b), _dp(r))
    return r.reshape(pb.nz, pb.ny, pb.nx)


def scaled_rhs(pb: Problem, f: np.ndarray) -> np.ndarray:
    """The right-hand side the solve inverts: f dz dz minus the Dirichlet lift."""
    dz = (pb.box[5] - pb.box[4]) / pb.nz
    b = (np.asarray(f, dtype=np.float64) * dz) * dz
    if pb.dirichlet_lift:
        b = b - dirichlet_lift(pb)
    return b


def rel_l2(a: np.ndarray, b: np.ndarray) -> float:
    a = np.asarray(a)
    b = np.asarray(b)
    den = np.linalg.norm(b.ravel())
    return float(np.linalg.norm((a - b).ravel()) / (den if den > 0 else 1.0))
