"""CPU solves of the benchmark configurations for the parity tests -- TEST
INFRASTRUCTURE ONLY.

The reference's own CPU path (oracle/_ref/libppref.so: PencilDcmp::pittPack
of the PittPack sources built single-rank by oracle/Makefile) and the oracle
restatement (oracle/pp_oracle.c) take from seconds (256^3) to a couple of
minutes (512^3) per solve on one core, so the tests run them in spawned worker
processes (started with "spawn": the test process has a CUDA context) while
the GPU solves the same inputs.  The RHS generators are deterministic, so a
worker rebuilds its input from the job's description instead of receiving it.
"""
from __future__ import annotations

import ctypes
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libppref.so")


def mode1d(pair: str, k: int, phase: int, c: np.ndarray) -> np.ndarray:
    """An eigenmode of a boundary pair on cell centres c in (0, 1)."""
    if pair == "PP":
        return np.cos(2 * np.pi * k * c) if phase == 0 else np.sin(2 * np.pi * k * c)
    if pair == "NN":
        return np.cos(np.pi * k * c)
    if pair == "DD":
        return np.sin(np.pi * (k + 1) * c)
    if pair == "ND":
        return np.cos(np.pi * (k + 0.5) * c)
    return np.sin(np.pi * (k + 0.5) * c)  # DN


def eigenmode_rhs(bc: str, n: int, seed: int) -> np.ndarray:
    """The 512^3 benchmark's RHS: a sum of 8 eigenmodes of the boundary set
    with integer wavenumbers below n/4 and N(0,1) amplitudes, plus 1e-3
    uniform noise; shape (n, n, n) = (z, y, x)."""
    rng = np.random.default_rng(seed)
    amps = rng.standard_normal(8)
    waves = rng.integers(0, n // 4, (8, 3))
    phase = rng.integers(0, 2, (8, 2))
    c = (np.arange(n) + 0.5) / n
    f = np.zeros((n, n, n))
    for m in range(8):
        mx = mode1d(bc[0:2], int(waves[m, 0]), int(phase[m, 0]), c)
        my = mode1d(bc[2:4], int(waves[m, 1]), int(phase[m, 1]), c)
        mz = mode1d(bc[4:6], int(waves[m, 2]), 0, c)
        f += amps[m] * mz[:, None, None] * (my[:, None] * mx[None, :])[None, :, :]
    f += rng.uniform(-1, 1, f.shape) * 1e-3
    return f


def uniform_rhs(n: int, seed: int) -> np.ndarray:
    """i.i.d. U(-1, 1), shape (n, n, n)."""
    return np.random.default_rng(seed).uniform(-1, 1, (n, n, n))


def make_rhs(spec: dict) -> np.ndarray:
    if spec["rhs"] == "eigenmode":
        return eigenmode_rhs(spec["bc"], spec["n"], spec["seed"])
    return uniform_rhs(spec["n"], spec["seed"])


def reference_solve(n: int, bc: str, f: np.ndarray) -> np.ndarray:
    """PencilDcmp::pittPack of the reference's CPU sources on the unit box
    (the FFTW calls served by the shim's FP64 mixed-radix DFT)."""
    os.environ["PP_SHIM_FFT"] = "fast"
    L = ctypes.CDLL(REF_LIB)
    dp = ctypes.POINTER(ctypes.c_double)
    L.ppref_solve.argtypes = [ctypes.c_int] * 3 + [ctypes.c_char_p, dp, dp, dp, dp, dp]
    f = np.ascontiguousarray(f, dtype=np.float64)
    out = np.zeros(2 * f.size)
    box = np.array([0, 1, 0, 1, 0, 1.0])
    sec = ctypes.c_double()
    # the reference prints its set-up; keep it off the test output
    fd = os.dup(1)
    nul = os.open(os.devnull, os.O_WRONLY)
    os.dup2(nul, 1)
    try:
        L.ppref_solve(n, n, n, bc.encode(), box.ctypes.data_as(dp), f.ctypes.data_as(dp), None,
                      out.ctypes.data_as(dp), ctypes.byref(sec))
    finally:
        os.dup2(fd, 1)
        os.close(fd)
        os.close(nul)
    return out.view(np.complex128).reshape(n, n, n)


def oracle_solve(n: int, bc: str, f: np.ndarray, compat: int) -> np.ndarray:
    if ROOT not in sys.path:
        sys.path.insert(0, ROOT)
    from oracle import oracle as O

    return O.solve(O.problem(n, n, n, bc, compat_zero_mode=compat), f)


def job(spec: dict):
    """One CPU solve: spec = {n, bc, rhs, seed, solver: "reference" | "oracle",
    compat}.  Returns (spec, P) with P complex128 (z, y, x)."""
    f = make_rhs(spec)
    if spec["solver"] == "reference":
        P = reference_solve(spec["n"], spec["bc"], f)
    else:
        P = oracle_solve(spec["n"], spec["bc"], f, spec.get("compat", 1))
    return spec, P


def long_line_rhs(nx: int, ny: int, nz: int, bc: str):
    """The long-line parity cases' RHS: N(0, 1) (seed nx ny), complex for a
    periodic x direction; (real, imaginary or None)."""
    rng = np.random.default_rng(nx * ny)
    fr = rng.standard_normal((nz, ny, nx))
    fi = rng.standard_normal((nz, ny, nx)) if bc[0] == "P" else None
    return fr, fi


def long_line_oracle(nx: int, ny: int, nz: int, bc: str, compat: int, cells: bool):
    """The oracle's solution of a long-line case (unit box, or unit cells)."""
    if ROOT not in sys.path:
        sys.path.insert(0, ROOT)
    from oracle import oracle as O

    fr, fi = long_line_rhs(nx, ny, nz, bc)
    box = (0, nx, 0, ny, 0, nz) if cells else (0, 1, 0, 1, 0, 1)
    return O.solve(O.problem(nx, ny, nz, bc, box=box, compat_zero_mode=compat), fr, fi)


def workers_for(bytes_per_job: float, jobs: int) -> int:
    """Worker processes that fit the host's free memory (and cores)."""
    try:
        import psutil

        avail = psutil.virtual_memory().available
    except Exception:
        avail = 16e9
    by_mem = int(max(1, (avail * 0.6) // max(bytes_per_job, 1)))
    return max(1, min(jobs, by_mem, os.cpu_count() or 1))
