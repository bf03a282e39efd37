"""GPU parity on the benchmark's own configurations, through the C ABI.

* Configuration 1: 64^3, periodic x and y, Dirichlet z, the reference's
  periodic manufactured solution (src/pencilDcmp.cpp:1982-1986), plain FP64:
  against a golden P recorded from the reference's own CPU solve
  (tests/golden/configs, made by tests/golden/make_golden.py configs), and the
  error against the analytic solution.
* Configuration 2: 256^3, Neumann-Neumann x, Dirichlet-Dirichlet y, Neumann z,
  RHS i.i.d. U(-1, 1) (seed 1): the plain FP64 solve and the refined
  mixed-precision solve after each of 0..3 sweeps against the oracle.
* Configuration 3: 512^3 (and 256^3), each x/y family (PP, NN, ND, DD) with
  Dirichlet z, RHS a seeded sum of 8 eigenmodes plus 1e-3 noise: the plain
  FP64 solve in the reference's zero-mode semantics (the mode the benchmark
  times) against the reference's own pittPack() (PP, NN, DD) or the oracle
  (ND, which the reference does not implement); the refined solve against
  the oracle's exact-zero-mode solution.

Tolerances: relative L2 <= 1e-12 for the plain FP64 solve, <= 1e-10 for the
refined solve after one sweep.  The CPU solves run in spawned worker
processes while the GPU works (ref_jobs.py).
"""
import multiprocessing as mp
import os

import numpy as np
import pytest

import ref_jobs as J
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-12
TOL_REFINED = 1e-10
HERE = os.path.dirname(os.path.abspath(__file__))
FAMILIES = ["PPPPDD", "NNNNDD", "NDNDDD", "DDDDDD"]
SEEDS = dict(zip(FAMILIES, (3, 4, 5, 6)))


def _need_reference():
    if not os.path.exists(J.REF_LIB):
        pytest.skip("reference build oracle/_ref/libppref.so absent (make -C oracle)")


def gpu_solve(n, bc, f, **opts):
    import pittpack_b200 as pp

    with pp.make_Poisson(n, n, n) as M:
        M.assignBoundary(bc)
        M.setBox([0, 1, 0, 1, 0, 1])
        M.setCoords(2)
        if opts:
            M.setOptions(**opts)
        if np.iscomplexobj(f):
            M.assignRhsComplex(f)
        else:
            M.assignRhs(f)
        M.pittPack()
        return M.getSolution()


class CpuSolves:
    """CPU solves submitted to a spawned pool when first needed."""

    def __init__(self, specs, bytes_per_job):
        self.ctx = mp.get_context("spawn")
        self.pool = self.ctx.Pool(J.workers_for(bytes_per_job, len(specs)))
        self.res = {self.key(s): self.pool.apply_async(J.job, (s,)) for s in specs}

    @staticmethod
    def key(s):
        return (s["n"], s["bc"], s["solver"], s.get("compat", 1))

    def get(self, n, bc, solver, compat=1, timeout=1800):
        _, P = self.res[(n, bc, solver, compat)].get(timeout=timeout)
        return P

    def close(self):
        self.pool.close()
        self.pool.join()


def _cfg3_specs(n):
    specs = []
    for bc in FAMILIES:
        base = dict(n=n, bc=bc, rhs="eigenmode", seed=SEEDS[bc])
        if bc[0] == "N" and bc[1] == "D":
            # the reference has no N-D family: the oracle; no zero mode, so
            # its compat and exact solutions are the same system
            specs.append(dict(base, solver="oracle", compat=1))
        else:
            specs.append(dict(base, solver="reference"))
            specs.append(dict(base, solver="oracle", compat=0))
    return specs


@pytest.fixture(scope="module")
def cpu256():
    _need_reference()
    specs = _cfg3_specs(256) + [dict(n=256, bc="NNDDNN", rhs="uniform", seed=1, solver="oracle", compat=1)]
    s = CpuSolves(specs, 1.2e9)
    yield s
    s.close()


@pytest.fixture(scope="module")
def cpu512():
    _need_reference()
    # the reference's solves (P, R and its scratch: ~10 GB each) and the
    # oracle's N-D solve; the exact-mode oracle solves of the other families
    # are left to 256^3
    specs = [s for s in _cfg3_specs(512) if s["solver"] == "reference" or s["bc"] == "NDNDDD"]
    s = CpuSolves(specs, 12e9)
    yield s
    s.close()


def test_config1_periodic_manufactured_64_vs_reference_golden():
    z = np.load(os.path.join(HERE, "golden", "configs", "cfg1_pppp_dd_mms_64.npz"))
    n, bc = int(z["n"]), str(z["bc"])
    pb = O.problem(n, n, n, bc)
    fr, fi, ur, ui = O.manufactured(pb)
    import hashlib

    h = hashlib.sha256(np.ascontiguousarray(fr).tobytes())
    h.update(np.ascontiguousarray(fi).tobytes())
    assert h.hexdigest() == str(z["f_sha256"]), "the manufactured RHS is not the one the golden P was solved for"
    P = gpu_solve(n, bc, fr + 1j * fi)
    assert O.rel_l2(P, z["P"]) <= TOL_FP64
    # second-order discretisation error against the analytic solution
    err = np.sqrt(np.mean(np.abs(P - (ur + 1j * ui)) ** 2))
    assert err < 2e-3 * np.sqrt(np.mean(np.abs(ur + 1j * ui) ** 2))


def test_config2_nn_dd_nn_256_refined_error_per_sweep(cpu256):
    n, bc = 256, "NNDDNN"
    f = J.uniform_rhs(n, 1)
    Q = cpu256.get(n, bc, "oracle", 1)
    P = gpu_solve(n, bc, f, precision=0)
    assert O.rel_l2(P, Q) <= TOL_FP64
    errs = []
    import pittpack_b200 as pp

    with pp.make_Poisson(n, n, n) as M:
        M.assignBoundary(bc)
        M.setBox([0, 1, 0, 1, 0, 1])
        M.assignRhs(f)
        for sweeps in range(4):
            M.setOptions(precision=1, max_sweeps=sweeps, compat_zero_mode=0)
            M.pittPack()
            errs.append(O.rel_l2(M.getSolution(), Q))
    print("config 2 refined rel L2 vs oracle per sweep 0..3:", ["%.2e" % e for e in errs])
    assert errs[0] < 1e-5                 # the FP32 solve alone
    assert errs[1] <= TOL_REFINED         # one sweep reaches the target
    assert max(errs[1:]) <= TOL_REFINED


@pytest.mark.parametrize("bc", FAMILIES)
def test_config3_256_vs_reference(cpu256, bc):
    n = 256
    f = J.eigenmode_rhs(bc, n, SEEDS[bc])
    P = gpu_solve(n, bc, f, precision=0, compat_zero_mode=1)
    solver = "oracle" if bc.startswith("ND") else "reference"
    Q = cpu256.get(n, bc, solver, 1 if solver == "oracle" else 1)
    assert O.rel_l2(P, Q) <= TOL_FP64
    # the refined solve inverts the true system: exact-zero-mode oracle
    Qe = Q if bc.startswith("ND") else cpu256.get(n, bc, "oracle", 0)
    R = gpu_solve(n, bc, f, precision=1, max_sweeps=1, compat_zero_mode=0)
    assert O.rel_l2(R, Qe) <= TOL_REFINED


@pytest.mark.parametrize("bc", FAMILIES)
def test_config3_512_vs_reference(cpu512, bc):
    """The benchmark's own size, in the mode it times."""
    n = 512
    f = J.eigenmode_rhs(bc, n, SEEDS[bc])
    P = gpu_solve(n, bc, f, precision=0, compat_zero_mode=1)
    if bc.startswith("ND"):
        Q = cpu512.get(n, bc, "oracle", 1)
        assert O.rel_l2(P, Q) <= TOL_FP64
        R = gpu_solve(n, bc, f, precision=1, max_sweeps=1, compat_zero_mode=0)
        assert O.rel_l2(R, Q) <= TOL_REFINED
    else:
        Q = cpu512.get(n, bc, "reference")
        assert O.rel_l2(P, Q) <= TOL_FP64
