"""Record golden input/output vectors from the reference's own CPU solve.

Run in a tree that has the PittPack sources (default /root/reference):
    make -C oracle && python tests/golden/make_golden.py
It loads oracle/_ref/libppref.so -- the reference's unmodified
pencilDcmp/signalProc/triDiag/chunkedArray/poissonCPU sources built against
single-rank MPI/FFTW shims by oracle/Makefile -- runs PencilDcmp::pittPack()
once per case and stores (bc, box, sizes, RHS, P) in tests/golden/*.npz.
The RHS is seeded (numpy default_rng) so the inputs can be regenerated; they
are stored anyway so the fixtures stand alone.

The cases in ZM_CASES go to tests/golden/zero_mean/: the same sources built
with the reference's ZERO_MEAN switch on (oracle/_ref/libppref_zm.so), whose
solve ends with subtractMeanValue (src/pencilDcmp.cpp:5649-5683).
    python tests/golden/make_golden.py zero_mean    # only that set
"""
import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
LIB = os.path.join(ROOT, "oracle", "_ref", "libppref.so")
LIB_ZM = os.path.join(ROOT, "oracle", "_ref", "libppref_zm.so")

# (name, nx, ny, nz, bc, box, complex rhs, rhs kind)
CASES = [
    ("pp_pp_dd_mms", 16, 16, 16, "PPPPDD", (0, 1, 0, 1, 0, 1), True, "mms"),
    ("nn_nn_dd_mms", 16, 12, 10, "NNNNDD", (0, 1, 0, 1, 0, 1), False, "mms"),
    ("dd_dd_dd_mms", 12, 16, 8, "DDDDDD", (0, 1, 0, 1, 0, 1), False, "mms"),
    ("nn_dd_nn_rand", 16, 8, 12, "NNDDNN", (0, 1, 0, 1, 0, 1), False, "rand"),
    ("dd_nn_nd_rand", 10, 12, 9, "DDNNND", (-1, 1, 0, 2, 0.5, 1.5), False, "rand"),
    ("pp_pp_pp_rand", 8, 12, 6, "PPPPPP", (0, 1, 0, 1, 0, 1), True, "rand0"),
    ("dd_pp_nn_rand", 12, 10, 9, "DDPPNN", (0, 2, 0, 1, 0, 1), False, "rand"),
    ("nn_pp_pp_rand", 9, 8, 10, "NNPPPP", (0, 1, 0, 1, 0, 1), False, "rand0"),
    ("nn_nn_nn_rand", 12, 10, 8, "NNNNNN", (0, 1, 0, 1, 0, 1), False, "rand0"),
    ("pp_pp_nn_rand", 15, 9, 7, "PPPPNN", (0, 1, 0, 3, 0, 1), True, "rand0"),
    ("dd_dd_pp_rand", 6, 10, 16, "DDDDPP", (0, 1, 0, 1, 0, 1), False, "rand"),
    ("pp_pp_dn_rand", 20, 18, 5, "PPPPDN", (0, 1, 0, 1, 0, 1), True, "rand"),
    ("pp_nn_dd_quirk", 8, 8, 8, "PPNNDD", (0, 1, 0, 1, 0, 1), False, "rand"),
    ("nn_dd_dd_mixed", 30, 24, 20, "NNDDDD", (0, 1, 0, 1, 0, 1), False, "rand"),
]

# ZERO_MEAN build; "pos" draws f from U(0, 1), so that the solution's mean is
# far from zero and its subtraction is visible
ZM_CASES = [
    ("nn_nn_nn_zm", 12, 10, 8, "NNNNNN", (0, 1, 0, 1, 0, 1), False, "rand0"),
    ("pp_pp_pp_zm", 8, 12, 6, "PPPPPP", (0, 1, 0, 1, 0, 1), True, "rand0"),
    ("nn_dd_dd_zm_pos", 16, 8, 12, "NNDDDD", (0, 1, 0, 2, 0, 1), False, "pos"),
    ("dd_nn_nd_zm", 10, 12, 9, "DDNNND", (-1, 1, 0, 2, 0.5, 1.5), False, "rand"),
]


def _manufactured(nx, ny, nz, bc, box):
    sys.path.insert(0, ROOT)
    from oracle import oracle as O

    return O.manufactured(O.problem(nx, ny, nz, bc, box))


def record(lib, cases, outdir, seed0):
    L = ctypes.CDLL(lib)
    dp = ctypes.POINTER(ctypes.c_double)
    L.ppref_solve.argtypes = [ctypes.c_int] * 3 + [ctypes.c_char_p, dp, dp, dp, dp, dp]
    os.makedirs(outdir, exist_ok=True)
    for idx, (name, nx, ny, nz, bc, box, cplx, kind) in enumerate(cases):
        rng = np.random.default_rng(seed0 + idx)
        shape = (nz, ny, nx)
        if kind == "mms":
            fr, fi, _, _ = _manufactured(nx, ny, nz, bc, box)
            if not cplx:
                fi = None
        elif kind == "pos":
            fr = rng.uniform(0, 1, shape)
            fi = rng.uniform(0, 1, shape) if cplx else None
        else:
            fr = rng.uniform(-1, 1, shape)
            fi = rng.uniform(-1, 1, shape) if cplx else None
            if kind == "rand0":  # compatible RHS for the singular families
                fr -= fr.mean()
                if fi is not None:
                    fi -= fi.mean()
        fr = np.ascontiguousarray(fr)
        out = np.zeros(2 * nx * ny * nz)
        b = np.array(box, dtype=np.float64)
        sec = ctypes.c_double()
        L.ppref_solve(nx, ny, nz, bc.encode(), b.ctypes.data_as(dp), fr.ctypes.data_as(dp),
                      None if fi is None else np.ascontiguousarray(fi).ctypes.data_as(dp),
                      out.ctypes.data_as(dp), ctypes.byref(sec))
        np.savez_compressed(
            os.path.join(outdir, name + ".npz"),
            nx=nx, ny=ny, nz=nz, bc=bc, box=b, f_re=fr,
            f_im=(fi if fi is not None else np.zeros(0)),
            P=out.view(np.complex128).reshape(shape),
        )
        print(name, "done", file=sys.stderr)


def main(argv):
    if "zero_mean" not in argv:
        record(LIB, CASES, HERE, 1000)
    record(LIB_ZM, ZM_CASES, os.path.join(HERE, "zero_mean"), 2000)


if __name__ == "__main__":
    main(sys.argv[1:])
