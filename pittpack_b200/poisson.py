"""Host-side mirror of PittPack's PencilDcmp / PoissonGPU interface.

The method names and their order of use follow the reference
(src/include/pencilDcmp.hpp:442-522, driven as in src/main.cpp:73-134):

    M = make_Poisson(nx, ny, nz)      # make_Poisson, src/pencilDcmp.cpp:6432-6440
    M.assignBoundary("NNNNDD")        # src/pencilDcmp.cpp:3578-3634
    M.setBox([0, 1, 0, 1, 0, 1])      # src/pencilDcmp.cpp:470-480
    M.setCoords(2)                    # single rank: the box is the whole grid
    M.assignRhs(rhs)                  # src/pencilDcmp.cpp:5591-5647
    M.pittPack()                      # src/pencilDcmp.cpp:5801-6430, one solve
    M.getError()                      # src/pencilDcmp.cpp:2040-2208 (non-destructive here)
    P = M.getSolution()               # the chunkedArray P, complex (nz, ny, nx)

Every call goes through the C ABI of libpittpack_b200.so; errors raise
PittPackError with the reference's PittPackResult code instead of exiting.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import Options, PittPackError, check


class PoissonGPU:
    """One nx*ny*nz grid on the current CUDA device."""

    def __init__(self, nx: int, ny: int, nz: int):
        L = _lib.load()
        self._L = L
        self.nx, self.ny, self.nz = int(nx), int(ny), int(nz)
        h = ctypes.c_void_p()
        check(L.pp_create(self.nx, self.ny, self.nz, ctypes.byref(h)), "pp_create")
        self._h = h
        self._box = np.array([0.0, 1.0, 0.0, 1.0, 0.0, 1.0])
        self.bc = None

    # -- set-up -------------------------------------------------------------
    def assignBoundary(self, bc) -> None:
        b = bc.encode() if isinstance(bc, str) else bytes(bc)
        if len(b) != 6:
            raise PittPackError(_lib.PP_INPUT_ARGS, "assignBoundary needs 6 letters")
        check(self._L.pp_assign_boundary(self._h, b), "assignBoundary")
        self.bc = b.decode()

    def setFaceValues(self, face: int, g) -> None:
        """Boundary data of one face (0..5 = xmin, xmax, ymin, ymax, zmin,
        zmax): the value on a Dirichlet face, the outward normal derivative on
        a Neumann face, at the face's cell centres -- shape (nz, ny) for x
        faces, (nz, nx) for y faces, (ny, nx) for z faces; None clears it."""
        if g is None:
            check(self._L.pp_set_face_values(self._h, int(face), None), "setFaceValues")
            return
        if not 0 <= int(face) < 6:
            raise PittPackError(_lib.PP_INPUT_ARGS, f"setFaceValues: face {face} is not 0..5")
        shape = [(self.nz, self.ny), (self.nz, self.nx), (self.ny, self.nx)][int(face) // 2]
        a = np.ascontiguousarray(g, dtype=np.float64)
        if a.size != shape[0] * shape[1]:
            raise PittPackError(_lib.PP_INPUT_ARGS, f"setFaceValues: face {face} needs {shape} values")
        check(self._L.pp_set_face_values(self._h, int(face), a.ctypes.data), "setFaceValues")

    def setBox(self, X) -> None:
        x = np.ascontiguousarray(X, dtype=np.float64)
        if x.size != 6:
            raise PittPackError(_lib.PP_INPUT_ARGS, "setBox needs 6 values")
        check(self._L.pp_set_box(self._h, x.ctypes.data_as(ctypes.POINTER(ctypes.c_double))), "setBox")
        self._box = x.copy()

    def setCoords(self, dir: int = 2) -> None:  # noqa: A002 - the reference's name
        """Single rank: the rank's box is the whole box; nothing to do."""

    def constructConnectivity(self) -> int:
        """The reference's MPI neighbourhood set-up
        (src/pencilDcmp.cpp:851): nothing to connect at one rank."""
        return _lib.PP_SUCCESS

    def graphCreate(self) -> None:
        """The reference's MPI graph communicators (src/pencilDcmp.cpp:1274):
        none at one rank."""

    def readIn(self) -> None:
        """The reference opens and closes PittPack.in without reading it
        (src/pencilDcmp.cpp:5790-5796); nothing to do."""

    def fillTrigonometric(self, rhs: np.ndarray | None = None) -> np.ndarray:
        """The reference's analytic RHS (src/pencilDcmp.cpp:5685-5759):
        f = -4 pi^2 cos(2 pi z) at the cell centres of the box, shape
        (nz, ny, nx); fills 'rhs' (contiguous float64) when given."""
        if rhs is None:
            rhs = np.empty((self.nz, self.ny, self.nx))
        if not (isinstance(rhs, np.ndarray) and rhs.dtype == np.float64 and rhs.flags.c_contiguous
                and rhs.size == self.nx * self.ny * self.nz):
            raise PittPackError(_lib.PP_INPUT_ARGS, "fillTrigonometric needs a contiguous float64 array of nx*ny*nz")
        box = np.ascontiguousarray(self._box, dtype=np.float64)
        check(self._L.pp_fill_trigonometric_box(self.nx, self.ny, self.nz,
                                                box.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), rhs.ctypes.data),
              "fillTrigonometric")
        return rhs

    def IO(self, app: int = 1, dir: int = 2, aligndir: int = 0) -> None:  # noqa: A002 - the reference's names
        """The reference's writer (src/pencilDcmp.cpp:1827-1832): the real part
        of P as soln/Pxdmf3d<app>.xmf with a raw float64 data file beside it
        (XDMF Binary item; no HDF5 library needed)."""
        check(self._L.pp_io(self._h, int(app), int(dir), int(aligndir)), "IO")

    def options(self) -> Options:
        o = Options()
        check(self._L.pp_get_options(self._h, ctypes.byref(o)), "pp_get_options")
        return o

    def setOptions(self, **kw) -> None:
        o = self.options()
        for k, v in kw.items():
            if not hasattr(o, k):
                raise TypeError(f"unknown option {k}")
            setattr(o, k, v)
        check(self._L.pp_set_options(self._h, ctypes.byref(o)), "pp_set_options")

    # -- data ---------------------------------------------------------------
    def _shape_ok(self, a: np.ndarray, n: int) -> np.ndarray:
        a = np.ascontiguousarray(a)
        if a.size != n:
            raise PittPackError(_lib.PP_INPUT_ARGS, f"expected {n} values, got {a.size}")
        return a

    def assignRhs(self, rhs) -> None:
        """Real RHS f (x fastest); the solve multiplies it by dz^2 like the reference."""
        n = self.nx * self.ny * self.nz
        if np.iscomplexobj(rhs):
            return self.assignRhsComplex(rhs)
        a = self._shape_ok(np.asarray(rhs, dtype=np.float64), n)
        check(self._L.pp_assign_rhs(self._h, a.ctypes.data), "assignRhs")

    def assignRhsComplex(self, rhs) -> None:
        n = self.nx * self.ny * self.nz
        a = self._shape_ok(np.asarray(rhs, dtype=np.complex128), n)
        check(self._L.pp_assign_rhs_complex(self._h, a.ctypes.data), "assignRhsComplex")

    def assignRhsDevice(self, ptr: int, is_complex: bool = False) -> None:
        check(self._L.pp_assign_rhs_device(self._h, ctypes.c_void_p(ptr), int(is_complex)), "assignRhsDevice")

    # -- solve --------------------------------------------------------------
    def pittPack(self) -> None:
        check(self._L.pp_solve(self._h), "pittPack")

    solve = pittPack

    STAGES = ("x_forward", "y_forward", "z_solve", "y_inverse", "x_inverse", "residual")

    def profileSolve(self) -> np.ndarray:
        """One solve with per-stage CUDA-event times (ms), in the order of
        STAGES (the residual stage exists only in the refined solve)."""
        ms = np.zeros(6)
        check(self._L.pp_profile_solve(self._h, ms.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), 6),
              "pp_profile_solve")
        return ms

    def timingBegin(self, max_solves: int) -> None:
        check(self._L.pp_timing_begin(self._h, int(max_solves)), "pp_timing_begin")

    def timingEnd(self):
        """(summed ms per stage [6, order of STAGES], number of solves recorded)."""
        ms = np.zeros(6)
        n = ctypes.c_int()
        check(self._L.pp_timing_end(self._h, ms.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), 6,
                                    ctypes.byref(n)), "pp_timing_end")
        return ms, n.value

    def getSolution(self, out: np.ndarray | None = None) -> np.ndarray:
        """P as complex (nz, ny, nx); 'out' may be a preallocated (pinned) array."""
        if out is None:
            out = np.empty((self.nz, self.ny, self.nx), dtype=np.complex128)
        if out.dtype != np.complex128 or out.size != self.nx * self.ny * self.nz or not out.flags.c_contiguous:
            raise PittPackError(_lib.PP_INPUT_ARGS, "getSolution needs a contiguous complex128 array")
        check(self._L.pp_get_solution(self._h, out.ctypes.data), "getSolution")
        return out

    def solutionToDevice(self, dptr: int) -> None:
        """Copy P (2*nx*ny*nz doubles) to device memory at dptr, on the solver's stream."""
        check(self._L.pp_get_solution_device(self._h, ctypes.c_void_p(dptr)), "pp_get_solution_device")

    def solutionDevicePtr(self) -> int:
        p = ctypes.c_void_p()
        check(self._L.pp_solution_device_ptr(self._h, ctypes.byref(p)), "pp_solution_device_ptr")
        return int(p.value)

    def getError(self) -> float:
        e = ctypes.c_double()
        check(self._L.pp_get_error_manufactured(self._h, ctypes.byref(e)), "getError")
        return e.value

    def zsolveStats(self):
        """Multigrid z solver: (most V-cycles of any system, systems stopped
        at the cycle bound above 1e-10) for the last solve."""
        c, u = ctypes.c_int(), ctypes.c_int()
        check(self._L.pp_zsolve_stats(self._h, ctypes.byref(c), ctypes.byref(u)), "pp_zsolve_stats")
        return c.value, u.value

    # -- zero copy, asynchronous copies, launch shapes --------------------------
    def bindDeviceBuffers(self, d_rhs: int = 0, is_complex: bool = False, d_P: int = 0) -> None:
        """Solve straight from / into caller-owned device buffers (pointers as
        ints, 0 keeps the handle's own buffer)."""
        check(self._L.pp_bind_device_buffers(self._h, ctypes.c_void_p(d_rhs or None), int(bool(is_complex)),
                                             ctypes.c_void_p(d_P or None)), "pp_bind_device_buffers")

    def assignRhsAsync(self, rhs: np.ndarray) -> None:
        """Real RHS copied on the handle's stream without waiting; keep rhs
        alive and unchanged until the stream has passed the next solve."""
        if not (isinstance(rhs, np.ndarray) and rhs.dtype == np.float64 and rhs.flags.c_contiguous
                and rhs.size == self.nx * self.ny * self.nz):
            raise PittPackError(_lib.PP_INPUT_ARGS, "assignRhsAsync needs a contiguous float64 array of nx*ny*nz")
        check(self._L.pp_assign_rhs_async(self._h, rhs.ctypes.data), "pp_assign_rhs_async")

    def getSolutionAsync(self, out: np.ndarray) -> None:
        """Solution copied into out (complex128, nx*ny*nz) on the handle's
        stream without waiting; synchronize() before reading it."""
        if not (isinstance(out, np.ndarray) and out.dtype == np.complex128 and out.flags.c_contiguous
                and out.size == self.nx * self.ny * self.nz):
            raise PittPackError(_lib.PP_INPUT_ARGS, "getSolutionAsync needs a contiguous complex128 array of nx*ny*nz")
        check(self._L.pp_get_solution_async(self._h, out.ctypes.data), "pp_get_solution_async")

    def kernelTimeouts(self) -> int:
        """Thread blocks whose bounded wait for their bulk-copied tile ran out
        (0 unless the copy engine failed; each such block wrote no output)."""
        c = ctypes.c_int()
        check(self._L.pp_kernel_timeouts(self._h, ctypes.byref(c)), "pp_kernel_timeouts")
        return c.value

    def getSolutionReal(self, out: np.ndarray | None = None) -> np.ndarray:
        """The real part of the solution alone (float64, shape (nz, ny, nx)):
        half the bytes of getSolution, for a real RHS (whose solution has a
        zero imaginary part)."""
        n = self.nx * self.ny * self.nz
        if out is None:
            out = np.empty((self.nz, self.ny, self.nx), dtype=np.float64)
        if not (isinstance(out, np.ndarray) and out.dtype == np.float64 and out.flags.c_contiguous and out.size == n):
            raise PittPackError(_lib.PP_INPUT_ARGS, "getSolutionReal needs a contiguous float64 array of nx*ny*nz")
        check(self._L.pp_get_solution_real(self._h, out.ctypes.data), "pp_get_solution_real")
        return out

    def getSolutionRealAsync(self, out: np.ndarray) -> None:
        """getSolutionReal on the handle's stream without waiting (out
        page-locked for an asynchronous copy); synchronize() before reading it."""
        if not (isinstance(out, np.ndarray) and out.dtype == np.float64 and out.flags.c_contiguous
                and out.size == self.nx * self.ny * self.nz):
            raise PittPackError(_lib.PP_INPUT_ARGS, "getSolutionRealAsync needs a contiguous float64 array of nx*ny*nz")
        check(self._L.pp_get_solution_real_async(self._h, out.ctypes.data), "pp_get_solution_real_async")

    def setTuning(self, zsolve_lanes: int = 0, line_tile: int = 0, zsolve_tile: int = 0) -> None:
        t = _lib.Tuning(int(zsolve_lanes), int(line_tile), int(zsolve_tile))
        check(self._L.pp_set_tuning(self._h, ctypes.byref(t)), "pp_set_tuning")

    def tuning(self):
        t = _lib.Tuning()
        check(self._L.pp_get_tuning(self._h, ctypes.byref(t)), "pp_get_tuning")
        return {"zsolve_lanes": t.zsolve_lanes, "line_tile": t.line_tile, "zsolve_tile": t.zsolve_tile}

    def autotune(self, reps: int = 3):
        """Time candidate launch shapes on the assigned RHS and keep the
        fastest; returns (shape dict, ms per solve)."""
        t = _lib.Tuning()
        ms = ctypes.c_double()
        check(self._L.pp_autotune(self._h, int(reps), ctypes.byref(t), ctypes.byref(ms)), "pp_autotune")
        return {"zsolve_lanes": t.zsolve_lanes, "line_tile": t.line_tile, "zsolve_tile": t.zsolve_tile}, ms.value

    def setStream(self, stream_ptr: int) -> None:
        check(self._L.pp_set_stream(self._h, ctypes.c_void_p(stream_ptr)), "pp_set_stream")

    def synchronize(self) -> None:
        check(self._L.pp_synchronize(self._h), "pp_synchronize")

    def workspaceBytes(self) -> int:
        b = ctypes.c_size_t()
        check(self._L.pp_workspace_bytes(self._h, ctypes.byref(b)), "pp_workspace_bytes")
        return int(b.value)

    # -- lifetime -----------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            self._L.pp_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def pinned_empty(shape, dtype=np.float64) -> np.ndarray:
    """A numpy array in page-locked host memory (pp_host_alloc), freed with the array."""
    L = _lib.load()
    dt = np.dtype(dtype)
    nbytes = int(np.prod(shape)) * dt.itemsize
    p = ctypes.c_void_p()
    check(L.pp_host_alloc(max(nbytes, 1), ctypes.byref(p)), "pp_host_alloc")
    buf = (ctypes.c_char * max(nbytes, 1)).from_address(p.value)
    arr = np.frombuffer(buf, dtype=dt, count=int(np.prod(shape))).reshape(shape)

    class _Owner:
        def __init__(self, ptr):
            self.ptr = ptr

        def __del__(self):
            try:
                L.pp_host_free(ctypes.c_void_p(self.ptr))
            except Exception:
                pass

    # keep the allocation alive as long as the array (or views of it) live
    holder = _Owner(p.value)
    arr = arr.view(_PinnedArray)
    arr._pp_owner = holder
    return arr


class _PinnedArray(np.ndarray):
    def __array_finalize__(self, obj):
        if obj is not None:
            self._pp_owner = getattr(obj, "_pp_owner", None)


def make_Poisson(nx: int, ny: int, nz: int) -> PoissonGPU:
    """The reference's factory (src/pencilDcmp.cpp:6432-6440); always the GPU solver."""
    return PoissonGPU(nx, ny, nz)
