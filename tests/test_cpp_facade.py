"""The C++ facade include/PoissonB200.hpp compiles with the usage that
PittPack's own driver has (make_Poisson -> assignBoundary -> setBox ->
setCoords -> constructConnectivity / graphCreate / readIn ->
fillTrigonometric -> assignRhs -> pittPack -> getSolution -> IO -> getError;
IO must throw UNSUPPORTED) and links
against the library.  Without a GPU the run must end in a thrown
pittpack_b200::Error carrying a status code, never in a crash; on a GPU it
solves, and the solution it writes out (with the RHS it solved) equals the
oracle's solve of the same problem -- caller face values on z-min, the
zero-mean option -- to 1e-12 relative L2."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "pittpack_b200")

SRC = r'''
#include <cstdio>
#include <vector>
#include "PoissonB200.hpp"

// argv[1] (optional): file that receives the RHS and then P, as raw doubles
static void dump(const char* path, const std::vector<double>& a, const std::vector<double>& b) {
    if (!path) return;
    FILE* f = std::fopen(path, "wb");
    if (!f) return;
    std::fwrite(a.data(), sizeof(double), a.size(), f);
    std::fwrite(b.data(), sizeof(double), b.size(), f);
    std::fclose(f);
}

int main(int argc, char* argv[]) {
    const int Nx = 16, Ny = 16, Nz = 8;
    std::vector<double> rhs(Nx * Ny * Nz, 1.0);
    try {
        using pittpack_b200::make_Poisson;
        auto M = make_Poisson(argc, argv, Nx, Ny, Nz);  // the reference's call
        char mybc[6] = {'N', 'N', 'N', 'N', 'D', 'D'};
        M->assignBoundary(mybc);
        double X[6] = {0, 1.0, 0, 1.0, 0, 1.0};
        M->setBox(X);
        M->setCoords(2);
        M->constructConnectivity();
        M->graphCreate();
        M->readIn();
        M->fillTrigonometric(rhs.data());  // the reference driver's RHS
        pp_options o = M->options();
        o.zero_mean = 1;
        M->setOptions(o);
        std::vector<double> g(Nx * Ny, 0.25);
        M->setFaceValues(4, g.data());
        M->assignRhs(rhs.data());
        M->pittPack();
        std::vector<double> P(2 * Nx * Ny * Nz);
        M->getSolution(P.data());
        dump(argc > 1 ? argv[1] : nullptr, rhs, P);
        M->IO(1, 2, 0);  // soln/Pxdmf3d1.xmf + soln/Pxdmf3d1_Q.bin in the working directory
        std::printf("solved err=%g\n", M->getError());
        return 0;
    } catch (const pittpack_b200::Error& e) {
        std::printf("error code=%d\n", e.code());
        return 3;
    }
}
'''


def _build(tmp_path):
    if shutil.which("g++") is None:
        pytest.skip("no C++ compiler")
    lib = os.path.join(LIBDIR, "libpittpack_b200.so")
    if not os.path.exists(lib):
        pytest.skip("library not built (python -m pittpack_b200.build)")
    src = tmp_path / "main.cpp"
    src.write_text(SRC)
    exe = tmp_path / "main"
    subprocess.run(["g++", "-std=c++17", str(src), "-I", os.path.join(ROOT, "include"), "-L", LIBDIR,
                    "-lpittpack_b200", f"-Wl,-rpath,{LIBDIR}", "-o", str(exe)], check=True)
    return exe


def test_facade_compiles_links_and_reports_errors(tmp_path):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present: test_facade_solves_on_gpu covers this machine")
    exe = _build(tmp_path)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 3 and r.stdout.startswith("error code="), r.stdout + r.stderr
    assert int(r.stdout.split("=")[1]) != 0


@pytest.mark.gpu
def test_facade_solves_on_gpu(tmp_path):
    import numpy as np

    from oracle import oracle as O

    exe = _build(tmp_path)
    out = tmp_path / "dump.bin"
    r = subprocess.run([str(exe), str(out)], capture_output=True, text=True, timeout=120, cwd=str(tmp_path))
    assert r.returncode == 0 and r.stdout.startswith("solved"), r.stdout + r.stderr
    nx, ny, nz = 16, 16, 8
    raw = np.fromfile(out, dtype=np.float64)
    n = nx * ny * nz
    rhs, P = raw[:n].reshape(nz, ny, nx), raw[n:].view(np.complex128).reshape(nz, ny, nx)
    # IO() wrote the real part of P beside its XDMF file
    assert (tmp_path / "soln" / "Pxdmf3d1.xmf").exists()
    assert np.array_equal(np.fromfile(tmp_path / "soln" / "Pxdmf3d1_Q.bin", dtype="<f8").reshape(nz, ny, nx), P.real)
    pb = O.problem(nx, ny, nz, "NNNNDD", faces={4: np.full((ny, nx), 0.25)}, zero_mean=1)
    assert O.rel_l2(P, O.solve(pb, rhs)) <= 1e-12
