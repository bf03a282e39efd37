"""The C++ facade include/PoissonB200.hpp compiles with the usage that
PittPack's own driver has (make_Poisson -> assignBoundary -> setBox ->
setCoords -> constructConnectivity / graphCreate / readIn ->
fillTrigonometric -> assignRhs -> pittPack -> getSolution -> IO -> getError;
IO must throw UNSUPPORTED) and links
against the library.  Without a GPU the run must end in a thrown
pittpack_b200::Error carrying a status code, never in a crash; with one it
solves and prints the manufactured-solution error."""
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
        try {
            M->IO(1, 2, 0);  // the HDF5 writer is not provided: must throw
            return 4;
        } catch (const pittpack_b200::Error& e) {
            if (e.code() != PP_UNSUPPORTED) return 5;
        }
        std::printf("solved err=%g\n", M->getError());
        return 0;
    } catch (const pittpack_b200::Error& e) {
        std::printf("error code=%d\n", e.code());
        return 3;
    }
}
'''


@pytest.mark.skipif(shutil.which("g++") is None, reason="no C++ compiler")
def test_facade_compiles_links_and_reports_errors(tmp_path):
    lib = os.path.join(LIBDIR, "libpittpack_b200.so")
    if not os.path.exists(lib):
        pytest.skip("library not built (python -m pittpack_b200.build)")
    src = tmp_path / "main.cpp"
    src.write_text(SRC)
    exe = tmp_path / "main"
    subprocess.run(["g++", "-std=c++17", str(src), "-I", os.path.join(ROOT, "include"), "-L", LIBDIR,
                    "-lpittpack_b200", f"-Wl,-rpath,{LIBDIR}", "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    import torch

    if torch.cuda.is_available():
        assert r.returncode == 0 and r.stdout.startswith("solved"), r.stdout + r.stderr
    else:
        assert r.returncode == 3 and r.stdout.startswith("error code="), r.stdout + r.stderr
        assert int(r.stdout.split("=")[1]) != 0
