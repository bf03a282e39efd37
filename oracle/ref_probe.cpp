// Probe driver for the single-rank reference build (oracle/_ref/libppref.so).
// TEST INFRASTRUCTURE ONLY: used by tests/golden/make_golden.py to record the
// reference's own outputs and by bench.py's "reference" arm as the CPU
// baseline.  Compiled together with the unmodified PittPack sources
// (pencilDcmp.cpp, signalProc.cpp, chunkedArray.cpp, triDiag.cpp,
// multiGrid.cpp, mathFunction.cpp, poissonCPU.cpp, poissonGPU.cpp) against the
// shims in ref_shim/.  It follows the call order of src/main.cpp:73-134:
//   make_Poisson -> assignBoundary -> setBox -> setCoords(2) -> assignRhs -> pittPack
// and reads P through ChunkedArray::operator()(int) (src/chunkedArray.cpp:240).
#include "pencilDcmp.hpp"

#include <cstring>
#include <memory>

// The HDF5 writer (src/phdf5.cpp) is not built; PencilDcmp::IO links to it
// but I_O = 0 keeps it off the solve path.
void Phdf5::writeMultiBlockCellCenter(ChunkedArray&, uint, int, int) {}

namespace {
class RefProbe : public PoissonCPU {
  public:
    RefProbe(int argc, char** argv, int nx, int ny, int nz) : PoissonCPU(argc, argv, nx, ny, nz) {}

    // imaginary part of the RHS, scaled by dz^2 like the real part
    // (assignRhs, src/pencilDcmp.cpp:5591-5647, stores only the real part)
    void assign_imag(const double* f_im)
    {
        double c3 = dxyz[2];
        long n = (long)nx * ny * nz;
        for (long p = 0; p < n; ++p) P(2 * p + 1) = f_im[p] * c3 * c3;
    }
    void read(double* out)
    {
        long n = 2L * nx * ny * nz;
        for (long p = 0; p < n; ++p) out[p] = P((int)p);
    }
    double seconds() const { return runTime; }
};
}  // namespace

extern "C" int ppref_solve(int nx, int ny, int nz, const char* bc, const double* box, const double* f_re,
                           const double* f_im, double* P_out, double* seconds)
{
    static char arg0[] = "ppref";
    char* argv[] = {arg0, nullptr};
    int argc = 1;
    std::unique_ptr<RefProbe> M(new RefProbe(argc, argv, nx, ny, nz));
    char mybc[6];
    std::memcpy(mybc, bc, 6);
    M->assignBoundary(mybc);
    double X[6];
    std::memcpy(X, box, sizeof X);
    M->setBox(X);
    M->setCoords(2);
    long n = (long)nx * ny * nz;
    double* rhs = new double[n];
    std::memcpy(rhs, f_re, sizeof(double) * n);
    M->assignRhs(rhs);
    delete[] rhs;
    if (f_im) M->assign_imag(f_im);
    M->pittPack();
    M->read(P_out);
    if (seconds) *seconds = M->seconds();
    return 0;
}

// fillTrigonometric (src/pencilDcmp.cpp:5685-5759) in the order of
// src/main.cpp:88-115: assignBoundary -> setBox -> setCoords(2) -> fill
extern "C" int ppref_fill_trigonometric(int nx, int ny, int nz, const char* bc, const double* box, double* rhs)
{
    static char arg0[] = "ppref";
    char* argv[] = {arg0, nullptr};
    int argc = 1;
    std::unique_ptr<RefProbe> M(new RefProbe(argc, argv, nx, ny, nz));
    char mybc[6];
    std::memcpy(mybc, bc, 6);
    M->assignBoundary(mybc);
    double X[6];
    std::memcpy(X, box, sizeof X);
    M->setBox(X);
    M->setCoords(2);
    M->fillTrigonometric(rhs);
    return 0;
}
