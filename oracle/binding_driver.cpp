// Driver of the reference-side binding check -- TEST INFRASTRUCTURE ONLY.
// Built by oracle/Makefile (target _ref/binding_check) against the
// reference's own headers and objects, the single-rank shims and
// libpittpack_b200.so; run by tests/test_reference_binding.py.
//
// In the order of src/main.cpp:73-134 (make_Poisson -> assignBoundary ->
// setBox -> setCoords(2) -> assignRhs) it solves one input twice: with the
// reference's own pittPack() and through PoissonB200Binding::solveOnB200(),
// and prints the binding's status and the relative L2 difference of P:
//     BINDING rc=<status> rel=<difference>
#include <cmath>
#include <cstdio>
#include <vector>

#include "poissonB200Binding.hpp"

namespace {
// read access to P for the comparison (the binding itself needs none)
struct Probe : PoissonB200Binding {
    using PoissonB200Binding::PoissonB200Binding;
    double value(int p) { return P(p); }
};
}  // namespace

int main()
{
    static char arg0[] = "binding";
    char* argv[] = {arg0, nullptr};
    const int nx = 12, ny = 10, nz = 8;
    char bc[6] = {'N', 'N', 'D', 'D', 'D', 'D'};
    double X[6] = {0, 1.0, 0, 2.0, 0, 1.0};
    std::vector<double> f(nx * ny * nz);
    for (int p = 0; p < nx * ny * nz; ++p) f[p] = std::sin(0.37 * p) + 0.25 * std::cos(1.3 * p);
    Probe R(1, argv, nx, ny, nz);  // the reference's own solve
    R.assignBoundary(bc);
    R.setBox(X);
    R.setCoords(2);
    R.assignRhs(f.data());
    R.pittPack();
    Probe M(1, argv, nx, ny, nz);  // the same input through the binding
    M.assignBoundary(bc);
    M.setBox(X);
    M.setCoords(2);
    M.assignRhs(f.data());
    const int rc = M.solveOnB200();
    double num = 0.0, den = 0.0;
    for (int p = 0; p < 2 * nx * ny * nz; ++p) {
        const double d = M.value(p) - R.value(p);
        num += d * d;
        den += R.value(p) * R.value(p);
    }
    std::printf("\nBINDING rc=%d rel=%.3e\n", rc, std::sqrt(num / den));
    return 0;
}
