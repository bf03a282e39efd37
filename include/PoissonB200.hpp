// PoissonB200.hpp -- header-only C++ facade over include/pittpack_b200.h with
// the method names of PittPack's PencilDcmp (src/include/pencilDcmp.hpp:442-466),
// so a driver written like src/main.cpp needs only the factory from this
// namespace (the same call):
//
//     using pittpack_b200::make_Poisson;
//     auto M = make_Poisson(argc, argv, nx, ny, nz);
//     char bc[6] = {'N','N','N','N','D','D'};
//     M->assignBoundary(bc);
//     double X[6] = {0, 1, 0, 1, 0, 1};
//     M->setBox(X);
//     M->setCoords(2);
//     M->assignRhs(rhs);
//     M->pittPack();
//     std::cout << M->getError();
//
// Errors throw pittpack_b200::Error carrying the PittPackResult-valued code
// (the reference prints the code and exits instead).
#pragma once

#include <memory>
#include <stdexcept>
#include <string>

#include "pittpack_b200.h"

namespace pittpack_b200 {

class Error : public std::runtime_error {
  public:
    Error(int code, const std::string& what)
        : std::runtime_error(what + ": " + pp_result_string(code)), code_(code) {}
    int code() const { return code_; }

  private:
    int code_;
};

inline void check(int rc, const char* what)
{
    if (rc != PP_SUCCESS) throw Error(rc, what);
}

class PoissonB200 {
  public:
    PoissonB200(int nx, int ny, int nz) : nx_(nx), ny_(ny), nz_(nz) { check(pp_create(nx, ny, nz, &h_), "pp_create"); }
    ~PoissonB200()
    {
        if (h_) pp_destroy(h_);
    }
    PoissonB200(const PoissonB200&) = delete;
    PoissonB200& operator=(const PoissonB200&) = delete;

    void assignBoundary(const char* bc) { check(pp_assign_boundary(h_, bc), "assignBoundary"); }
    void setBox(const double X[6]) { check(pp_set_box(h_, X), "setBox"); }
    void setCoords(int /*dir*/) {}  // one rank owns the whole box
    // the reference's MPI neighbourhood and graph set-up: nothing at one rank
    int constructConnectivity() { return PP_SUCCESS; }
    void graphCreate() {}
    // the reference opens and closes PittPack.in without reading it
    void readIn() {}
    // the reference's analytic RHS, -4 pi^2 cos(2 pi z) at the cell centres
    // (src/pencilDcmp.cpp:5685-5759): nx*ny*nz doubles
    void fillTrigonometric(double* rhs) { check(pp_fill_trigonometric(h_, rhs), "fillTrigonometric"); }
    // the reference's writer: soln/Pxdmf3d<app>.xmf (XDMF, the real part of P
    // as a raw float64 Binary data item beside it; no HDF5 library needed)
    void IO(int app, int dir, int aligndir) { check(pp_io(h_, (unsigned)app, dir, aligndir), "IO"); }
    void setOptions(const pp_options& o) { check(pp_set_options(h_, &o), "setOptions"); }
    pp_options options() const
    {
        pp_options o;
        check(pp_get_options(h_, &o), "options");
        return o;
    }
    // boundary data of one face (0..5 = xmin .. zmax), see pp_set_face_values;
    // nullptr clears it
    void setFaceValues(int face, const double* g) { check(pp_set_face_values(h_, face, g), "setFaceValues"); }
    void assignRhs(const double* rhs) { check(pp_assign_rhs(h_, rhs), "assignRhs"); }
    void assignRhsComplex(const double* rhs) { check(pp_assign_rhs_complex(h_, rhs), "assignRhsComplex"); }
    void pittPack() { check(pp_solve(h_), "pittPack"); }
    // P in the chunkedArray layout: 2*nx*ny*nz doubles
    void getSolution(double* P) { check(pp_get_solution(h_, P), "getSolution"); }
    // the real part alone (nx*ny*nz doubles): half the bytes, for a real RHS
    void getSolutionReal(double* u) { check(pp_get_solution_real(h_, u), "getSolutionReal"); }
    double getError()
    {
        double e = 0.0;
        check(pp_get_error_manufactured(h_, &e), "getError");
        return e;
    }
    pp_handle handle() const { return h_; }
    int nx() const { return nx_; }
    int ny() const { return ny_; }
    int nz() const { return nz_; }

  private:
    pp_handle h_ = nullptr;
    int nx_, ny_, nz_;
};

// the reference's factory, src/pencilDcmp.cpp:6432-6440
inline std::unique_ptr<PoissonB200> make_Poisson(int nx, int ny, int nz)
{
    return std::unique_ptr<PoissonB200>(new PoissonB200(nx, ny, nz));
}
// with the reference's signature: argc / argv only fed MPI_Init there
// (src/pencilDcmp.cpp:232-452); one rank needs neither
inline std::unique_ptr<PoissonB200> make_Poisson(int /*argc*/, char** /*argv*/, int nx, int ny, int nz)
{
    return make_Poisson(nx, ny, nz);
}

}  // namespace pittpack_b200
