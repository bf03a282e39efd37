// Reference-side binding: a PittPack source file a maintainer adds to the
// PittPack tree (next to src/include/pencilDcmp.hpp) to keep PencilDcmp --
// its RHS set-up, its HDF5 output, its driver -- and hand only the solve to
// the B200 library through the C ABI of pittpack_b200.h.
//
// It replaces PencilDcmp::pittPack() (src/pencilDcmp.cpp:5801-6430) at one
// rank (p0 = 1), where P (ChunkedArray, src/chunkedArray.cpp:100-199) is the
// whole grid in the chunkedArray layout.  assignRhs (src/pencilDcmp.cpp:
// 5591-5647) has left f dz^2 in P; the library takes the unscaled RHS.  The
// library's default options are the reference's semantics: modifyRhsDirichlet
// (src/pencilDcmp.cpp:4623-4835) and the zero-mode row replacement
// (src/triDiag.cpp:1753-1776) run inside pp_solve.
//
// solveOnB200() returns a PittPackResult-valued status (0 = success), never
// exits; P keeps its previous contents when a call fails.
#pragma once

#include <vector>

#include "pencilDcmp.hpp"
#include "pittpack_b200.h"

class PoissonB200Binding : public PoissonCPU {
  public:
    using PoissonCPU::PoissonCPU;

    int solveOnB200()
    {
        const int n2 = 2 * nx * ny * nz;  // ChunkedArray indexes with int
        pp_handle h = nullptr;
        int rc = pp_create(nx, ny, nz, &h);
        if (rc != PP_SUCCESS) return rc;
        double X[6] = {Xbox[0], Xbox[1], Xbox[2], Xbox[3], Xbox[4], Xbox[5]};
        std::vector<double> f(n2), out(n2);
        for (int p = 0; p < n2; ++p) f[p] = P(p) / (dxyz[2] * dxyz[2]);
        if ((rc = pp_set_box(h, X)) == PP_SUCCESS && (rc = pp_assign_boundary(h, bc)) == PP_SUCCESS &&
            (rc = pp_assign_rhs_complex(h, f.data())) == PP_SUCCESS && (rc = pp_solve(h)) == PP_SUCCESS &&
            (rc = pp_get_solution(h, out.data())) == PP_SUCCESS)
            for (int p = 0; p < n2; ++p) P(p) = out[p];
        pp_destroy(h);
        return rc;
    }
};
