// FP64 residual of the refined mixed-precision solve.
//
// The refined solve inverts the true discrete problem A u = b of the
// reference's cell-centred 7-point Laplacian, scaled by dz^2 as the reference
// scales its RHS (src/pencilDcmp.cpp:4405-4414, src/pencilDcmp.cpp:5591-5647):
//   (A u)_ijk = Cx (u_{i-1} - 2u + u_{i+1}) + Cy (u_{j-1} - 2u + u_{j+1}) + (u_{k-1} - 2u + u_{k+1}),
//   Cx = (dz/dx)^2, Cy = (dz/dy)^2, ghost cells: Dirichlet u_g = -u, Neumann
//   u_g = u, periodic wrap-around (src/triDiag.cpp:1733-1751, 1961-2108);
//   b = f dz dz - lift, lift = modifyRhsDirichlet's face terms
//   (src/pencilDcmp.cpp:4623-4835).
// Each sweep computes r = b - A u in FP64, stores it as FP32 for the FP32
// correction solve, and accumulates the FP64 sum of r over every z-plane: the
// kx = ky = 0 spectral column, which is solved separately in FP64.
//
// Singular problems (no Dirichlet end in any direction): A has the constant
// vector in its null space, so the residual cannot see a constant offset of
// u.  The FP32 inverse transforms leave a tiny spurious mean in every
// correction (their kx = ky = 0 input is zero, their output's plane sums are
// zero only to FP32 rounding), and that mean would accumulate unchecked.  The
// residual pass therefore also sums u in FP64, and after each zero-mode solve
// the constant of the zero-mode column is re-anchored so that the mean of the
// updated u equals the mean of the pinned FP64 zero-mode solution of b (the
// same pin the FP64 solve applies).
#include "pp_common.cuh"
#include "pp_kernels.h"

namespace {

PP_D double lift3(const PPLift& L, int i, int j, int k, int nx, int ny, int nz)
{
    double s = 0.0;
    if (L.z0 && k == 0) s += L.z0[i + (long)nx * j];
    if (L.z1 && k == nz - 1) s += L.z1[i + (long)nx * j];
    if (L.x0 && i == 0) s += L.x0[j + (long)ny * k];
    if (L.x1 && i == nx - 1) s += L.x1[j + (long)ny * k];
    if (L.y0 && j == 0) s += L.y0[i + (long)nx * k];
    if (L.y1 && j == ny - 1) s += L.y1[i + (long)nx * k];
    return s;
}

// neighbour across a face: code 0 Dirichlet (-u), 1 Neumann (+u), 2 periodic
PP_D double ghost(int code, double uc, double uw) { return code == 2 ? uw : (code == 1 ? uc : -uc); }

// One CTA per (group of RESID_ROWS rows j, plane k): its threads walk each
// row with stride blockDim, so that the plane sums need one atomic per CTA
// (a few per plane) rather than one per half row.
constexpr int RESID_ROWS = 16;

__global__ void __launch_bounds__(256) resid_kernel(PPResidArgs a)
{
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    const int k = blockIdx.y;
    const int j0 = blockIdx.x * RESID_ROWS;
    const int rows = min(RESID_ROWS, ny - j0);
    const long plane = (long)nx * ny;
    double rs = 0.0, us = 0.0;
    for (int jj = 0; jj < rows; ++jj)
    for (int i = threadIdx.x; i < nx; i += blockDim.x) {
        const int j = j0 + jj;
        const long p = i + (long)nx * j + plane * k;
        double b = a.f[p] * a.dz * a.dz;
        if (a.lift.any) b = b - lift3(a.lift, i, j, k, nx, ny, nz);
        double r;
        if (a.u) {
            const double* u = a.u;
            const double uc = u[p];
            const double uw = i > 0 ? u[p - 1] : ghost(a.bc[0], uc, u[p + nx - 1]);
            const double ue = i < nx - 1 ? u[p + 1] : ghost(a.bc[1], uc, u[p - (nx - 1)]);
            const double us_ = j > 0 ? u[p - nx] : ghost(a.bc[2], uc, u[p + (long)nx * (ny - 1)]);
            const double un = j < ny - 1 ? u[p + nx] : ghost(a.bc[3], uc, u[p - (long)nx * (ny - 1)]);
            const double ub = k > 0 ? u[p - plane] : ghost(a.bc[4], uc, u[p + plane * (nz - 1)]);
            const double ut = k < nz - 1 ? u[p + plane] : ghost(a.bc[5], uc, u[p - plane * (nz - 1)]);
            const double au = a.Cx * (uw - 2.0 * uc + ue) + a.Cy * (us_ - 2.0 * uc + un) + (ub - 2.0 * uc + ut);
            r = b - au;
            if (a.usum) us += uc;
        } else {
            r = b;
        }
        a.r[p] = (float)r;
        rs += r;
    }
    if (a.psum) {
        // FP64 plane sum of r (and sum of u): block reduction, one atomic per CTA
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            rs += __shfl_xor_sync(0xffffffffu, rs, o);
            us += __shfl_xor_sync(0xffffffffu, us, o);
        }
        __shared__ double ws[8], wu[8];
        const int w = threadIdx.x >> 5, ln = threadIdx.x & 31;
        if (ln == 0) {
            ws[w] = rs;
            wu[w] = us;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            double t = 0.0, tu = 0.0;
            for (int q = 0; q < (int)(blockDim.x >> 5); ++q) {
                t += ws[q];
                tu += wu[q];
            }
            atomicAdd(&a.psum[k], t * a.psum_scale);
            if (a.usum) atomicAdd(a.usum, tu);
        }
    }
}

// zcol: the zero-mode column just solved (one value per z-plane); the
// epilogue adds zscale * zcol[k] to every point of plane k.  first: sweep 0,
// whose zero-mode solution fixes the target mean mstar.
__global__ void zero_mode_anchor_kernel(double* zcol, int nz, const double* usum, double* mstar, double zscale,
                                        double npts, int first)
{
    __shared__ double red[256];
    double s = 0.0;
    for (int k = threadIdx.x; k < nz; k += blockDim.x) s += zcol[k];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    const double m = red[0] / nz;  // mean of this sweep's zero-mode column
    if (first) {
        if (threadIdx.x == 0) *mstar = zscale * m;
        return;
    }
    // shift so that mean(u + update) = mstar
    const double shift = (*mstar - *usum / npts) / zscale - m;
    for (int k = threadIdx.x; k < nz; k += blockDim.x) zcol[k] += shift;
}

}  // namespace

cudaError_t pp_launch_zero_mode_anchor(double* zcol, int nz, const double* usum, double* mstar, double zscale,
                                       double npts, int first, cudaStream_t st)
{
    zero_mode_anchor_kernel<<<1, 256, 0, st>>>(zcol, nz, usum, mstar, zscale, npts, first);
    return cudaGetLastError();
}

cudaError_t pp_launch_resid(const PPResidArgs& a, cudaStream_t st)
{
    dim3 grid((a.ny + RESID_ROWS - 1) / RESID_ROWS, a.nz), block(256);
    resid_kernel<<<grid, block, 0, st>>>(a);
    return cudaGetLastError();
}
