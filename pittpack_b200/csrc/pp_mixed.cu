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
// Each sweep computes r = b - A u in FP64, rounds it to FP32 for the FP32
// correction solve, and forms the FP64 sum of r over every z-plane: the
// kx = ky = 0 spectral column, which is solved separately in FP64.  The plane
// sums come from per-(plane, tile) partial sums added in a fixed order
// (zero_mode_sums_kernel), so a refined solve gives the same bits every time.
//
// The residual is a 2.5-D stencil pass (resid_kernel): a CTA owns a 64 x 8
// tile of the xy plane and walks a chunk of z planes.  Each plane's tile of u
// with its one-point halo, and its tile of f, are copied into rings of
// shared-memory buffers by cp.async RZ_D planes ahead of use, so u is read
// from memory about once (the halo adds 2/8 + 2/64), the x, y and z
// neighbours of a point come from shared memory, f is read once and r
// written once: about 20 bytes per point of DRAM traffic in FP64 / FP32.
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
#include <stdint.h>

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

constexpr int RT_X = 64;   // tile columns (four per thread)
constexpr int RT_Y = 8;    // tile rows (16 threads per row)
constexpr int RT_KZ = 32;  // z planes per CTA
constexpr int RT_THREADS = RT_X / 4 * RT_Y;  // 128
// the halo tile: rows j0 - 1 .. j0 + 8; columns i0 - 2 .. i0 + 65 at slots
// 0 .. 67, so that the tile's own columns start on a 16-byte boundary (slot 2)
constexpr int RH_X = RT_X + 4, RH_Y = RT_Y + 2;
constexpr int RZ_D = 2;            // planes of prefetch
constexpr int RZ_NU = RZ_D + 2;    // u ring: planes k, k + 1 read, k + 2 .. k + 1 + D in flight
constexpr int RZ_NF = RZ_D + 1;    // f ring: plane k read, k + 1 .. k + D in flight

// cp.async of one double / of two (16 bytes, both addresses 16-byte aligned)
PP_D void cp8(double* smem, const double* g)
{
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(g) : "memory");
}
PP_D void cp16(double* smem, const double* g)
{
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(g) : "memory");
}

// index along one direction of a halo point: inside, wrapped (periodic), or -1
// (a Dirichlet / Neumann ghost, formed from the centre value instead)
PP_D int halo_index(int g, int n, int lo_code, int hi_code)
{
    // a tile row or column past a short grid can lie more than one period out:
    // those are never read, and give -1 too (every index returned is in [0, n))
    if (g < 0) return lo_code == 2 && g + n >= 0 ? g + n : -1;
    if (g >= n) return hi_code == 2 && g - n < n ? g - n : -1;
    return g;
}

// copy plane kk of u (tile + halo) into a ring slot; nothing for kk < 0.
// VEC: the grid's rows are whole 16-byte units (nx even, u aligned), so the
// tile's 64 columns go in 16-byte pieces where they lie inside the grid
template <bool VEC>
PP_D void load_u(const PPResidArgs& a, double (*buf)[RH_X], int kk, int i0, int j0)
{
    if (kk < 0) return;
    const long plane = (long)a.nx * a.ny;
    const double* src = a.u + kk * plane;
    if (VEC) {
        // 32 pieces per row for the tile's columns, then the two halo columns
        for (int e = threadIdx.x; e < RH_Y * (RT_X / 2); e += RT_THREADS) {
            const int r = e >> 5, c = (e & 31) * 2;
            const int gj = halo_index(j0 - 1 + r, a.ny, a.bc[2], a.bc[3]);
            if (gj < 0) continue;
            const int gi = i0 + c;
            const double* row = src + (long)gj * a.nx;
            if (gi + 1 < a.nx) cp16(&buf[r][2 + c], row + gi);
            else if (gi < a.nx) cp8(&buf[r][2 + c], row + gi);
        }
        for (int e = threadIdx.x; e < 2 * RH_Y; e += RT_THREADS) {
            const int r = e >> 1, side = e & 1;
            const int gj = halo_index(j0 - 1 + r, a.ny, a.bc[2], a.bc[3]);
            const int gi = halo_index(side ? i0 + RT_X : i0 - 1, a.nx, a.bc[0], a.bc[1]);
            // the east halo column of a tile that ends inside the grid, or at its end
            if (gj >= 0 && gi >= 0 && (side == 0 || i0 + RT_X <= a.nx))
                cp8(&buf[r][side ? 2 + RT_X : 1], src + (long)gj * a.nx + gi);
        }
        // a tile that ends inside the grid's last columns: the east halo of the
        // grid's last point is the column after it (wrapped, or a ghost)
        if (i0 + RT_X > a.nx && threadIdx.x < RH_Y) {
            const int r = threadIdx.x;
            const int gj = halo_index(j0 - 1 + r, a.ny, a.bc[2], a.bc[3]);
            const int gi = halo_index(a.nx, a.nx, a.bc[0], a.bc[1]);
            if (gj >= 0 && gi >= 0) cp8(&buf[r][2 + (a.nx - i0)], src + (long)gj * a.nx + gi);
        }
    } else {
        for (int e = threadIdx.x; e < RH_Y * (RT_X + 2); e += RT_THREADS) {
            const int r = e / (RT_X + 2), c = e - r * (RT_X + 2);
            const int gj = halo_index(j0 - 1 + r, a.ny, a.bc[2], a.bc[3]);
            int gi = i0 - 1 + c;
            if (gi > a.nx) continue;
            gi = halo_index(gi, a.nx, a.bc[0], a.bc[1]);
            if (gi >= 0 && gj >= 0) cp8(&buf[r][1 + c], src + (long)gj * a.nx + gi);
        }
    }
}

// copy plane kk of f (the tile) into a ring slot
template <bool VEC>
PP_D void load_f(const PPResidArgs& a, double (*buf)[RT_X], int kk, int i0, int j0)
{
    const double* src = a.f + kk * (long)a.nx * a.ny;
    if (VEC) {
        for (int e = threadIdx.x; e < RT_Y * (RT_X / 2); e += RT_THREADS) {
            const int r = e >> 5, c = (e & 31) * 2;
            if (j0 + r >= a.ny) continue;
            const double* row = src + (long)(j0 + r) * a.nx;
            if (i0 + c + 1 < a.nx) cp16(&buf[r][c], row + i0 + c);
            else if (i0 + c < a.nx) cp8(&buf[r][c], row + i0 + c);
        }
    } else {
        for (int e = threadIdx.x; e < RT_Y * RT_X; e += RT_THREADS) {
            const int r = e >> 6, c = e & 63;
            if (i0 + c < a.nx && j0 + r < a.ny) cp8(&buf[r][c], src + (long)(j0 + r) * a.nx + i0 + c);
        }
    }
}

// the z neighbour plane of k on the side d (-1 / +1): an index, or -1 for a ghost
PP_D int z_neighbour(const PPResidArgs& a, int k, int d)
{
    const int kk = k + d;
    if (kk < 0) return a.bc[4] == 2 ? a.nz - 1 : -1;
    if (kk >= a.nz) return a.bc[5] == 2 ? 0 : -1;
    return kk;
}

PP_D double ghost_of(int code, double uc) { return code == 1 ? uc : -uc; }

// the copies of pipeline step s (one cp.async group): u plane s + 1 + D (the
// upper z neighbour of plane s + D) and f plane s + D, where they belong to
// the chunk [k0, k1)
template <bool VEC>
PP_D void issue_step(const PPResidArgs& a, double (*ub)[RH_Y][RH_X], double (*fb)[RT_Y][RT_X], int s, int k0,
                     int k1, int i0, int j0)
{
    const int kf = s + RZ_D;
    if (kf < k1) {
        if (a.u) load_u<VEC>(a, ub[(kf + 1) % RZ_NU], z_neighbour(a, kf, +1), i0, j0);
        load_f<VEC>(a, fb[kf % RZ_NF], kf, i0, j0);
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
}

// grid: (x tiles) x (y tiles) x (z chunks), flattened; 128 threads: row
// j0 + tid / 16, columns i0 + 4 (tid % 16) .. + 3
template <bool VEC>
__global__ void __launch_bounds__(RT_THREADS) resid_kernel(PPResidArgs a, int ntx, int nty)
{
    __shared__ __align__(16) double ub[RZ_NU][RH_Y][RH_X];
    __shared__ __align__(16) double fb[RZ_NF][RT_Y][RT_X];
    __shared__ double wsum[RT_KZ][RT_Y];
    __shared__ double usum_w[RT_THREADS / 32];
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    const long plane = (long)nx * ny;
    const int bx = blockIdx.x % ntx, by = (blockIdx.x / ntx) % nty, bz = blockIdx.x / (ntx * nty);
    const int i0 = bx * RT_X, j0 = by * RT_Y, k0 = bz * RT_KZ, k1 = min(nz, k0 + RT_KZ);
    const int row = threadIdx.x >> 4, q = threadIdx.x & 15;
    const int j = j0 + row, ia = i0 + 4 * q;
    const bool jl = j < ny;
    bool live[4];
#pragma unroll
    for (int m = 0; m < 4; ++m) live[m] = jl && ia + m < nx;
    const double* u = a.u;
    const int cx = 2 + 4 * q, cy = 1 + row;  // the first point's slot in the halo tile
    const double dz = a.dz, Cx = a.Cx, Cy = a.Cy;
    const bool xlo = ia == 0 && a.bc[0] != 2;               // west ghost of point 0
    const int mlast = nx - 1 - ia;                           // the point on the east face, if in 0..3
    const bool xhi = mlast >= 0 && mlast < 4 && a.bc[1] != 2;
    const bool ylo = j == 0 && a.bc[2] != 2, yhi = j == ny - 1 && a.bc[3] != 2;
    // prologue: u planes k0 .. k0 + D, f planes k0 .. k0 + D - 1, and u at k0 - 1
    if (u) load_u<VEC>(a, ub[k0 % RZ_NU], k0, i0, j0);
    for (int s = k0 - RZ_D; s < k0; ++s) issue_step<VEC>(a, ub, fb, s, k0, k1, i0, j0);
    double ubv[4] = {0.0, 0.0, 0.0, 0.0};  // u at plane k - 1
    if (u) {
        const int kb = z_neighbour(a, k0, -1);
        if (kb >= 0)
#pragma unroll
            for (int m = 0; m < 4; ++m)
                if (live[m]) ubv[m] = u[kb * plane + (long)j * nx + ia + m];
    }
    double usum = 0.0;
    for (int k = k0; k < k1; ++k) {
        // the copies of step k - D (u planes <= k + 1, f plane k) are done
        asm volatile("cp.async.wait_group %0;\n" ::"n"(RZ_D - 1) : "memory");
        __syncthreads();
        issue_step<VEC>(a, ub, fb, k, k0, k1, i0, j0);
        const int bk = k % RZ_NU, bn = (k + 1) % RZ_NU, fk = k % RZ_NF;
        const double2 f01 = *reinterpret_cast<const double2*>(&fb[fk][row][4 * q]);
        const double2 f23 = *reinterpret_cast<const double2*>(&fb[fk][row][4 * q + 2]);
        double r[4] = {f01.x * dz * dz, f01.y * dz * dz, f23.x * dz * dz, f23.y * dz * dz};
        if (a.lift.any && jl && (ia == 0 || ia + 3 >= nx - 1 || j == 0 || j == ny - 1 || k == 0 || k == nz - 1)) {
#pragma unroll
            for (int m = 0; m < 4; ++m)
                if (live[m]) r[m] = r[m] - lift3(a.lift, ia + m, j, k, nx, ny, nz);
        }
        if (u) {
            const int kt = z_neighbour(a, k, +1), kb = z_neighbour(a, k, -1);
            double c[6], s_[4], n_[4], t_[4];
            {
                const double2 c01 = *reinterpret_cast<const double2*>(&ub[bk][cy][cx]);
                const double2 c23 = *reinterpret_cast<const double2*>(&ub[bk][cy][cx + 2]);
                c[1] = c01.x; c[2] = c01.y; c[3] = c23.x; c[4] = c23.y;
                c[0] = ub[bk][cy][cx - 1];
                c[5] = ub[bk][cy][cx + 4];
                const double2 s01 = *reinterpret_cast<const double2*>(&ub[bk][cy - 1][cx]);
                const double2 s23 = *reinterpret_cast<const double2*>(&ub[bk][cy - 1][cx + 2]);
                const double2 n01 = *reinterpret_cast<const double2*>(&ub[bk][cy + 1][cx]);
                const double2 n23 = *reinterpret_cast<const double2*>(&ub[bk][cy + 1][cx + 2]);
                const double2 t01 = *reinterpret_cast<const double2*>(&ub[bn][cy][cx]);
                const double2 t23 = *reinterpret_cast<const double2*>(&ub[bn][cy][cx + 2]);
                s_[0] = s01.x; s_[1] = s01.y; s_[2] = s23.x; s_[3] = s23.y;
                n_[0] = n01.x; n_[1] = n01.y; n_[2] = n23.x; n_[3] = n23.y;
                t_[0] = t01.x; t_[1] = t01.y; t_[2] = t23.x; t_[3] = t23.y;
            }
            if (xlo) c[0] = ghost_of(a.bc[0], c[1]);
#pragma unroll
            for (int m = 0; m < 4; ++m) {
                const double cc = c[m + 1];
                const double w = c[m];
                const double e = (xhi && m == mlast) ? ghost_of(a.bc[1], cc) : c[m + 2];
                const double sv = ylo ? ghost_of(a.bc[2], cc) : s_[m];
                const double nv = yhi ? ghost_of(a.bc[3], cc) : n_[m];
                const double bv = kb < 0 ? ghost_of(a.bc[4], cc) : ubv[m];
                const double tv = kt < 0 ? ghost_of(a.bc[5], cc) : t_[m];
                const double au = Cx * (w - 2.0 * cc + e) + Cy * (sv - 2.0 * cc + nv) + (bv - 2.0 * cc + tv);
                r[m] = r[m] - au;
                if (live[m]) usum += cc;
                ubv[m] = cc;
            }
        }
        const long p = k * plane + (long)j * nx + ia;
        if (VEC && live[3]) {
            *reinterpret_cast<float4*>(a.r + p) = make_float4((float)r[0], (float)r[1], (float)r[2], (float)r[3]);
        } else {
#pragma unroll
            for (int m = 0; m < 4; ++m)
                if (live[m]) a.r[p + m] = (float)r[m];
        }
        // the plane's sum over this row of the tile: the 16 threads' tree
        double sr = 0.0;
#pragma unroll
        for (int m = 0; m < 4; ++m) sr += live[m] ? r[m] : 0.0;
#pragma unroll
        for (int o = 8; o > 0; o >>= 1) sr += __shfl_xor_sync(0xffffffffu, sr, o);
        if (q == 0) wsum[k - k0][row] = sr;
    }
    // the chunk's sum of u: the warps' trees, then the warps in order
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) usum += __shfl_xor_sync(0xffffffffu, usum, o);
    if ((threadIdx.x & 31) == 0) usum_w[threadIdx.x >> 5] = usum;
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    __syncthreads();
    // partial sums of this tile, one per plane: [k][tile]; the u sum of the
    // chunk goes to the slot of its first plane (the total is all that is used)
    const int tpp = ntx * nty, tile = by * ntx + bx;
    for (int kk = threadIdx.x; kk < k1 - k0; kk += RT_THREADS) {
        double sr = 0.0;
        for (int rr = 0; rr < RT_Y; ++rr) sr += wsum[kk][rr];
        if (a.part) a.part[(long)(k0 + kk) * tpp + tile] = sr;
        if (a.upart) {
            double su = 0.0;
            if (kk == 0)
                for (int w = 0; w < RT_THREADS / 32; ++w) su += usum_w[w];
            a.upart[(long)(k0 + kk) * tpp + tile] = su;
        }
    }
}

// the 256 threads' values added in a fixed tree; the total in red[0]
PP_D void zm_tree(double* red)
{
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
}

// one block per plane k: zcol[k] = scale * (the plane's partials: each
// thread's stride-256 share in order, then a fixed tree); uplane[k] = the
// plane's u partials alike
__global__ void zero_mode_sums_kernel(const double* part, const double* upart, int tpp, double scale, double* zcol,
                                      double* uplane)
{
    __shared__ double red[256], redu[256];
    const int k = blockIdx.x;
    const double* p = part + (long)k * tpp;
    const double* q = upart ? upart + (long)k * tpp : nullptr;
    double s = 0.0, us = 0.0;
    for (int t = threadIdx.x; t < tpp; t += blockDim.x) {
        s += p[t];
        if (q) us += q[t];
    }
    red[threadIdx.x] = s;
    redu[threadIdx.x] = us;
    zm_tree(red);
    if (q) zm_tree(redu);
    if (threadIdx.x == 0) {
        zcol[k] = scale * red[0];
        if (q) uplane[k] = redu[0];
    }
}

// *usum = the planes' u sums added in a fixed tree
__global__ void zero_mode_usum_kernel(const double* uplane, int nz, double* usum)
{
    __shared__ double red[256];
    double us = 0.0;
    for (int k = threadIdx.x; k < nz; k += blockDim.x) us += uplane[k];
    red[threadIdx.x] = us;
    zm_tree(red);
    if (threadIdx.x == 0) *usum = red[0];
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

int pp_resid_tiles(int nx, int ny) { return ((nx + RT_X - 1) / RT_X) * ((ny + RT_Y - 1) / RT_Y); }

cudaError_t pp_launch_resid(const PPResidArgs& a, cudaStream_t st)
{
    const int ntx = (a.nx + RT_X - 1) / RT_X, nty = (a.ny + RT_Y - 1) / RT_Y, nzc = (a.nz + RT_KZ - 1) / RT_KZ;
    // 16-byte pieces need even rows and aligned arrays (r: float4 stores, 16 bytes)
    const bool vec = a.nx % 4 == 0 && reinterpret_cast<uintptr_t>(a.f) % 16 == 0 &&
                     reinterpret_cast<uintptr_t>(a.r) % 16 == 0 &&
                     (!a.u || reinterpret_cast<uintptr_t>(a.u) % 16 == 0);
    if (vec) resid_kernel<true><<<ntx * nty * nzc, RT_THREADS, 0, st>>>(a, ntx, nty);
    else resid_kernel<false><<<ntx * nty * nzc, RT_THREADS, 0, st>>>(a, ntx, nty);
    return cudaGetLastError();
}

cudaError_t pp_launch_zero_mode_sums(const double* part, const double* upart, int tpp, int nz, double scale,
                                     double* zcol, double* usum, double* uplane, cudaStream_t st)
{
    zero_mode_sums_kernel<<<nz, 256, 0, st>>>(part, upart, tpp, scale, zcol, uplane);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess || !upart) return e;
    zero_mode_usum_kernel<<<1, 256, 0, st>>>(uplane, nz, usum);
    return cudaGetLastError();
}
