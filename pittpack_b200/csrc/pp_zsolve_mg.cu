// Alternate z solve: 1-D geometric multigrid V-cycles on every (kx, ky) system.
//
// The reference keeps a 1-D multigrid solver as an alternate to its Thomas
// path (MultiGrid::solveMulti / solveMono, src/multiGrid.cpp:1105-1189,
// 1415-1515, driven by PencilDcmp::solveMG, src/pencilDcmp.cpp:4047-4135):
// red-black Gauss-Seidel smoothing (src/multiGrid.cpp:1015-1055), residual
// (:783-821), full-weighting restriction (:676-711), linear prolongation
// (:556-606) and an exact solve on the coarsest level (:1404-1408), cycled
// until the residual is below 1e-10.  There it is vertex-centred with zero
// ghost values and needs nz = 2^L - 1, and no SOLUTIONMETHOD dispatches it.
//
// Here the alternate solves the same z systems as the default partition-method
// kernel (pp_zsolve.cu), so the two paths give the same answer:
//     x_{k-1} + lambda x_k + x_{k+1} = r_k, ends lambda - 1 (Dirichlet),
//     lambda + 1 (Neumann) or cyclic (periodic),
// by cell-centred multigrid, which takes any nz:
//   * level l has n_l = nz / 2^l cells of width h = 2^l (fine units); its
//     operator, scaled by h^2, is (1, -2 + h^2 sigma, 1), sigma = lambda + 2,
//     with the same ghost rules at the ends (level 0 uses lambda itself);
//   * restriction: the residual of two child cells averaged (times h^2 of the
//     coarse level); prolongation: linear in the cell centres, ghosts by the
//     boundary rule; 2 red-black Gauss-Seidel sweeps before and after;
//   * coarsening stops at <= 16 cells or an odd count; that level is solved
//     directly (Thomas, or Sherman-Morrison for the cyclic system);
//   * V-cycles run until the residual is 1e-15 of the RHS norm, stops
//     shrinking (FP64 rounding floor), or max_cycles -- a fixed bound, so the
//     kernel always ends; systems stopped by the bound above 1e-10 are counted.
// Zero-mode systems that the default path pins (row 0 replaced, see
// pp_zsolve.cu) are solved directly, with the same pinned rows.
//
// Layout: one warp per system, G systems (adjacent kx) per CTA; the tile is
// read and written with G consecutive elements per z-plane; all levels of u
// and f live in shared memory.
#include <type_traits>

#include "pp_common.cuh"
#include "pp_kernels.h"

// bytes of one system's shared-memory block (u and f of every level, plus nz
// doubles of scratch), rounded up to 16 so that every block stays aligned
static PP_HD size_t mg_block_bytes(int tot, int nz, bool cplx)
{
    const size_t b = (size_t)2 * tot * (cplx ? 16 : 8) + (size_t)nz * 8;
    return (b + 15) & ~(size_t)15;
}

namespace {

PP_D double mz(double s, double x) { return s * x; }
PP_D double2 mz(double s, double2 x) { return make_double2(s * x.x, s * x.y); }
PP_D double az(double a, double b) { return a + b; }
PP_D double2 az(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
PP_D double sz(double a, double b) { return a - b; }
PP_D double2 sz(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
PP_D double nz2(double a) { return a * a; }
PP_D double nz2(double2 a) { return a.x * a.x + a.y * a.y; }
template <typename T>
PP_D T zz();
template <>
PP_D double zz<double>() { return 0.0; }
template <>
PP_D double2 zz<double2>() { return make_double2(0.0, 0.0); }

// coefficients of one level: interior (1, d, 1); row 0 (b0, c0); row n-1
// (an, bn); cyclic corners of 1 when periodic
struct Lev {
    int n;
    double d, b0, c0, an, bn;
    bool periodic;
};

PP_D double lev_diag(const Lev& L, int i) { return i == 0 ? L.b0 : (i == L.n - 1 ? L.bn : L.d); }

// (A u)_i of one level
template <typename T>
PP_D T lev_apply(const Lev& L, const T* u, int i)
{
    const int n = L.n;
    T s = mz(lev_diag(L, i), u[i]);
    if (i > 0) s = az(s, i == n - 1 ? mz(L.an, u[i - 1]) : u[i - 1]);
    else if (L.periodic) s = az(s, u[n - 1]);
    if (i < n - 1) s = az(s, i == 0 ? mz(L.c0, u[i + 1]) : u[i + 1]);
    else if (L.periodic) s = az(s, u[0]);
    return s;
}

// Serial direct solve (one lane) of the level's system, f -> u.  Thomas for
// the open system; the cyclic one by Sherman-Morrison: with gamma = -b0, the
// corners moved onto the diagonal (b0 - gamma, bn - 1/gamma) give a
// tridiagonal T; solve T y = f and T z = (gamma, 0, .., 0, 1), then
// x = y - z (y_0 + y_{n-1}/gamma) / (1 + z_0 + z_{n-1}/gamma).
// Scratch: c' is kept in the .x slot of u until the back substitution reads
// it, the second right-hand side in zs (n doubles); f is overwritten.
template <typename T>
PP_D void serial_solve(const Lev& L, T* f, T* u, double* zs)
{
    const int n = L.n;
    double* cp = reinterpret_cast<double*>(u);
    const int cs = sizeof(T) / sizeof(double);
    const double gam = -L.b0;
    const double b0 = L.periodic ? L.b0 - gam : L.b0;
    const double bn = L.periodic ? L.bn - 1.0 / gam : L.bn;
    if (n == 1) {
        u[0] = mz(1.0 / (L.b0 + (L.periodic ? 2.0 : 0.0)), f[0]);
        return;
    }
    // forward elimination (f becomes d', zs the second RHS's d')
    double bet = b0;
    f[0] = mz(1.0 / bet, f[0]);
    double zp = gam / bet;
    zs[0] = zp;
    double cprev = L.c0 / bet;
    cp[0] = cprev;
    for (int i = 1; i < n; ++i) {
        const double a = (i == n - 1) ? L.an : 1.0;
        const double b = (i == n - 1) ? bn : L.d;
        const double c = (i == n - 1) ? 0.0 : 1.0;
        bet = b - a * cprev;
        const double ib = 1.0 / bet;
        f[i] = mz(ib, sz(f[i], mz(a, f[i - 1])));
        const double v = (i == n - 1) ? 1.0 : 0.0;
        zp = ib * (v - a * zp);
        zs[i] = zp;
        cprev = c * ib;
        cp[(size_t)i * cs] = cprev;
    }
    // back substitution of both right-hand sides
    T y = f[n - 1];
    double z = zs[n - 1];
    u[n - 1] = y;
    for (int i = n - 2; i >= 0; --i) {
        const double c = cp[(size_t)i * cs];
        y = sz(f[i], mz(c, y));
        z = zs[i] - c * z;
        u[i] = y;
        zs[i] = z;
    }
    if (L.periodic) {
        const T fac = mz(1.0 / (1.0 + zs[0] + zs[n - 1] / gam), az(u[0], mz(1.0 / gam, u[n - 1])));
        for (int i = 0; i < n; ++i) u[i] = sz(u[i], mz(zs[i], fac));
    }
}

// one red-black Gauss-Seidel sweep of a level by a warp
template <typename T>
PP_D void rbgs(const Lev& L, const T* f, T* u, int lane)
{
    const int n = L.n;
    for (int color = 0; color < 2; ++color) {
        for (int i = 2 * lane + color; i < n; i += 64) {
            T s = f[i];
            if (i > 0) s = sz(s, i == n - 1 ? mz(L.an, u[i - 1]) : u[i - 1]);
            else if (L.periodic) s = sz(s, u[n - 1]);
            if (i < n - 1) s = sz(s, i == 0 ? mz(L.c0, u[i + 1]) : u[i + 1]);
            else if (L.periodic) s = sz(s, u[0]);
            u[i] = mz(1.0 / lev_diag(L, i), s);
        }
        __syncwarp();
    }
}

PP_D double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

template <bool CPLX>
__global__ void __launch_bounds__(128) zsolve_mg_kernel(PPZMgArgs a)
{
    using T = typename std::conditional<CPLX, double2, double>::type;
    extern __shared__ __align__(16) unsigned char mg_smem[];
    const int G = a.G;
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int tiles_x = (nx + G - 1) / G;
    const int ky = blockIdx.x / tiles_x;
    const int kx0 = (blockIdx.x - ky * tiles_x) * G;
    const int ts = min(G, nx - kx0);
    const long pstride = (long)nx * ny;
    T* base = reinterpret_cast<T*>(a.data) + (long)ky * nx + kx0;

    // per system: u levels, f levels (a.tot entries each), zs (nz doubles)
    const size_t per = mg_block_bytes(a.tot, nz, CPLX);
    unsigned char* mine = mg_smem + per * (w < G ? w : 0);
    T* U = reinterpret_cast<T*>(mine);
    T* F = U + a.tot;
    double* zs = reinterpret_cast<double*>(F + a.tot);

    // ---- load the tile: ts consecutive kx per z-plane --------------------------------
    for (int idx = threadIdx.x; idx < ts * nz; idx += blockDim.x) {
        const int g = idx % ts, k = idx / ts;
        T* Fg = reinterpret_cast<T*>(mg_smem + per * g) + a.tot;
        Fg[k] = base[(long)k * pstride + g];
    }
    __syncthreads();

    if (w < ts) {
        const int kx = kx0 + w;
        const double lam = (-2.0 + a.ax[kx] * a.Cx) + a.ay[ky] * a.Cy;
        const bool periodic = a.zlo == PP_Z_PERIODIC;
        const bool has_d = a.zlo == PP_Z_DIRICHLET || a.zhi == PP_Z_DIRICHLET;
        const bool zero = fabs(lam + 2.) < 1.e-10;
        const bool pin = zero && (periodic || a.pin_always || !has_d);
        const double sig = lam + 2.0;
        auto level = [&](int l) {
            Lev L;
            L.n = nz >> l;
            L.periodic = periodic;
            L.d = l == 0 ? lam : -2.0 + (double)(1 << (2 * l)) * sig;
            L.c0 = 1.0;
            L.an = 1.0;
            if (periodic) {
                L.b0 = L.d;
                L.bn = L.d;
            } else {
                L.b0 = a.zlo == PP_Z_NEUMANN ? L.d + 1.0 : L.d - 1.0;
                L.bn = a.zhi == PP_Z_NEUMANN ? L.d + 1.0 : L.d - 1.0;
            }
            return L;
        };
        if (pin) {
            // the default path's pinned rows: x_0 = r_0 (open), or
            // x_{n-1} + x_0 = (r_0 + r_{n-1}) / 2 (cyclic: row 0 keeps its
            // corner coefficient 1 on x_{n-1})
            if (lane == 0) {
                Lev L = level(0);
                L.b0 = 1.0;
                L.c0 = 0.0;
                if (periodic) F[0] = mz(0.5, az(F[0], F[nz - 1]));
                serial_solve(L, F, U, zs);
            }
            __syncwarp();
        } else {
            // levels: halve while even and above 16 cells
            int nl = 0;
            while (nl < 12 && ((nz >> nl) % 2) == 0 && (nz >> nl) > 16) ++nl;
            double part = 0.0;
            for (int i = lane; i < nz; i += 32) {
                part += nz2(F[i]);
                U[i] = zz<T>();
            }
            const double r0 = sqrt(warp_sum(part));
            __syncwarp();
            double prev = r0, rn = 0.0;
            int cycles = 0;
            const int maxc = nl == 0 ? 1 : a.max_cycles;
            while (r0 > 0.0 && cycles < maxc) {
                ++cycles;
                // descend: smooth, restrict the residual, zero the coarse guess
                int off = 0;
                for (int l = 0; l < nl; ++l) {
                    const Lev L = level(l);
                    T* u = U + off;
                    T* f = F + off;
                    rbgs(L, f, u, lane);
                    rbgs(L, f, u, lane);
                    T* uc = u + L.n;
                    T* fc = f + L.n;
                    for (int I = lane; I < L.n / 2; I += 32) {
                        const T ra = sz(f[2 * I], lev_apply(L, u, 2 * I));
                        const T rb = sz(f[2 * I + 1], lev_apply(L, u, 2 * I + 1));
                        fc[I] = mz(2.0, az(ra, rb));
                        uc[I] = zz<T>();
                    }
                    __syncwarp();
                    off += L.n;
                }
                // coarsest level: direct
                if (lane == 0) serial_solve(level(nl), F + off, U + off, zs);
                __syncwarp();
                // ascend: prolong the correction, smooth
                for (int l = nl - 1; l >= 0; --l) {
                    const Lev L = level(l);
                    off -= L.n;
                    T* u = U + off;
                    const T* e = U + off + L.n;
                    const int nc = L.n / 2;
                    for (int i = lane; i < L.n; i += 32) {
                        const int I = i >> 1;
                        const int J = (i & 1) ? I + 1 : I - 1;  // the other neighbour cell
                        T eJ;
                        if (J >= 0 && J < nc) eJ = e[J];
                        else if (periodic) eJ = e[(J + nc) % nc];
                        else eJ = ((J < 0 ? a.zlo : a.zhi) == PP_Z_NEUMANN) ? e[I] : mz(-1.0, e[I]);
                        u[i] = az(u[i], az(mz(0.75, e[I]), mz(0.25, eJ)));
                    }
                    __syncwarp();
                    rbgs(L, F + off, u, lane);
                    rbgs(L, F + off, u, lane);
                }
                if (nl == 0) break;
                // residual norm of level 0
                const Lev L0 = level(0);
                part = 0.0;
                for (int i = lane; i < nz; i += 32) part += nz2(sz(F[i], lev_apply(L0, U, i)));
                rn = sqrt(warp_sum(part));
                if (rn <= 1e-15 * r0 || rn > 0.5 * prev) break;
                prev = rn;
            }
            if (lane == 0 && a.stats) {
                atomicMax(&a.stats[0], cycles);
                // at the bound without reaching the tolerance (a system that
                // stops shrinking earlier is at the rounding floor of its
                // condition number)
                if (nl > 0 && cycles >= maxc && rn > 1e-10 * r0) atomicAdd(&a.stats[1], 1);
            }
        }
    }
    __syncthreads();

    // ---- store ------------------------------------------------------------------------
    for (int idx = threadIdx.x; idx < ts * nz; idx += blockDim.x) {
        const int g = idx % ts, k = idx / ts;
        const T* Ug = reinterpret_cast<const T*>(mg_smem + per * g);
        base[(long)k * pstride + g] = Ug[k];
    }
}

}  // namespace

int pp_zsolve_mg_levels_total(int nz)
{
    int tot = nz, n = nz, nl = 0;
    while (nl < 12 && (n % 2) == 0 && n > 16) {
        n /= 2;
        tot += n;
        ++nl;
    }
    return tot;
}

size_t pp_zsolve_mg_smem(int G, int nz, bool cplx)
{
    return (size_t)G * mg_block_bytes(pp_zsolve_mg_levels_total(nz), nz, cplx);
}

cudaError_t pp_launch_zsolve_mg(PPZMgArgs a, bool cplx, cudaStream_t st)
{
    if (a.nz < 3 || a.max_cycles < 1) return cudaErrorInvalidValue;
    a.tot = pp_zsolve_mg_levels_total(a.nz);
    // systems per CTA: up to 4 within ~100 KB, at least 1 within 227 KB
    int G = 4;
    while (G > 1 && pp_zsolve_mg_smem(G, a.nz, cplx) > 100 * 1024) --G;
    const size_t smem = pp_zsolve_mg_smem(G, a.nz, cplx);
    if (smem > 227 * 1024) return cudaErrorInvalidValue;
    a.G = G;
    dim3 grid(((a.nx + G - 1) / G) * a.ny), block(32 * G);
    cudaError_t e;
    if (cplx) {
        e = cudaFuncSetAttribute(zsolve_mg_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        zsolve_mg_kernel<true><<<grid, block, smem, st>>>(a);
    } else {
        e = cudaFuncSetAttribute(zsolve_mg_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        zsolve_mg_kernel<false><<<grid, block, smem, st>>>(a);
    }
    return cudaGetLastError();
}
