// Batched z-direction tridiagonal solve, one system per warp.
//
// The reference gathers each strided z-line into a buffer and runs a serial
// Thomas sweep per line (solveThmBatch, src/pencilDcmp.cpp:5066-5105 ->
// TriDiag::thomasLowMem, src/triDiag.cpp:1693-1822; periodic z through
// TriDiag::shermanMorrisonThomas, src/triDiag.cpp:1961-2108).  The system of
// mode (kx, ky) is
//     x_{k-1} + lambda x_k + x_{k+1} = r_k,   lambda = getEigenVal(ky, kx)
//     (src/pencilDcmp.cpp:4393-4417), computed here on the fly per system,
// with the ends modified by the z boundary: Dirichlet b = lambda - 1, Neumann
// b = lambda + 1 (src/triDiag.cpp:1733-1751), periodic: cyclic corners 1.
// Zero mode (|lambda + 2| < 1e-10): the reference replaces row 0 by x_0 = r_0
// (src/triDiag.cpp:1753-1776); for periodic z it solves the cyclic system
// with row 0 replaced by x_0 + x_{N-1} = (r_0 + r_{N-1}) / 2
// (shermanMorrisonThomasV1, src/triDiag.cpp:2112-2255).
//
// B200 layout and algorithm:
//   * a CTA owns TS adjacent kx columns of one ky row; it reads the TS x nz
//     tile with coalesced row segments into shared memory (rows skewed by one
//     slot every 16 to spread banks), solves, and writes the tile back;
//   * each warp solves one system at a time by the partition method: lane L
//     owns a contiguous block of M ~ nz/32 rows, eliminates it to express
//     every interior unknown through the block's first and last unknown
//     (forward sweep + backward sweep, one division per row), which leaves two
//     equations per lane.  The 2P-row reduced tridiagonal system is solved by
//     parallel cyclic reduction in shared memory; periodic systems apply
//     Sherman-Morrison on the reduced system.  Each lane then recovers its
//     interior rows from its two solved end values.
#include <type_traits>

#include "pp_common.cuh"
#include "pp_kernels.h"

namespace {

PP_D double zmul(double s, double x) { return s * x; }
PP_D double2 zmul(double s, double2 x) { return make_double2(s * x.x, s * x.y); }
PP_D double zsub(double a, double b) { return a - b; }
PP_D double2 zsub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
PP_D double zadd(double a, double b) { return a + b; }
PP_D double2 zadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
template <typename T>
PP_D T zzero();
template <>
PP_D double zzero<double>() { return 0.0; }
template <>
PP_D double2 zzero<double2>() { return make_double2(0.0, 0.0); }

// skewed position of row k inside a system's column of the tile
PP_HD int zpos(int k) { return k + (k >> 4); }
PP_HD int zpitch(int nz) { return (zpos(nz - 1) + 1) | 1; }

constexpr int RED_ROWS = 64;

template <bool CPLX, int MMAX>
__global__ void __launch_bounds__(PP_Z_THREADS) zsolve_kernel(PPZArgs a)
{
    using T = typename std::conditional<CPLX, double2, double>::type;
    extern __shared__ double zsm[];
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    const int pitch = zpitch(nz);
    T* tile = reinterpret_cast<T*>(zsm);
    const int nwarps = blockDim.x >> 5;
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    double* red = zsm + (size_t)a.TS * pitch * (CPLX ? 2 : 1);
    double* ra = red + (size_t)warp * RED_ROWS * (CPLX ? 5 : 4);
    double* rc = ra + RED_ROWS;
    double* ru = rc + RED_ROWS;
    T* rd = reinterpret_cast<T*>(ru + RED_ROWS);

    const int ky = blockIdx.x / a.tiles_x;
    const int kx0 = (blockIdx.x - ky * a.tiles_x) * a.TS;
    const int ts = min(a.TS, nx - kx0);
    T* g = reinterpret_cast<T*>(a.data);
    const long plane = (long)nx * ny;
    const long col0 = (long)ky * nx + kx0;

    for (int idx = threadIdx.x; idx < ts * nz; idx += blockDim.x) {
        const int k = idx / ts;
        const int s = idx - k * ts;
        tile[s * pitch + zpos(k)] = g[k * plane + col0 + s];
    }
    __syncthreads();

    const int P = min(32, nz / 2);
    const int bsz = nz / P;
    const int rem = nz - bsz * P;
    const bool active = lane < P;
    const int M = active ? bsz + (lane < rem ? 1 : 0) : 0;
    const int s0 = lane * bsz + min(lane, rem);
    const int m = 2 * P;
    const bool periodic = a.zlo == PP_Z_PERIODIC;
    const bool has_d = a.zlo == PP_Z_DIRICHLET || a.zhi == PP_Z_DIRICHLET;

    for (int s = warp; s < ts; s += nwarps) {
        const int kx = kx0 + s;
        const double lam = (-2.0 + a.ax[kx] * a.Cx) + a.ay[ky] * a.Cy;
        const bool zero = fabs(lam + 2.) < 1.e-10;
        const bool pin = zero && (periodic || a.pin_always || !has_d);
        T* col = tile + s * pitch;

        // coefficients of the first and last rows
        double A0, B0, C0, AN, BN, CN;
        if (periodic) {
            A0 = 1.0;
            B0 = pin ? 1.0 : lam;
            C0 = pin ? 0.0 : 1.0;
            AN = 1.0;
            BN = lam;
            CN = 1.0;
        } else {
            A0 = 0.0;
            B0 = pin ? 1.0 : (a.zlo == PP_Z_NEUMANN ? lam + 1. : lam - 1.);
            C0 = pin ? 0.0 : 1.0;
            AN = 1.0;
            BN = a.zhi == PP_Z_NEUMANN ? lam + 1.0 : lam - 1.;
            CN = 0.0;
        }

        // ---- local elimination of the lane's block ----------------------------
        // alpha (coefficient of the block's first unknown) and gamma (of the
        // next unknown) stay in registers; delta overwrites the RHS in the
        // tile column, which only this lane touches for these rows.
        double al[MMAX], ga[MMAX];
        double rA0 = 0, rB0 = 1, rC0 = 0;
        T rD0 = zzero<T>();
        double e1a = 0, e1c = 0;
        T e1d = zzero<T>();
        T dprev = zzero<T>();
#pragma unroll
        for (int i = 0; i < MMAX; ++i) {
            if (i < M) {
                const int gk = s0 + i;
                double A = 1.0, B = lam, C = 1.0;
                if (gk == 0) {
                    A = A0;
                    B = B0;
                    C = C0;
                } else if (gk == nz - 1) {
                    A = AN;
                    B = BN;
                    C = CN;
                }
                T D = col[zpos(gk)];
                if (gk == 0 && periodic && pin) D = zmul(0.5, zadd(D, col[zpos(nz - 1)]));
                if (i == 0) {
                    rA0 = A;
                    rB0 = B;
                    rC0 = C;
                    rD0 = D;
                    al[0] = 0.0;
                    ga[0] = 0.0;
                } else {
                    T dn;
                    if (i == 1) {
                        const double inv = 1.0 / B;
                        al[1] = A * inv;
                        ga[1] = C * inv;
                        dn = zmul(inv, D);
                    } else {
                        const double p = 1.0 / (B - A * ga[i - 1]);
                        al[i] = -A * al[i - 1] * p;
                        ga[i] = C * p;
                        dn = zmul(p, zsub(D, zmul(A, dprev)));
                    }
                    col[zpos(gk)] = dn;
                    dprev = dn;
                    if (i == M - 1) {
                        e1a = al[i];
                        e1c = ga[i];
                        e1d = dn;
                    }
                }
            }
        }
        // backward sweep: row 1 in terms of the block's first and last unknowns
        double br = 0, cr = 0;
        T dr = zzero<T>();
#pragma unroll
        for (int i = MMAX - 1; i >= 1; --i) {
            if (i <= M - 2) {
                const T di = col[zpos(s0 + i)];
                if (i == M - 2) {
                    br = al[i];
                    cr = ga[i];
                    dr = di;
                } else {
                    dr = zsub(di, zmul(ga[i], dr));
                    br = al[i] - ga[i] * br;
                    cr = -ga[i] * cr;
                }
            }
        }
        double e0a, e0c;
        T e0d;
        if (M == 2) {
            const double inv = 1.0 / rB0;
            e0a = rA0 * inv;
            e0c = rC0 * inv;
            e0d = zmul(inv, rD0);
        } else {
            const double q = 1.0 / (rB0 - rC0 * br);
            e0a = rA0 * q;
            e0c = -rC0 * cr * q;
            e0d = zmul(q, zsub(rD0, zmul(rC0, dr)));
        }

        // ---- reduced system: rows 2L (first) and 2L+1 (last), unit diagonal ---
        if (active) {
            ra[2 * lane] = e0a;
            rc[2 * lane] = e0c;
            rd[2 * lane] = e0d;
            ru[2 * lane] = 0.0;
            ra[2 * lane + 1] = e1a;
            rc[2 * lane + 1] = e1c;
            rd[2 * lane + 1] = e1d;
            ru[2 * lane + 1] = 0.0;
        }
        __syncwarp();
        double beta = 0.0;
        const double gam = -1.0;
        if (periodic && lane == 0) {
            // Sherman-Morrison on the reduced cyclic system: corners move into
            // u v^T with u = (gam, 0, .., alpha), v = (1, 0, .., beta / gam)
            beta = ra[0];
            const double alpha = rc[m - 1];
            ra[0] = 0.0;
            rc[m - 1] = 0.0;
            const double b0 = 1.0 - gam;
            rc[0] /= b0;
            rd[0] = zmul(1.0 / b0, rd[0]);
            ru[0] = gam / b0;
            const double bl = 1.0 - alpha * beta / gam;
            ra[m - 1] /= bl;
            rd[m - 1] = zmul(1.0 / bl, rd[m - 1]);
            ru[m - 1] = alpha / bl;
        }
        __syncwarp();
        for (int st = 1; st < m; st <<= 1) {
            double na[2], nc[2], nu[2];
            T nd[2];
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int r = 2 * lane + h;
                if (active) {
                    const double k1 = ra[r], k2 = rc[r];
                    double a1 = 0, c1 = 0, u1 = 0, a2 = 0, c2 = 0, u2 = 0;
                    T d1 = zzero<T>(), d2 = zzero<T>();
                    if (r - st >= 0) {
                        a1 = ra[r - st];
                        c1 = rc[r - st];
                        u1 = ru[r - st];
                        d1 = rd[r - st];
                    }
                    if (r + st < m) {
                        a2 = ra[r + st];
                        c2 = rc[r + st];
                        u2 = ru[r + st];
                        d2 = rd[r + st];
                    }
                    const double inv = 1.0 / (1.0 - k1 * c1 - k2 * a2);
                    na[h] = -k1 * a1 * inv;
                    nc[h] = -k2 * c2 * inv;
                    nu[h] = (ru[r] - k1 * u1 - k2 * u2) * inv;
                    nd[h] = zmul(inv, zsub(zsub(rd[r], zmul(k1, d1)), zmul(k2, d2)));
                }
            }
            __syncwarp();
            if (active) {
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int r = 2 * lane + h;
                    ra[r] = na[h];
                    rc[r] = nc[h];
                    ru[r] = nu[h];
                    rd[r] = nd[h];
                }
            }
            __syncwarp();
        }
        T xf = zzero<T>(), xl = zzero<T>();
        if (periodic) {
            // fact = (y_0 + (beta/gam) y_{m-1}) / (1 + z_0 + (beta/gam) z_{m-1})
            const double b = __shfl_sync(0xffffffffu, beta, 0);
            const double bg = b / gam;
            const T y0 = rd[0], yl = rd[m - 1];
            const double den = 1.0 + ru[0] + bg * ru[m - 1];
            const T fact = zmul(1.0 / den, zadd(y0, zmul(bg, yl)));
            if (active) {
                xf = zsub(rd[2 * lane], zmul(ru[2 * lane], fact));
                xl = zsub(rd[2 * lane + 1], zmul(ru[2 * lane + 1], fact));
            }
        } else if (active) {
            xf = rd[2 * lane];
            xl = rd[2 * lane + 1];
        }
        __syncwarp();

        // ---- recover the block's rows -----------------------------------------
        if (active) {
            T xn = xl;
            col[zpos(s0 + M - 1)] = xl;
#pragma unroll
            for (int i = MMAX - 1; i >= 1; --i) {
                if (i <= M - 2) {
                    xn = zsub(zsub(col[zpos(s0 + i)], zmul(al[i], xf)), zmul(ga[i], xn));
                    col[zpos(s0 + i)] = xn;
                }
            }
            col[zpos(s0)] = xf;
        }
        __syncwarp();
    }
    __syncthreads();

    for (int idx = threadIdx.x; idx < ts * nz; idx += blockDim.x) {
        const int k = idx / ts;
        const int s = idx - k * ts;
        g[k * plane + col0 + s] = tile[s * pitch + zpos(k)];
    }
}

template <bool CPLX>
cudaError_t launch_m(const PPZArgs& a, size_t smem, cudaStream_t st)
{
    const int P = a.nz / 2 < 32 ? a.nz / 2 : 32;
    const int mneed = (a.nz + P - 1) / P;
    dim3 grid(a.ny * a.tiles_x), block(PP_Z_THREADS);
#define PP_ZL(MM)                                                                                           \
    do {                                                                                                    \
        auto kfn = zsolve_kernel<CPLX, MM>;                                                                 \
        cudaError_t e = cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem); \
        if (e != cudaSuccess) return e;                                                                     \
        kfn<<<grid, block, smem, st>>>(a);                                                                  \
        return cudaGetLastError();                                                                          \
    } while (0)
    if (mneed <= 4) PP_ZL(4);
    if (mneed <= 8) PP_ZL(8);
    if (mneed <= 16) PP_ZL(16);
    if (mneed <= 32) PP_ZL(32);
#undef PP_ZL
    return cudaErrorInvalidValue;
}

}  // namespace

size_t pp_zsolve_smem(int TS, int nz, bool cplx)
{
    const size_t e = cplx ? 2 : 1;
    return (size_t)TS * zpitch(nz) * e * sizeof(double) +
           (size_t)(PP_Z_THREADS / 32) * RED_ROWS * (3 + e) * sizeof(double);
}

cudaError_t pp_launch_zsolve(const PPZArgs& a, bool cplx, cudaStream_t st)
{
    if (a.nz < 3 || a.nz > PP_Z_MAX_NZ) return cudaErrorInvalidValue;
    const size_t smem = pp_zsolve_smem(a.TS, a.nz, cplx);
    return cplx ? launch_m<true>(a, smem, st) : launch_m<false>(a, smem, st);
}
