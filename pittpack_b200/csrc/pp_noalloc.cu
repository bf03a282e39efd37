// pp_solve_noalloc: the plain FP64 solve for callers that cannot allocate
// device memory.
//
// Who needs it: code that runs where cudaMalloc is not an option -- inside a
// host callback or a memory-pool-restricted service, a plugin that must not
// grow the device heap of the process that loads it, or a caller whose own
// allocator owns all device memory.  Those callers can still hand over their
// RHS and solution buffers; everything else the solve needs (the two spectral
// workspaces and the twiddle / eigenvalue / boundary tables) lives in one
// fixed file-scope device array instead of being allocated per handle.
//
// Limits and sharing:
//   * the array is PP_NOALLOC_SCRATCH_BYTES (32 MiB); every GPU that loads the
//     library holds it until the process exits.  Grids whose workspaces and
//     tables do not fit are rejected with PP_NOALLOC_TOO_LARGE before anything
//     is launched (16 B per point for the real families, 32 B per point when x
//     or y is periodic, plus a few tables);
//   * every call uses the same array and leaves the last call's contents in
//     it; nothing in it needs to start at zero (each call writes all it reads).
//     Calls whose work overlaps on the GPU (different streams, different host
//     threads) race on the array: serialise them on one stream;
//   * the first call on a device resolves the array's device address with
//     cudaGetSymbolAddress (that device current) and caches it; make that first
//     call before any stream capture.
#include <cmath>
#include <mutex>
#include <vector>

#include "../../include/pittpack_b200.h"
#include "pp_common.cuh"
#include "pp_kernels.h"

#define PP_NOALLOC_SCRATCH_BYTES (32u << 20)

static __device__ __align__(256) unsigned char pp_noalloc_scratch[PP_NOALLOC_SCRATCH_BYTES];

namespace {

const double NA_PI = 3.1415926535897932384;  // the reference's pi constant

std::mutex g_mu;
void* g_scratch[128];  // device address of the array, per device

// device address of the scratch array on the current device (set-up on first use)
int scratch_ptr(void** out)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 128) return PP_GPU_INIT_FAILURE;
    std::lock_guard<std::mutex> g(g_mu);
    if (!g_scratch[dev]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, pp_noalloc_scratch) != cudaSuccess || !p) return PP_CUDA_ERROR;
        g_scratch[dev] = p;
    }
    *out = g_scratch[dev];
    return PP_SUCCESS;
}

int na_kind(char lo, char hi)
{
    if (lo == 'D' && hi == 'D') return PP_KIND_DST2;
    if (lo == 'N' && hi == 'N') return PP_KIND_DCT2;
    if (lo == 'P' && hi == 'P') return PP_KIND_FFT;
    if (lo == 'N' && hi == 'D') return PP_KIND_DCT4;
    if (lo == 'D' && hi == 'N') return PP_KIND_DST4;
    return -1;
}

bool na_radix(int n, PPFftPlan& P)
{
    int m = n, k = 0;
    auto push = [&](int r) { P.radix[k++] = r; m /= r; };
    while (m % 8 == 0 && k < PP_FFT_MAXPASS) push(8);
    while (m % 4 == 0 && k < PP_FFT_MAXPASS) push(4);
    while (m % 2 == 0 && k < PP_FFT_MAXPASS) push(2);
    while (m % 3 == 0 && k < PP_FFT_MAXPASS) push(3);
    while (m % 5 == 0 && k < PP_FFT_MAXPASS) push(5);
    P.n = n;
    P.npass = k;
    return m == 1;
}

// host copies of one direction's tables (the same values the handle path uploads)
struct NaDir {
    int n = 0, kind = -1;
    PPFftPlan fft{};
    std::vector<double2> tw, cs;
    std::vector<double> eig;
};

int na_dir(NaDir& d, int n, int kind)
{
    d.n = n;
    d.kind = kind;
    const bool quarter = pp_kind_is_quarter(kind);
    if (quarter && n % 2) return PP_UNSUPPORTED;
    const int nf = quarter ? n / 2 : n;
    if (!na_radix(nf, d.fft)) return PP_UNSUPPORTED;
    const long double two_pi = 6.283185307179586476925286766559005768L;
    const long double pi_l = 3.141592653589793238462643383279502884L;
    d.tw.resize(nf);
    for (int m = 0; m < nf; ++m) {
        const long double a = -two_pi * (long double)m / (long double)nf;
        d.tw[m] = make_double2((double)cosl(a), (double)sinl(a));
    }
    d.cs.resize(n);
    if (quarter) {
        for (int m = 0; m < nf; ++m) {
            const long double a = -pi_l * (long double)m / (long double)n;
            d.cs[m] = make_double2((double)cosl(a), (double)sinl(a));
        }
        for (int p = 0; p < nf; ++p) {
            const long double a = -pi_l * (long double)(4 * p + 1) / (4.0L * n);
            d.cs[nf + p] = make_double2((double)cosl(a), (double)sinl(a));
        }
    } else {
        for (int k = 0; k < n; ++k) {
            const double theta = (NA_PI / 2. / n) * k;
            d.cs[k] = make_double2(cos(theta), sin(theta));
        }
    }
    double num = 0.0, freq = NA_PI;
    if (kind == PP_KIND_DST2) num = 1.0;
    else if (kind == PP_KIND_FFT) freq = 2. * NA_PI;
    else if (quarter) num = 0.5;
    d.eig.resize(n);
    for (int k = 0; k < n; ++k) d.eig[k] = -2.0 + 2. * cos((k + num) * freq / (n + 0.0));
    return PP_SUCCESS;
}

double na_exact(double omega, double x, int tg)
{
    if (fabs(omega) < 1.0e-6) return 1.0;
    if (tg == 0 || tg == -1 || tg == -2) return sin(omega * x);
    if (tg == 1) return cos(omega * x);
    return 0.0;
}

int na_tag_xy(int kind) { return kind == PP_KIND_DST2 ? 0 : kind == PP_KIND_DCT2 ? 1 : kind == PP_KIND_FFT ? 2 : -1; }

int na_tag_z(const char* bc)
{
    int t[3], count = 0;
    for (int d = 0; d < 3; ++d) {
        const char lo = bc[2 * d], hi = bc[2 * d + 1];
        if (lo == 'D' && hi == 'D') t[d] = 0;
        else if (lo == 'N' && hi == 'N') t[d] = 1;
        else if (lo == 'P' && hi == 'P') t[d] = 2;
        else {
            t[d] = -1;
            count++;
        }
    }
    if (count == 0) t[2] = -1;
    if (bc[4] == 'D') return -1;
    if (bc[4] == 'N') return -2;
    return t[2];
}

// a bump allocator over the scratch array (256-byte aligned pieces)
struct Carve {
    unsigned char* base;
    size_t used = 0;
    bool ok = true;
    template <typename T>
    T* take(size_t count)
    {
        const size_t off = (used + 255) & ~(size_t)255;
        const size_t bytes = count * sizeof(T);
        if (off + bytes > PP_NOALLOC_SCRATCH_BYTES) {
            ok = false;
            return nullptr;
        }
        used = off + bytes;
        return reinterpret_cast<T*>(base + off);
    }
};

cudaError_t na_line_pass(PPLinePassArgs a, const NaDir& d, const double2* tw, const double2* cs, bool inverse,
                         bool strided, bool in_cplx, bool out_cplx, cudaStream_t st)
{
    a.fft = d.fft;
    a.fft.tw = tw;
    a.cs = cs;
    const int lpc2 = pp_lp2_lpc(d.n), lpc = lpc2 ? lpc2 : pp_lpm_lpc(d.n);
    if (lpc > 0) {
        a.tw = tw;
        a.cs2 = cs;
        a.in_cplx = in_cplx;
        a.out_cplx = out_cplx;
        const int dl = d.kind == PP_KIND_FFT ? lpc : 2 * lpc;
        a.L = dl;
        a.tiles_per_plane = (a.nlines + dl - 1) / dl;
        return lpc2 ? pp_launch_line_pass_pow2<double, double, double>(a, inverse, strided, st)
                    : pp_launch_line_pass_mixed(a, inverse, strided, st);
    }
    int L = 16;
    while (L > 1 && pp_line_pass_smem(L, d.fft.n) > 64 * 1024) L >>= 1;
    a.L = L;
    a.tiles_per_plane = (a.nlines + L - 1) / L;
    return pp_launch_line_pass(a, inverse, strided, in_cplx, out_cplx, st);
}

}  // namespace

extern "C" int pp_solve_noalloc(int nx, int ny, int nz, const char bc[6], const double box[6], const double* d_rhs,
                                double* d_P, void* stream)
{
    if (nx < 2 || ny < 2 || nz < 3 || !bc || !box || !d_rhs || !d_P) return PP_INPUT_ARGS;
    for (int i = 0; i < 6; ++i)
        if (bc[i] != 'P' && bc[i] != 'N' && bc[i] != 'D') return PP_INPUT_ARGS;
    const int kx = na_kind(bc[0], bc[1]), ky = na_kind(bc[2], bc[3]);
    if (kx < 0 || ky < 0 || (bc[4] == 'P') != (bc[5] == 'P')) return PP_INPUT_ARGS;
    for (int d = 0; d < 3; ++d)
        if (!(box[2 * d + 1] > box[2 * d])) return PP_INPUT_ARGS;
    if (nz > PP_Z_MAX_NZ) return PP_UNSUPPORTED;

    NaDir tx, ty;
    int rc;
    if ((rc = na_dir(tx, nx, kx)) != PP_SUCCESS) return rc;
    if ((rc = na_dir(ty, ny, ky)) != PP_SUCCESS) return rc;

    const bool x_cplx = kx == PP_KIND_FFT;
    const bool s_cplx = ky == PP_KIND_FFT;
    const size_t n = (size_t)nx * ny * nz;

    // carve the scratch: workspaces first, then the tables; reject before any launch
    void* sp = nullptr;
    if ((rc = scratch_ptr(&sp)) != PP_SUCCESS) return rc;
    Carve cv{static_cast<unsigned char*>(sp)};
    double* A = cv.take<double>(n * ((x_cplx || s_cplx) ? 2 : 1));
    double* B = cv.take<double>(n * (s_cplx ? 2 : 1));
    double2* twx = cv.take<double2>(tx.tw.size());
    double2* csx = cv.take<double2>(tx.cs.size());
    double* eigx = cv.take<double>(nx);
    double2* twy = cv.take<double2>(ty.tw.size());
    double2* csy = cv.take<double2>(ty.cs.size());
    double* eigy = cv.take<double>(ny);

    // Dirichlet face corrections (modifyRhsDirichlet, src/pencilDcmp.cpp:4623-4835)
    const double pi = 4. * atan(1.0);
    const double Xa = box[0], Ya = box[2], Za = box[4];
    const double c1 = -(box[0] - box[1]) / nx, c2 = -(box[2] - box[3]) / ny, c3 = -(box[4] - box[5]) / nz;
    const double omega[3] = {1 * pi, 2 * pi, 3 * pi};
    const int t0 = na_tag_xy(kx), t1 = na_tag_xy(ky), t2 = na_tag_z(bc);
    std::vector<double> face[6];
    for (int f = 0; f < 2; ++f)
        if (bc[4 + f] == 'D') {
            face[f].resize((size_t)nx * ny);
            const double z = f == 0 ? Za : Za + (nz - 1) * c3 + c3;
            for (int i = 0; i < nx; ++i)
                for (int j = 0; j < ny; ++j)
                    face[f][i + (size_t)nx * j] = 2. * na_exact(omega[0], Xa + i * c1 + c1 * .5, t0) *
                                                  na_exact(omega[1], Ya + j * c2 + c2 * 0.5, t1) *
                                                  na_exact(omega[2], z, t2);
        }
    for (int f = 0; f < 2; ++f)
        if (bc[f] == 'D') {
            face[2 + f].resize((size_t)ny * nz);
            const double x = f == 0 ? Xa : Xa + nx * c1;
            for (int k = 0; k < nz; ++k)
                for (int j = 0; j < ny; ++j)
                    face[2 + f][j + (size_t)ny * k] = 2. * na_exact(omega[0], x, t0) *
                                                      na_exact(omega[1], Ya + j * c2 + c2 * 0.5, t1) *
                                                      na_exact(omega[2], Za + k * c3 + c3 * .5, t2);
        }
    for (int f = 0; f < 2; ++f)
        if (bc[2 + f] == 'D') {
            face[4 + f].resize((size_t)nx * nz);
            const double y = f == 0 ? Ya : Ya + ny * c2;
            for (int k = 0; k < nz; ++k)
                for (int i = 0; i < nx; ++i)
                    face[4 + f][i + (size_t)nx * k] = 2. * na_exact(omega[0], Xa + i * c1 + c1 * 0.5, t0) *
                                                      na_exact(omega[1], y, t1) *
                                                      na_exact(omega[2], Za + k * c3 + c3 * .5, t2);
        }
    double* fdev[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    for (int f = 0; f < 6; ++f) {
        bool nonzero = false;
        for (double v : face[f]) nonzero |= v != 0.0;
        if (nonzero) fdev[f] = cv.take<double>(face[f].size());
    }
    if (!cv.ok) return PP_NOALLOC_TOO_LARGE;

    cudaStream_t st = (cudaStream_t)stream;
#define PP_NA_UP(dst, vec)                                                                                     \
    if (cudaMemcpyAsync(dst, (vec).data(), sizeof((vec)[0]) * (vec).size(), cudaMemcpyHostToDevice, st) !=      \
        cudaSuccess)                                                                                           \
        return PP_CUDA_ERROR;
    PP_NA_UP(twx, tx.tw);
    PP_NA_UP(csx, tx.cs);
    PP_NA_UP(eigx, tx.eig);
    PP_NA_UP(twy, ty.tw);
    PP_NA_UP(csy, ty.cs);
    PP_NA_UP(eigy, ty.eig);
    for (int f = 0; f < 6; ++f)
        if (fdev[f]) {
            PP_NA_UP(fdev[f], face[f]);
        }
#undef PP_NA_UP
    PPLift lift{fdev[0], fdev[1], fdev[2], fdev[3], fdev[4], fdev[5], 0};
    lift.any = (fdev[0] || fdev[1] || fdev[2] || fdev[3] || fdev[4] || fdev[5]) ? 1 : 0;

    // the five passes of the solve (as pp_solve, default options)
    const long plane = (long)nx * ny;
    PPLinePassArgs ax{};
    ax.n = nx;
    ax.kind = kx;
    ax.nlines = ny;
    ax.nplanes = nz;
    ax.elem_stride = 1;
    ax.line_stride = nx;
    ax.plane_stride = plane;
    ax.nx = nx;
    ax.ny = ny;
    ax.nz = nz;
    ax.dz = c3;
    ax.out_scale = 1.0;
    PPLinePassArgs ay = ax;
    ay.n = ny;
    ay.kind = ky;
    ay.nlines = nx;
    ay.elem_stride = nx;
    ay.line_stride = 1;

    PPLinePassArgs a1 = ax;
    a1.src = d_rhs;
    a1.dst = A;
    a1.rhs_scale = 1;
    a1.lift = lift;
    if (na_line_pass(a1, tx, twx, csx, false, false, false, x_cplx, st) != cudaSuccess) return PP_CUFFT_FAIL_X;
    PPLinePassArgs a2 = ay;
    a2.src = A;
    a2.dst = B;
    if (na_line_pass(a2, ty, twy, csy, false, true, x_cplx, s_cplx, st) != cudaSuccess) return PP_CUFFT_FAIL_Y;
    PPZArgs z{};
    z.data = B;
    z.nx = nx;
    z.ny = ny;
    z.nz = nz;
    int zthreads = 0;
    pp_zsolve_config(nz, s_cplx, nx, &z.TS, &zthreads);
    z.tiles_x = (nx + z.TS - 1) / z.TS;
    z.ax = eigx;
    z.ay = eigy;
    const double dx = c1, dy = c2, dz = c3;
    z.Cx = (dz / dx) * (dz / dx);
    z.Cy = (dz / dy) * (dz / dy);
    z.zlo = bc[4] == 'P' ? PP_Z_PERIODIC : (bc[4] == 'N' ? PP_Z_NEUMANN : PP_Z_DIRICHLET);
    z.zhi = bc[5] == 'P' ? PP_Z_PERIODIC : (bc[5] == 'N' ? PP_Z_NEUMANN : PP_Z_DIRICHLET);
    z.pin_always = 1;  // the reference's zero-mode row replacement
    if (pp_launch_zsolve(z, s_cplx, st) != cudaSuccess) return PP_THOMAS_FAIL;
    PPLinePassArgs a3 = ay;
    a3.src = B;
    a3.dst = A;
    if (na_line_pass(a3, ty, twy, csy, true, true, s_cplx, s_cplx, st) != cudaSuccess) return PP_CUFFT_FAIL_INV_Y;
    PPLinePassArgs a4 = ax;
    a4.src = A;
    a4.dst = d_P;
    a4.out_scale = 1. / ((double)(nx * ny));
    if (na_line_pass(a4, tx, twx, csx, true, false, s_cplx, true, st) != cudaSuccess) return PP_CUFFT_FAIL_INV_X;
    return PP_SUCCESS;
}
