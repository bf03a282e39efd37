// pp_solve_noalloc: the plain FP64 solve for callers that cannot allocate
// device memory.
//
// Who needs it: code that runs where cudaMalloc is not an option -- a service
// whose device memory is all owned by its own pool allocator, a plugin that
// must not grow the device heap of the process that loads it, or an
// allocation-restricted context that still owns its input and output
// buffers.  Those callers hand over their RHS and solution buffers;
// everything else the solve needs (the two spectral workspaces and the
// twiddle / eigenvalue / boundary tables) lives in one fixed file-scope
// device array instead of being allocated per handle, and the tables are
// computed on the device by a small kernel, so the call copies nothing from
// the host and returns once its kernels are enqueued.
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
//     call before any stream capture;
//   * like every call that launches work, it must not be made from a stream
//     callback (cudaLaunchHostFunc / cudaStreamAddCallback), where CUDA
//     forbids CUDA calls.
#include <algorithm>
#include <cmath>
#include <mutex>

#include "../../include/pittpack_b200.h"
#include "pp_common.cuh"
#include "pp_kernels.h"
#include "pp_tables.cuh"

#define PP_NOALLOC_SCRATCH_BYTES (32u << 20)

static __device__ __align__(256) unsigned char pp_noalloc_scratch[PP_NOALLOC_SCRATCH_BYTES];

namespace {

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

// one direction of the solve: its length, family and FFT plan
struct NaDir {
    int n = 0, nf = 0, kind = -1;
    PPFftPlan fft{};
};

int na_dir(NaDir& d, int n, int kind)
{
    d.n = n;
    d.kind = kind;
    d.nf = pp_fft_len(n, kind);
    if (!pp_fft_plan(d.nf, &d.fft)) return PP_UNSUPPORTED;
    if (pp_lp2_lpc(n) == 0 && pp_lpm_lpc(n) == 0 && pp_line_pass_smem(1, d.nf) > 227 * 1024) return PP_UNSUPPORTED;
    return PP_SUCCESS;
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

// The tables of one call, written by one kernel into the scratch array:
// segments 0-2 / 3-5 are the FFT twiddles, family twiddles and eigenvalue
// parts of x / y, 6-11 the manufactured Dirichlet faces (slots 0-5, null
// where the face is not subtracted).  Values: the handle path's formulas
// (pp_tables.cuh); the FFT twiddles e^{-2 pi i m / nf} through sincospi.
struct NaTables {
    double2* tw[2];
    double2* cs[2];
    double* eig[2];
    double* face[6];
    int n[2], nf[2], kind[2];
    long len[12];
    PPMmsFaces mp;
};

__global__ void na_tables_kernel(NaTables t)
{
    long total = 0;
    for (int s = 0; s < 12; ++s) total += t.len[s];
    for (long g = blockIdx.x * (long)blockDim.x + threadIdx.x; g < total; g += (long)gridDim.x * blockDim.x) {
        long q = g;
        int s = 0;
        while (q >= t.len[s]) q -= t.len[s++];
        const int idx = (int)q;
        if (s < 6) {
            const int d = s / 3, part = s % 3;
            const int n = t.n[d], nf = t.nf[d], kind = t.kind[d];
            if (part == 0) {
                double sn, c;
                sincospi(-2.0 * idx / nf, &sn, &c);
                t.tw[d][idx] = make_double2(c, sn);
            } else if (part == 1) {
                if (pp_kind_is_quarter(kind)) {
                    long num, den;
                    pp_quarter_angle(n, idx, &num, &den);
                    double sn, c;
                    sincospi(-(double)num / (double)den, &sn, &c);
                    t.cs[d][idx] = make_double2(c, sn);
                } else {
                    t.cs[d][idx] = pp_family_twiddle(n, idx);
                }
            } else {
                t.eig[d][idx] = pp_eigen_part(n, kind, idx);
            }
        } else {
            const int slot = s - 6;
            int na, nb;
            pp_mms_face_dims(t.mp, slot, &na, &nb);
            const int a = idx % na, b = idx / na;
            t.face[slot][idx] = pp_mms_face_value(t.mp, slot, a, b);
        }
    }
}

// whether a manufactured face has a nonzero value: its values are
// 2 A(a) B(b) C, products of O(1) sines and cosines (no underflow), so it is
// nonzero exactly when each factor is nonzero somewhere; checked on the
// factors, without forming the face
bool na_face_nonzero(const PPMmsFaces& p, int slot)
{
    auto any = [](int n, auto f) {
        for (int i = 0; i < n; ++i)
            if (f(i) != 0.0) return true;
        return false;
    };
    const double w = pp_mms_face_plane(p, slot);
    auto X = [&](int i) { return pp_exact_value(p.omega[0], pp_mms_x(p, i), p.t0); };
    auto Y = [&](int j) { return pp_exact_value(p.omega[1], pp_mms_y(p, j), p.t1); };
    auto Z = [&](int k) { return pp_exact_value(p.omega[2], pp_mms_z(p, k), p.t2); };
    if (slot < 2) return any(p.nx, X) && any(p.ny, Y) && pp_exact_value(p.omega[2], w, p.t2) != 0.0;
    if (slot < 4) return pp_exact_value(p.omega[0], w, p.t0) != 0.0 && any(p.ny, Y) && any(p.nz, Z);
    return any(p.nx, X) && pp_exact_value(p.omega[1], w, p.t1) != 0.0 && any(p.nz, Z);
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
    if (nz > pp_zsolve_max_nz(ky == PP_KIND_FFT, false)) return PP_UNSUPPORTED;

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
    NaTables tb{};
    const NaDir* dirs[2] = {&tx, &ty};
    for (int d = 0; d < 2; ++d) {
        tb.n[d] = dirs[d]->n;
        tb.nf[d] = dirs[d]->nf;
        tb.kind[d] = dirs[d]->kind;
        tb.tw[d] = cv.take<double2>(dirs[d]->nf);
        tb.cs[d] = cv.take<double2>(pp_family_table_len(dirs[d]->n, dirs[d]->kind));
        tb.eig[d] = cv.take<double>(dirs[d]->n);
        tb.len[3 * d] = dirs[d]->nf;
        tb.len[3 * d + 1] = pp_family_table_len(dirs[d]->n, dirs[d]->kind);
        tb.len[3 * d + 2] = dirs[d]->n;
    }

    // manufactured Dirichlet faces (modifyRhsDirichlet, src/pencilDcmp.cpp:4623-4835)
    PPMmsFaces& mp = tb.mp;
    mp.nx = nx;
    mp.ny = ny;
    mp.nz = nz;
    const double pi = 4. * atan(1.0);
    mp.Xa = box[0];
    mp.Ya = box[2];
    mp.Za = box[4];
    mp.c1 = -(box[0] - box[1]) / nx;
    mp.c2 = -(box[2] - box[3]) / ny;
    mp.c3 = -(box[4] - box[5]) / nz;
    mp.omega[0] = 1 * pi;
    mp.omega[1] = 2 * pi;
    mp.omega[2] = 3 * pi;
    mp.t0 = na_tag_xy(kx);
    mp.t1 = na_tag_xy(ky);
    mp.t2 = na_tag_z(bc);
    static const int face_of_slot[6] = {4, 5, 0, 1, 2, 3};  // slot -> xmin, xmax, ymin, ymax, zmin, zmax
    for (int slot = 0; slot < 6; ++slot) {
        if (bc[face_of_slot[slot]] != 'D' || !na_face_nonzero(mp, slot)) continue;
        int na, nb;
        pp_mms_face_dims(mp, slot, &na, &nb);
        tb.face[slot] = cv.take<double>((size_t)na * nb);
        tb.len[6 + slot] = (long)na * nb;
    }
    if (!cv.ok) return PP_NOALLOC_TOO_LARGE;

    cudaStream_t st = (cudaStream_t)stream;
    long total = 0;
    for (int q = 0; q < 12; ++q) total += tb.len[q];
    const int tblocks = (int)std::min<long>((total + 255) / 256, 1184);
    na_tables_kernel<<<tblocks, 256, 0, st>>>(tb);
    if (cudaGetLastError() != cudaSuccess) return PP_CUDA_ERROR;
    PPLift lift{tb.face[0], tb.face[1], tb.face[2], tb.face[3], tb.face[4], tb.face[5], 0};
    lift.any = (lift.z0 || lift.z1 || lift.x0 || lift.x1 || lift.y0 || lift.y1) ? 1 : 0;
    const double2 *twx = tb.tw[0], *csx = tb.cs[0], *twy = tb.tw[1], *csy = tb.cs[1];
    const double *eigx = tb.eig[0], *eigy = tb.eig[1];
    const double c1 = mp.c1, c2 = mp.c2, c3 = mp.c3;

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
    // the handle path's launch shape for this grid (lanes per system chosen
    // by the number of systems; the launch derives the same lane count)
    pp_zsolve_config_p(nz, s_cplx, nx, 0, &z.TS, &zthreads, 0, ny);
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
