// Host side of the solver: plan tables, device buffers, the launch sequence
// of one solve, and the C ABI declared in include/pittpack_b200.h.
#include <algorithm>
#include <cmath>
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include <sys/stat.h>

#include "../../include/pittpack_b200.h"
#include "pp_common.cuh"
#include "pp_kernels.h"
#include "pp_tables.cuh"

namespace {

int kind_from_bc(char lo, char hi)
{
    if (lo == 'D' && hi == 'D') return PP_KIND_DST2;
    if (lo == 'N' && hi == 'N') return PP_KIND_DCT2;
    if (lo == 'P' && hi == 'P') return PP_KIND_FFT;
    if (lo == 'N' && hi == 'D') return PP_KIND_DCT4;
    if (lo == 'D' && hi == 'N') return PP_KIND_DST4;
    return -1;
}

// factor n into the radices of the Stockham passes (pp_fft_plan: every length)
bool radix_plan(int n, std::vector<int>& r)
{
    PPFftPlan P{};
    const bool ok = pp_fft_plan(n, &P);
    r.assign(P.radix, P.radix + P.npass);
    return ok;
}

struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    cudaError_t alloc(size_t b)
    {
        free();
        cudaError_t e = cudaMalloc(&p, b);
        if (e == cudaSuccess) bytes = b;
        else p = nullptr;
        return e;
    }
    void free()
    {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    template <typename T>
    T* as() const { return static_cast<T*>(p); }
};

// one direction's transform tables
struct DirTables {
    int n = 0, kind = -1;
    PPFftPlan fft{};
    DevBuf tw;   // FFT twiddles of length fft.n
    DevBuf cs;   // family pre/post twiddles
    DevBuf eig;  // -2 + 2 cos((k + num) f / (n + den)), k < n
    DevBuf twf;  // FP32 copies for the refined mixed-precision solve
    DevBuf csf;
    // lines past one tile of the generic kernel: the four-step split of
    // fft.n (n1 = 0: not used), its plans and twiddles, the handle's scratch
    int n1 = 0, n2 = 0;
    PPFftPlan f1{}, f2{};
    DevBuf tw1, tw2, tw1f, tw2f;
    void* scratch = nullptr;
    // fft.n with a prime factor past one tile: the chirp z-transform over
    // M = n1 n2 points (M = 0: not used), W_M twiddles, chirp, kernel spectra
    int M = 0;
    DevBuf twm, twmf, chirp, chirpf, bhat[2], bhatf[2];
    void free_all()
    {
        tw.free(); cs.free(); eig.free(); twf.free(); csf.free();
        tw1.free(); tw2.free(); tw1f.free(); tw2f.free();
        twm.free(); twmf.free(); chirp.free(); chirpf.free();
        for (int b = 0; b < 2; ++b) {
            bhat[b].free();
            bhatf[b].free();
        }
    }
    size_t long_bytes() const
    {
        size_t b = tw1.bytes + tw2.bytes + tw1f.bytes + tw2f.bytes + twm.bytes + twmf.bytes + chirp.bytes + chirpf.bytes;
        for (int q = 0; q < 2; ++q) b += bhat[q].bytes + bhatf[q].bytes;
        return b;
    }
};

// upload a table in FP64 and its FP32 rounding
cudaError_t upload_pair(const std::vector<double2>& v, DevBuf& t64, DevBuf& t32)
{
    std::vector<float2> f(v.size());
    for (size_t m = 0; m < v.size(); ++m) f[m] = make_float2((float)v[m].x, (float)v[m].y);
    cudaError_t e;
    if ((e = t64.alloc(sizeof(double2) * v.size())) != cudaSuccess ||
        (e = t32.alloc(sizeof(float2) * v.size())) != cudaSuccess ||
        (e = cudaMemcpy(t64.p, v.data(), sizeof(double2) * v.size(), cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(t32.p, f.data(), sizeof(float2) * v.size(), cudaMemcpyHostToDevice)) != cudaSuccess)
        return e;
    return cudaSuccess;
}

// in-place radix-2 FFT (sign -1) of a power-of-two length in long double
void host_fft_pow2(std::vector<long double>& re, std::vector<long double>& im)
{
    const size_t n = re.size();
    for (size_t i = 1, j = 0; i < n; ++i) {
        size_t bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) {
            std::swap(re[i], re[j]);
            std::swap(im[i], im[j]);
        }
    }
    const long double pi_l = 3.141592653589793238462643383279502884L;
    for (size_t len = 2; len <= n; len <<= 1) {
        const size_t h = len / 2;
        for (size_t k = 0; k < h; ++k) {
            const long double a = -2.0L * pi_l * (long double)k / (long double)len;
            const long double wr = cosl(a), wi = sinl(a);
            for (size_t s = 0; s < n; s += len) {
                const size_t u = s + k, v = s + k + h;
                const long double xr = re[v] * wr - im[v] * wi, xi = re[v] * wi + im[v] * wr;
                re[v] = re[u] - xr;
                im[v] = im[u] - xi;
                re[u] += xr;
                im[u] += xi;
            }
        }
    }
}

// the chirp z-transform's tables for an FFT of nf points over M = n1 n2:
// c_k = e^{i pi k^2 / nf} (k^2 reduced mod 2 nf), and the spectra of the
// chirp kernel b (b_j = c_j, b_{M-j} = c_j for 0 < j < nf; conjugated for the
// backward transform) in the four-step output order (k at (k mod n1) n2 + k / n1)
cudaError_t build_chirp_tables(DirTables& t, int nf)
{
    const long double pi_l = 3.141592653589793238462643383279502884L;
    const int M = t.M, n1 = t.n1, n2 = t.n2;
    std::vector<long double> cr(nf), ci(nf);
    std::vector<double2> c(nf);
    for (int k = 0; k < nf; ++k) {
        const long q = (long)((long long)k * k % (2LL * nf));
        const long double a = pi_l * (long double)q / (long double)nf;
        cr[k] = cosl(a);
        ci[k] = sinl(a);
        c[k] = make_double2((double)cr[k], (double)ci[k]);
    }
    cudaError_t e = upload_pair(c, t.chirp, t.chirpf);
    for (int back = 0; back < 2 && e == cudaSuccess; ++back) {
        std::vector<long double> re(M, 0.0L), im(M, 0.0L);
        const long double s = back ? -1.0L : 1.0L;
        for (int j = 0; j < nf; ++j) {
            re[j] = cr[j];
            im[j] = s * ci[j];
            if (j > 0) {
                re[M - j] = cr[j];
                im[M - j] = s * ci[j];
            }
        }
        host_fft_pow2(re, im);
        std::vector<double2> b(M);
        for (int k = 0; k < M; ++k) b[(size_t)(k % n1) * n2 + k / n1] = make_double2((double)re[k], (double)im[k]);
        e = upload_pair(b, t.bhat[back], t.bhatf[back]);
    }
    return e;
}

// the smallest prime factor of an FFT length that the chirp z-transform takes
constexpr int PP_CHIRP_MIN_PRIME = 73;

int largest_prime_factor(int n)
{
    int q = 1;
    for (int p = 2; (long)p * p <= n; ++p)
        while (n % p == 0) {
            q = p;
            n /= p;
        }
    return n > 1 ? n : q;
}

// FFT twiddles W_n^m, m < n, in long double rounded to FP64 and FP32
cudaError_t upload_twiddles(int n, DevBuf& t64, DevBuf& t32)
{
    const long double two_pi = 6.283185307179586476925286766559005768L;
    std::vector<double2> tw(n);
    std::vector<float2> twf(n);
    for (int m = 0; m < n; ++m) {
        const long double a = -two_pi * (long double)m / (long double)n;
        tw[m] = make_double2((double)cosl(a), (double)sinl(a));
        twf[m] = make_float2((float)tw[m].x, (float)tw[m].y);
    }
    cudaError_t e;
    if ((e = t64.alloc(sizeof(double2) * n)) != cudaSuccess || (e = t32.alloc(sizeof(float2) * n)) != cudaSuccess ||
        (e = cudaMemcpy(t64.p, tw.data(), sizeof(double2) * n, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(t32.p, twf.data(), sizeof(float2) * n, cudaMemcpyHostToDevice)) != cudaSuccess)
        return e;
    return cudaSuccess;
}

}  // namespace

struct pp_solver_s {
    int nx = 0, ny = 0, nz = 0;
    int device = 0;
    double box[6] = {0, 1, 0, 1, 0, 1};
    char bc[6] = {0};
    bool have_bc = false, have_rhs = false, rhs_complex = false;
    bool solved = false;  // a solve has been issued (the solution buffer holds one)
    // a z-slab of a grid decomposed over several GPUs (pp_set_slab): the
    // staged entry points run, the z faces the slab does not own take no lift,
    // and the spectrum keeps the usual [k][ky][kx] layout
    bool slab = false, zface_lo = true, zface_hi = true;
    pp_options opt{};
    cudaStream_t stream = 0;
    DirTables tx, ty;
    DevBuf rhs, bufA, bufB, out;
    // caller-owned device buffers bound by pp_bind_device_buffers (zero copy):
    // the solve reads the RHS from ext_rhs and writes P to ext_out
    const double* ext_rhs = nullptr;
    double* ext_out = nullptr;
    pp_tuning tune{0, 0, 0};  // launch-shape choices (0 = built-in default)
    DevBuf psum;   // refined solve: zero-mode column, sum of u, target mean, planes' sums of u (2 nz + 2 doubles)
    DevBuf part;   // refined solve: per-CTA partial sums of r and of u (2 x nz x tiles)
    DevBuf errc;   // CTAs whose bounded waits ran out (one int)
    DevBuf zero1;  // one double 0.0 (eigen table of the zero-mode system)
    DevBuf mgstats;  // multigrid z solve: max cycles, unconverged systems (2 ints)
    DevBuf zmean;    // zero-mean option: partial sums and the mean
    DevBuf wlong;    // four-step scratch of the directions past one generic-kernel tile
    int last_sweeps = 0;
    DevBuf lift[6];
    PPLift liftv{};
    // caller's boundary data per face (xmin, xmax, ymin, ymax, zmin, zmax);
    // empty: none (pp_set_face_values)
    std::vector<double> uface[6];
    std::mutex mu;
    std::string last_error;
    // live per-stage timing (pp_timing_begin / pp_timing_end): events from a
    // pool, (stage, start event, end event) records, solves counted
    struct TRec {
        int slot, e0, e1;
    };
    std::vector<cudaEvent_t> tev;
    std::vector<TRec> trec;
    int tnext = 0, tmax = 0, tcount = 0;
    bool timing = false;
};

namespace {

int set_cuda_error(pp_solver_s* h, cudaError_t e, int code)
{
    if (h) h->last_error = cudaGetErrorString(e);
    return code;
}

// tables of one direction: FFT twiddles in long double, family twiddles as
// the reference computes them (theta = (pi/2/N) k with its pi constant)
int build_dir(pp_solver_s* h, DirTables& t, int n, int kind)
{
    t.n = n;
    t.kind = kind;
    const bool quarter = pp_kind_is_quarter(kind);
    const int nf = pp_fft_len(n, kind);
    std::vector<int> r;
    if (!radix_plan(nf, r)) return PP_UNSUPPORTED;
    // the generic kernel holds a tile of at least one line (two buffers) in
    // shared memory: longer lines, outside the register kernels, run the
    // four-step FFT through global memory (pp_longline.cu) where nf splits
    t.n1 = t.n2 = t.M = 0;
    // lines past one generic-kernel tile, and lengths whose largest prime
    // factor p makes the generic kernel's direct p-point pass (p^2 work per
    // butterfly) slower than the chirp z-transform: measured on 64 x 64
    // planes, p = 67 0.34 ms generic / 0.39 ms chirp per solve, p = 131
    // 2.28 / 0.62, p = 1031 937 / 3.6, p = 4099 29500 / 14.4
    const bool long_line = pp_line_pass_smem(1, nf) > 227 * 1024;
    const bool big_prime = largest_prime_factor(nf) >= PP_CHIRP_MIN_PRIME;
    if (pp_lp2_lpc(n) == 0 && pp_lpm_lpc(n) == 0 && (long_line || big_prime)) {
        // four-step where nf splits into two tiles, else the chirp z-transform
        int n1 = 0, n2 = 0, M = 0;
        if ((big_prime || !pp_long_split(nf, &n1, &n2)) && !pp_bluestein_split(nf, &M, &n1, &n2)) return PP_UNSUPPORTED;
        if (!pp_fft_plan(n1, &t.f1) || !pp_fft_plan(n2, &t.f2)) return PP_UNSUPPORTED;
        t.n1 = n1;
        t.n2 = n2;
        t.M = M;
        cudaError_t e;
        if ((e = upload_twiddles(n1, t.tw1, t.tw1f)) != cudaSuccess ||
            (e = upload_twiddles(n2, t.tw2, t.tw2f)) != cudaSuccess ||
            (M && (e = upload_twiddles(M, t.twm, t.twmf)) != cudaSuccess) ||
            (M && (e = build_chirp_tables(t, nf)) != cudaSuccess)) {
            t.n1 = t.n2 = t.M = 0;
            return set_cuda_error(h, e, e == cudaErrorMemoryAllocation ? PP_ALLOCATION_FAIL : PP_CUDA_ERROR);
        }
        t.f1.tw = t.tw1.as<double2>();
        t.f2.tw = t.tw2.as<double2>();
    }
    t.fft.n = nf;
    t.fft.npass = (int)r.size();
    for (size_t i = 0; i < r.size(); ++i) t.fft.radix[i] = r[i];
    const long double two_pi = 6.283185307179586476925286766559005768L;
    const long double pi_l = 3.141592653589793238462643383279502884L;
    std::vector<double2> tw(nf);
    for (int m = 0; m < nf; ++m) {
        long double a = -two_pi * (long double)m / (long double)nf;
        tw[m] = make_double2((double)cosl(a), (double)sinl(a));
    }
    std::vector<double2> cs;
    if (quarter) {
        // pre- and post-twiddles e^{-i pi num / den}
        cs.resize(pp_family_table_len(n, kind));
        for (size_t m = 0; m < cs.size(); ++m) {
            long num, den;
            pp_quarter_angle(n, (int)m, &num, &den);
            long double a = -pi_l * (long double)num / (long double)den;
            cs[m] = make_double2((double)cosl(a), (double)sinl(a));
        }
    } else {
        cs.resize(n);
        for (int k = 0; k < n; ++k) cs[k] = pp_family_twiddle(n, k);
    }
    std::vector<double> eig(n);
    for (int k = 0; k < n; ++k) eig[k] = pp_eigen_part(n, kind, k);

    cudaError_t e;
    if ((e = t.tw.alloc(sizeof(double2) * nf)) != cudaSuccess) return set_cuda_error(h, e, PP_ALLOCATION_FAIL);
    if ((e = t.cs.alloc(sizeof(double2) * cs.size())) != cudaSuccess) return set_cuda_error(h, e, PP_ALLOCATION_FAIL);
    if ((e = t.eig.alloc(sizeof(double) * n)) != cudaSuccess) return set_cuda_error(h, e, PP_ALLOCATION_FAIL);
    if ((e = cudaMemcpy(t.tw.p, tw.data(), sizeof(double2) * nf, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(t.cs.p, cs.data(), sizeof(double2) * cs.size(), cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(t.eig.p, eig.data(), sizeof(double) * n, cudaMemcpyHostToDevice)) != cudaSuccess)
        return set_cuda_error(h, e, PP_CUDA_ERROR);
    t.fft.tw = t.tw.as<double2>();
    // FP32 copies of the twiddles (rounded from the long-double / reference values)
    std::vector<float2> twf(nf), csf(cs.size());
    for (int m = 0; m < nf; ++m) twf[m] = make_float2((float)tw[m].x, (float)tw[m].y);
    for (size_t m = 0; m < cs.size(); ++m) csf[m] = make_float2((float)cs[m].x, (float)cs[m].y);
    if ((e = t.twf.alloc(sizeof(float2) * nf)) != cudaSuccess) return set_cuda_error(h, e, PP_ALLOCATION_FAIL);
    if ((e = t.csf.alloc(sizeof(float2) * csf.size())) != cudaSuccess) return set_cuda_error(h, e, PP_ALLOCATION_FAIL);
    if ((e = cudaMemcpy(t.twf.p, twf.data(), sizeof(float2) * nf, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(t.csf.p, csf.data(), sizeof(float2) * csf.size(), cudaMemcpyHostToDevice)) != cudaSuccess)
        return set_cuda_error(h, e, PP_CUDA_ERROR);
    return PP_SUCCESS;
}

// the reference's tags for exactValue (extractTag, src/pencilDcmp.cpp:3636-3668)
int ref_tag_xy(int kind)
{
    if (kind == PP_KIND_DST2) return 0;
    if (kind == PP_KIND_DCT2) return 1;
    if (kind == PP_KIND_FFT) return 2;
    return -1;
}

int ref_tag_z(const char* bc)
{
    int t[3], count = 0;
    for (int d = 0; d < 3; ++d) {
        char lo = bc[2 * d], hi = bc[2 * d + 1];
        if (lo == 'D' && hi == 'D') t[d] = 0;
        else if (lo == 'N' && hi == 'N') t[d] = 1;
        else if (lo == 'P' && hi == 'P') t[d] = 2;
        else { t[d] = -1; count++; }
    }
    if (count == 0) t[2] = -1;
    if (bc[4] == 'D') return -1;
    if (bc[4] == 'N') return -2;
    return t[2];
}

// the manufactured-solution face parameters of a handle (modifyRhsDirichlet,
// src/pencilDcmp.cpp:4623-4835): box corner, cell sizes, omega = {1, 2, 3} pi
// and the reference's tags
PPMmsFaces mms_faces(int nx, int ny, int nz, const char* bc, const double* box)
{
    PPMmsFaces p{};
    p.nx = nx;
    p.ny = ny;
    p.nz = nz;
    const double pi = 4. * atan(1.0);
    p.Xa = box[0];
    p.Ya = box[2];
    p.Za = box[4];
    p.c1 = -(box[0] - box[1]) / (nx);
    p.c2 = -(box[2] - box[3]) / (ny);
    p.c3 = -(box[4] - box[5]) / (nz);
    p.omega[0] = 1 * pi;
    p.omega[1] = 2 * pi;
    p.omega[2] = 3 * pi;
    p.t0 = ref_tag_xy(kind_from_bc(bc[0], bc[1]));
    p.t1 = ref_tag_xy(kind_from_bc(bc[2], bc[3]));
    p.t2 = ref_tag_z(bc);
    return p;
}

// face corrections subtracted from the dz^2-scaled RHS: the caller's boundary
// data where pp_set_face_values set some, else (option dirichlet_lift) the
// manufactured-solution faces of modifyRhsDirichlet
// (src/pencilDcmp.cpp:4623-4835), evaluated with the reference's expressions
// (pp_mms_face_value)
int build_lift(pp_solver_s* h)
{
    for (auto& b : h->lift) b.free();
    h->liftv = PPLift{};
    bool user = false;
    for (int f = 0; f < 6; ++f) user |= !h->uface[f].empty() && h->bc[f] != 'P';
    if (!h->opt.dirichlet_lift && !user) return PP_SUCCESS;
    const PPMmsFaces mp = mms_faces(h->nx, h->ny, h->nz, h->bc, h->box);
    const double c1 = mp.c1, c2 = mp.c2, c3 = mp.c3;
    auto upload = [&](int face, const std::vector<double>& v) -> int {
        bool nonzero = false;
        for (double x : v) nonzero |= (x != 0.0);
        if (!nonzero) return PP_SUCCESS;  // nothing to subtract
        cudaError_t e = h->lift[face].alloc(sizeof(double) * v.size());
        if (e != cudaSuccess) return set_cuda_error(h, e, PP_ALLOCATION_FAIL);
        if ((e = cudaMemcpy(h->lift[face].p, v.data(), sizeof(double) * v.size(), cudaMemcpyHostToDevice)) !=
            cudaSuccess)
            return set_cuda_error(h, e, PP_CUDA_ERROR);
        return PP_SUCCESS;
    };
    int rc;
    if (h->opt.dirichlet_lift) {
        // device slots: z faces 0, 1; x faces 2, 3; y faces 4, 5 (the caller's
        // face numbers are xmin, xmax, ymin, ymax, zmin, zmax)
        static const int face_of_slot[6] = {4, 5, 0, 1, 2, 3};
        for (int slot = 0; slot < 6; ++slot) {
            const int f = face_of_slot[slot];
            if (h->bc[f] != 'D' || !h->uface[f].empty()) continue;
            if ((slot == 0 && !h->zface_lo) || (slot == 1 && !h->zface_hi)) continue;  // inside a decomposed grid
            int na, nb;
            pp_mms_face_dims(mp, slot, &na, &nb);
            std::vector<double> v((size_t)na * nb);
            for (int b = 0; b < nb; ++b)
                for (int a = 0; a < na; ++a) v[a + (size_t)na * b] = pp_mms_face_value(mp, slot, a, b);
            if ((rc = upload(slot, v)) != PP_SUCCESS) return rc;
        }
    }
    // the caller's data through the ghost-cell relations of the 7-point operator
    // scaled by dz^2: a face's neighbour term has weight w = (dz/dx)^2,
    // (dz/dy)^2 or 1; Dirichlet u_ghost = 2 g - u_0 moves 2 w g to the right-hand
    // side, Neumann (outward derivative g) u_ghost = u_0 + h g moves w h g
    {
        const double wgt[3] = {(c3 / c1) * (c3 / c1), (c3 / c2) * (c3 / c2), 1.0};
        const double hh[3] = {c1, c2, c3};
        for (int f = 0; f < 6; ++f) {
            if (h->uface[f].empty() || h->bc[f] == 'P') continue;
            if ((f == 4 && !h->zface_lo) || (f == 5 && !h->zface_hi)) continue;  // inside a decomposed grid
            const int d = f / 2;
            const double c = h->bc[f] == 'D' ? 2.0 * wgt[d] : wgt[d] * hh[d];
            std::vector<double> v(h->uface[f].size());
            for (size_t q = 0; q < v.size(); ++q) v[q] = c * h->uface[f][q];
            const int slot = d == 2 ? f - 4 : (d == 0 ? 2 + f : 4 + (f - 2));
            if ((rc = upload(slot, v)) != PP_SUCCESS) return rc;
        }
    }
    PPLift& L = h->liftv;
    L.z0 = h->lift[0].as<double>();
    L.z1 = h->lift[1].as<double>();
    L.x0 = h->lift[2].as<double>();
    L.x1 = h->lift[3].as<double>();
    L.y0 = h->lift[4].as<double>();
    L.y1 = h->lift[5].as<double>();
    L.any = (L.z0 || L.z1 || L.x0 || L.x1 || L.y0 || L.y1) ? 1 : 0;
    return PP_SUCCESS;
}

int valid_bc(const char* bc)
{
    for (int i = 0; i < 6; ++i)
        if (bc[i] != 'P' && bc[i] != 'N' && bc[i] != 'D') return 0;
    if (kind_from_bc(bc[0], bc[1]) < 0 || kind_from_bc(bc[2], bc[3]) < 0) return 0;
    if ((bc[4] == 'P') != (bc[5] == 'P')) return 0;
    return 1;
}

int rebuild_tables(pp_solver_s* h)
{
    // complex spectra (periodic y) make the z solve's column twice as long
    if (kind_from_bc(h->bc[2], h->bc[3]) == PP_KIND_FFT && h->nz > pp_zsolve_max_nz(true, false))
        return PP_UNSUPPORTED;
    int rc = build_dir(h, h->tx, h->nx, kind_from_bc(h->bc[0], h->bc[1]));
    if (rc != PP_SUCCESS) return rc;
    rc = build_dir(h, h->ty, h->ny, kind_from_bc(h->bc[2], h->bc[3]));
    if (rc != PP_SUCCESS) return rc;
    return build_lift(h);
}

// lines per CTA tile of a transform pass: a power of two that keeps the two
// shared-memory buffers within 64 KB
int pick_lines(int nfft)
{
    int L = 16;
    while (L > 1 && pp_line_pass_smem(L, nfft) > 64 * 1024) L >>= 1;
    return L;
}

// timing stamps around one stage (no-ops unless timing is on)
int stamp(pp_solver_s* h)
{
    if (!h->timing || h->tnext >= (int)h->tev.size()) return -1;
    const int i = h->tnext++;
    cudaEventRecord(h->tev[i], h->stream);
    return i;
}
void stage_done(pp_solver_s* h, int slot, int i0)
{
    if (i0 < 0) return;
    const int i1 = stamp(h);
    if (i1 >= 0) h->trec.push_back({slot, i0, i1});
}
enum { SLOT_XF = 0, SLOT_YF = 1, SLOT_Z = 2, SLOT_YI = 3, SLOT_XI = 4, SLOT_RES = 5 };

// lines per CTA tile of the FP32 generic kernel (same 64 KB rule)
int pick_lines_fp32(int nfft)
{
    int L = 16;
    while (L > 1 && pp_line_pass_smem(L, nfft, true) > 64 * 1024) L >>= 1;
    return L;
}

// whether every contiguous run of a transform tile starts on a 16-byte
// boundary: the source pointer and the plane / line (contiguous pass) or
// element (strided pass) strides, in bytes
int runs_aligned16(const PPLinePassArgs& a, bool strided, size_t elem_bytes, int dl)
{
    if (reinterpret_cast<uintptr_t>(a.src) % 16) return 0;
    const size_t st = strided ? (size_t)a.elem_stride : (size_t)a.line_stride;
    const size_t ts = a.tile_stride ? (size_t)a.tile_stride : (size_t)a.line_stride;  // per line of l0
    return ((size_t)a.plane_stride * elem_bytes) % 16 == 0 && (st * elem_bytes) % 16 == 0 &&
           ((size_t)dl * ts * elem_bytes) % 16 == 0;
}

// one transform pass: the register-resident kernel for power-of-two lengths,
// the generic shared-memory Stockham kernel otherwise (which uses the input
// strides for its output too: it never sees the z-tiled layout)
cudaError_t line_pass(PPLinePassArgs a, const DirTables& d, bool inverse, bool strided, bool in_cplx,
                      bool out_cplx, cudaStream_t st, bool fp32 = false)
{
    if (a.o_elem_stride == 0) {
        a.o_elem_stride = a.elem_stride;
        a.o_line_stride = a.line_stride;
        a.o_plane_stride = a.plane_stride;
        a.o_tile_stride = a.tile_stride;
    }
    int lpc = pp_lp2_lpc(d.n);
    const bool mixed = lpc == 0 && pp_lpm_lpc(d.n) > 0;
    if (mixed) lpc = pp_lpm_lpc(d.n);
    if (d.n1 > 0) {
        PPLongPlan lp{};
        lp.n1 = d.n1;
        lp.n2 = d.n2;
        lp.f1 = d.f1;
        lp.f2 = d.f2;
        lp.tw1f = d.tw1f.p;
        lp.tw2f = d.tw2f.p;
        lp.twl = d.M ? d.twm.as<double2>() : d.tw.as<double2>();
        lp.twlf = d.M ? d.twmf.p : d.twf.p;
        lp.scratch = d.scratch;
        lp.M = d.M;
        lp.nf = d.fft.n;
        lp.chirp = d.chirp.as<double2>();
        lp.chirpf = d.chirpf.p;
        for (int b = 0; b < 2; ++b) {
            lp.bhat[b] = d.bhat[b].as<double2>();
            lp.bhatf[b] = d.bhatf[b].p;
        }
        a.cs2 = d.csf.p;
        return pp_launch_long_line_pass(a, lp, inverse, strided, in_cplx, out_cplx, st, fp32);
    }
    if (fp32 && lpc == 0) {
        a.fft = d.fft;
        a.tw = d.twf.p;
        a.cs2 = d.csf.p;
        a.L = pick_lines_fp32(d.fft.n);
        a.tiles_per_plane = (a.nlines + a.L - 1) / a.L;
        return pp_launch_line_pass(a, inverse, strided, in_cplx, out_cplx, st, true);
    }
    if (lpc > 0) {
        // data lines per tile: one per complex FFT line for the full complex
        // family, two (packed real lines) for the others and the half spectra
        const int dl = (d.kind == PP_KIND_FFT && !a.half) ? lpc : 2 * lpc;
        a.tw = fp32 ? d.twf.p : d.tw.p;
        a.cs2 = fp32 ? d.csf.p : d.cs.p;
        a.in_cplx = in_cplx;
        a.out_cplx = out_cplx;
        a.vec16 = runs_aligned16(a, strided, (in_cplx ? 2 : 1) * (fp32 ? sizeof(float) : sizeof(double)), dl);
        a.L = dl;
        a.tiles_per_plane = (a.nlines + dl - 1) / dl;
        if (mixed)
            return fp32 ? pp_launch_line_pass_mixed_f32(a, inverse, strided, st)
                        : pp_launch_line_pass_mixed(a, inverse, strided, st);
        return fp32 ? pp_launch_line_pass_pow2<float, float, float>(a, inverse, strided, st)
                    : pp_launch_line_pass_pow2<double, double, double>(a, inverse, strided, st);
    }
    return pp_launch_line_pass(a, inverse, strided, in_cplx, out_cplx, st);
}

// strides of the z-tiled spectrum for the y passes: line kx of plane k at
// row ky is at ky (nx nz) + (kx / TS) (nz TS) + k TS + kx % TS; a y tile of
// TS lines starting at l0 (a multiple of TS) begins at k TS + l0 nz
void set_z_tiled_out(PPLinePassArgs& a, int nx, int nz, int ts)
{
    a.o_elem_stride = (long)nx * nz;
    a.o_line_stride = 1;
    a.o_plane_stride = ts;
    a.o_tile_stride = nz;
}
void set_z_tiled_in(PPLinePassArgs& a, int nx, int nz, int ts)
{
    a.o_elem_stride = a.elem_stride;  // the output keeps the usual layout
    a.o_line_stride = a.line_stride;
    a.o_plane_stride = a.plane_stride;
    a.o_tile_stride = 0;
    a.elem_stride = (long)nx * nz;
    a.line_stride = 1;
    a.plane_stride = ts;
    a.tile_stride = nz;
}

// the periodic x pass on half spectra: ncol complex columns per row of the
// spectrum; the forward pass writes there, the inverse pass reads there and
// writes the usual nx-wide layout
void set_half_out(PPLinePassArgs& a, int ncol, long splane)
{
    a.half = 1;
    a.o_elem_stride = 1;
    a.o_line_stride = ncol;
    a.o_plane_stride = splane;
    a.o_tile_stride = 0;
}
void set_half_in(PPLinePassArgs& a, int ncol, long splane, int nx, long plane)
{
    a.half = 1;
    a.elem_stride = 1;
    a.line_stride = ncol;
    a.plane_stride = splane;
    a.tile_stride = 0;
    a.o_elem_stride = 1;
    a.o_line_stride = nx;
    a.o_plane_stride = plane;
    a.o_tile_stride = 0;
}

// Width of the z-tiled spectrum layout for this solve, 0 for the usual one.
// The forward y pass writes, and the inverse y pass reads, the spectrum as
// contiguous z tiles (TS adjacent kx x all nz of one ky), so that the z solve
// moves whole contiguous blocks; TS is the y pass's lines per tile.  Used
// when the y pass is the register-resident kernel (power-of-two lengths,
// 3 2^k and 5 2^k) with full tiles (nx a multiple of TS), the z solve is the
// direct one and takes TS systems per CTA.
int reg_lines(int n)
{
    const int lpc = pp_lp2_lpc(n);
    return lpc ? lpc : pp_lpm_lpc(n);
}
int z_tile_width(const pp_solver_s* h, bool s_cplx, int ncol)
{
    if (h->opt.z_solver != PP_ZSOLVE_DIRECT || h->slab) return 0;
    const int lpc = reg_lines(h->ny);
    if (lpc == 0) return 0;
    const int dl = s_cplx ? lpc : 2 * lpc;
    if (dl < 2 || dl > 16 || ncol % dl != 0) return 0;
    if (h->tune.zsolve_tile != 0 && h->tune.zsolve_tile != dl) return 0;
    int ts = 0, threads = 0;
    pp_zsolve_config_p(h->nz, s_cplx, ncol, h->tune.zsolve_lanes, &ts, &threads, dl, h->ny);
    return ts == dl ? dl : 0;
}

// Periodic x with a real RHS: the x spectrum of every line is Hermitian, so
// only k = 0..nx/2 is kept (the rest is its conjugate mirror, and the
// eigenvalue is symmetric in kx): the y passes and the z solve then handle
// ~half the columns.  Columns of the spectrum: nx/2 + 1, rounded up to the
// y pass's lines per tile (<= 16) so that the z-tiled layout still applies;
// 0 when the path does not apply (the full complex spectrum is used).
int half_spectrum_cols(const pp_solver_s* h)
{
    if (h->tx.kind != PP_KIND_FFT || h->rhs_complex || h->nx < 32 || reg_lines(h->nx) == 0) return 0;
    const int lpy = reg_lines(h->ny);
    int q = lpy ? (h->ty.kind == PP_KIND_FFT ? lpy : 2 * lpy) : 1;
    if (q > 16) q = 16;
    const int c = ((h->nx / 2 + 1 + q - 1) / q) * q;
    return c <= h->nx ? c : 0;
}

// lines per tile of the generic transform kernel: the tuned value when it fits
int tuned_lines(const pp_solver_s* h, int nfft)
{
    const int L = h->tune.line_tile;
    if (L >= 1 && L <= 32 && pp_line_pass_smem(L, nfft) <= 160 * 1024) return L;
    return pick_lines(nfft);
}

// the zero-mean option (the reference's ZERO_MEAN): after the solve, the mean
// of the solution's real part is subtracted from it
int zero_mean(pp_solver_s* h)
{
    if (!h->opt.zero_mean) return PP_SUCCESS;
    double* P = h->ext_out ? h->ext_out : h->out.as<double>();
    const cudaError_t e = pp_launch_zero_mean(P, (long)h->nx * h->ny * h->nz, h->zmean.as<double>(), h->stream);
    return e == cudaSuccess ? PP_SUCCESS : set_cuda_error(h, e, PP_CUDA_ERROR);
}

// the four-step scratch of the long directions, sized for the larger pass
// (x: ny x nz lines, y: spectrum columns x nz lines, of fft.n points)
int ensure_long_scratch(pp_solver_s* h)
{
    if (h->tx.n1 == 0 && h->ty.n1 == 0) return PP_SUCCESS;
    const int hc = half_spectrum_cols(h);
    const long ncol = hc ? hc : h->nx;
    size_t need = 0;
    // lines of fft.n points, or of the chirp z-transform's M
    if (h->tx.n1) need = std::max(need, pp_long_scratch_bytes((long)h->ny * h->nz, h->tx.n1 * h->tx.n2));
    if (h->ty.n1) need = std::max(need, pp_long_scratch_bytes(ncol * h->nz, h->ty.n1 * h->ty.n2));
    if (h->wlong.bytes < need) {
        const cudaError_t e = h->wlong.alloc(need);
        if (e != cudaSuccess) return set_cuda_error(h, e, PP_ALLOCATION_FAIL);
    }
    h->tx.scratch = h->wlong.p;
    h->ty.scratch = h->wlong.p;
    return PP_SUCCESS;
}

// the z solve of a staged (slab) solve: gathered columns [nz][rows][ncol] of
// spectrum rows j0 .. j0 + rows - 1
struct StageZ {
    double* data;
    int nz, rows, j0;
};
enum { STAGE_FWD = 1, STAGE_Z = 2, STAGE_INV = 4, STAGE_ALL = 7 };

int launch_solve(pp_solver_s* h, int stages = STAGE_ALL, const StageZ* sz = nullptr)
{
    if (const int rc = ensure_long_scratch(h)) return rc;
    const int nx = h->nx, ny = h->ny, nz = h->nz;
    const int kx = h->tx.kind, ky = h->ty.kind;
    const bool x_cplx = kx == PP_KIND_FFT;  // after the x transform
    const bool s_cplx = ky == PP_KIND_FFT;  // spectrum (after the y transform)
    const double dz = -(h->box[4] - h->box[5]) / (nz);
    const long plane = (long)nx * ny;
    // spectrum columns: nx, or the half spectra of the periodic x pass
    const int hc = half_spectrum_cols(h);
    const int ncol = hc ? hc : nx;
    const long splane = (long)ncol * ny;
    cudaError_t e;
    int t0;

    PPLinePassArgs ax{};
    ax.n = nx;
    ax.kind = kx;
    ax.nlines = ny;
    ax.nplanes = nz;
    ax.elem_stride = 1;
    ax.line_stride = nx;
    ax.plane_stride = plane;
    ax.fft = h->tx.fft;
    ax.cs = h->tx.cs.as<double2>();
    ax.L = tuned_lines(h, ax.fft.n);
    ax.tiles_per_plane = (ny + ax.L - 1) / ax.L;
    ax.nx = nx;
    ax.ny = ny;
    ax.nz = nz;
    ax.dz = dz;
    ax.out_scale = 1.0;
    ax.err = h->errc.as<int>();

    PPLinePassArgs ay = ax;
    ay.n = ny;
    ay.kind = ky;
    ay.nlines = ncol;
    ay.elem_stride = ncol;
    ay.line_stride = 1;
    ay.plane_stride = splane;
    ay.fft = h->ty.fft;
    ay.cs = h->ty.cs.as<double2>();
    ay.L = tuned_lines(h, ay.fft.n);
    ay.tiles_per_plane = (ncol + ay.L - 1) / ay.L;

    const int zt = z_tile_width(h, s_cplx, ncol);
    if (stages & STAGE_FWD) {
    // forward x: rhs -> A
    PPLinePassArgs a1 = ax;
    a1.src = h->ext_rhs ? h->ext_rhs : h->rhs.as<double>();
    a1.dst = h->bufA.as<double>();
    a1.rhs_scale = 1;
    a1.lift = h->liftv;
    if (hc) set_half_out(a1, ncol, splane);
    t0 = stamp(h);
    if ((e = line_pass(a1, h->tx, false, false, h->rhs_complex, x_cplx, h->stream)) != cudaSuccess)
        return set_cuda_error(h, e, PP_CUFFT_FAIL_X);
    stage_done(h, SLOT_XF, t0);
    // forward y: A -> B
    PPLinePassArgs a2 = ay;
    a2.src = h->bufA.as<double>();
    a2.dst = h->bufB.as<double>();
    if (zt) set_z_tiled_out(a2, ncol, nz, zt);
    t0 = stamp(h);
    if ((e = line_pass(a2, h->ty, false, true, x_cplx, s_cplx, h->stream)) != cudaSuccess)
        return set_cuda_error(h, e, PP_CUFFT_FAIL_Y);
    stage_done(h, SLOT_YF, t0);
    }
    if (stages & STAGE_Z) {
    // z solve in B, or (staged) in the gathered columns of several slabs
    const int zny = sz ? sz->rows : ny, znz = sz ? sz->nz : nz;
    PPZArgs z{};
    z.data = sz ? sz->data : h->bufB.as<double>();
    z.nx = ncol;
    z.ny = zny;
    z.nz = znz;
    int zthreads = 0;
    pp_zsolve_config_p(znz, s_cplx, ncol, h->tune.zsolve_lanes, &z.TS, &zthreads, zt ? zt : h->tune.zsolve_tile, zny);
    z.P = h->tune.zsolve_lanes;
    z.tiled = zt ? 1 : 0;
    z.err = h->errc.as<int>();
    z.tiles_x = (ncol + z.TS - 1) / z.TS;
    z.ax = h->tx.eig.as<double>();
    z.ay = h->ty.eig.as<double>() + (sz ? sz->j0 : 0);
    const double dx = -(h->box[0] - h->box[1]) / (nx);
    const double dy = -(h->box[2] - h->box[3]) / (ny);
    z.Cx = (dz / dx) * (dz / dx);
    z.Cy = (dz / dy) * (dz / dy);
    z.zlo = h->bc[4] == 'P' ? PP_Z_PERIODIC : (h->bc[4] == 'N' ? PP_Z_NEUMANN : PP_Z_DIRICHLET);
    z.zhi = h->bc[5] == 'P' ? PP_Z_PERIODIC : (h->bc[5] == 'N' ? PP_Z_NEUMANN : PP_Z_DIRICHLET);
    z.pin_always = h->opt.compat_zero_mode ? 1 : 0;
    t0 = stamp(h);
    if (h->opt.z_solver == PP_ZSOLVE_MULTIGRID) {
        if (!h->mgstats.p && (e = h->mgstats.alloc(2 * sizeof(int))) != cudaSuccess)
            return set_cuda_error(h, e, PP_ALLOCATION_FAIL);
        if ((e = cudaMemsetAsync(h->mgstats.p, 0, 2 * sizeof(int), h->stream)) != cudaSuccess)
            return set_cuda_error(h, e, PP_CUDA_ERROR);
        PPZMgArgs m{};
        m.data = z.data;
        m.nx = ncol;
        m.ny = zny;
        m.nz = znz;
        m.ax = z.ax;
        m.ay = z.ay;
        m.Cx = z.Cx;
        m.Cy = z.Cy;
        m.zlo = z.zlo;
        m.zhi = z.zhi;
        m.pin_always = z.pin_always;
        m.max_cycles = 60;
        m.stats = h->mgstats.as<int>();
        e = pp_launch_zsolve_mg(m, s_cplx, h->stream);
        if (e == cudaErrorInvalidValue) return PP_UNSUPPORTED;  // levels exceed shared memory
        if (e != cudaSuccess) return set_cuda_error(h, e, PP_THOMAS_FAIL);
    } else if (h->opt.z_solver == PP_ZSOLVE_REF_PCR || h->opt.z_solver == PP_ZSOLVE_REF_CRP) {
        PPZRefArgs r{};
        r.data = z.data;
        r.nx = ncol;
        r.ny = zny;
        r.nz = znz;
        r.parts = s_cplx ? 2 : 1;
        r.ax = z.ax;
        r.ay = z.ay;
        r.Cx = z.Cx;
        r.Cy = z.Cy;
        r.zlo = z.zlo;
        r.zhi = z.zhi;
        r.method = h->opt.z_solver;
        if (!pp_zsolve_ref_defined(r.method, znz, r.zlo, r.zhi)) return PP_UNSUPPORTED;
        if ((e = pp_launch_zsolve_ref(r, h->stream)) != cudaSuccess) return set_cuda_error(h, e, PP_THOMAS_FAIL);
    } else if ((e = pp_launch_zsolve(z, s_cplx, h->stream)) != cudaSuccess) {
        return set_cuda_error(h, e, PP_THOMAS_FAIL);
    }
    stage_done(h, SLOT_Z, t0);
    }
    if (!(stages & STAGE_INV)) return PP_SUCCESS;
    // inverse y: B -> A
    PPLinePassArgs a3 = ay;
    a3.src = h->bufB.as<double>();
    a3.dst = h->bufA.as<double>();
    if (zt) set_z_tiled_in(a3, ncol, nz, zt);
    t0 = stamp(h);
    if ((e = line_pass(a3, h->ty, true, true, s_cplx, s_cplx, h->stream)) != cudaSuccess)
        return set_cuda_error(h, e, PP_CUFFT_FAIL_INV_Y);
    stage_done(h, SLOT_YI, t0);
    // inverse x + rescale: A -> out (always complex-interleaved)
    PPLinePassArgs a4 = ax;
    a4.src = h->bufA.as<double>();
    a4.dst = h->ext_out ? h->ext_out : h->out.as<double>();
    a4.out_scale = 1. / ((double)(nx * ny));
    if (hc) set_half_in(a4, ncol, splane, nx, plane);
    t0 = stamp(h);
    if ((e = line_pass(a4, h->tx, true, false, s_cplx, true, h->stream)) != cudaSuccess)
        return set_cuda_error(h, e, PP_CUFFT_FAIL_INV_X);
    stage_done(h, SLOT_XI, t0);
    return zero_mean(h);
}

bool has_zero_mode(int kx, int ky)
{
    return (kx == PP_KIND_DCT2 || kx == PP_KIND_FFT) && (ky == PP_KIND_DCT2 || ky == PP_KIND_FFT);
}

// Refined mixed-precision solve of the true discrete system A u = b:
//   sweep 0:  r = b (FP64 -> FP32);            u = M32(r)
//   sweep s:  r = b - A u (FP64 -> FP32);      u += M32(r)
// M32 = FP32 transforms + FP64-arithmetic z solve on the FP32 spectrum with
// the kx = ky = 0 column left out; that column (the only singular or nearly
// singular one) is solved in FP64 from FP64 plane sums of r and added to u in
// FP64.  The last sweep writes P.  The residual kernel (a z-marching 2.5-D
// stencil) writes r (FP32) into the solution buffer; its per-(plane, tile)
// FP64 partial sums of r are added in a fixed order for the zero-mode column
// (the solve is bitwise reproducible).  Buffers: r (FP32) in the solution
// buffer, FP32 spectra in the first halves of A and B, u (FP64) in the second
// half of B.
int launch_mixed(pp_solver_s* h)
{
    if (const int rc = ensure_long_scratch(h)) return rc;
    const int nx = h->nx, ny = h->ny, nz = h->nz;
    const int kx = h->tx.kind, ky = h->ty.kind;
    const bool x_cplx = kx == PP_KIND_FFT;
    const bool s_cplx = ky == PP_KIND_FFT;
    const bool zm = has_zero_mode(kx, ky);
    const double dz = -(h->box[4] - h->box[5]) / (nz);
    const double dx = -(h->box[0] - h->box[1]) / (nx);
    const double dy = -(h->box[2] - h->box[3]) / (ny);
    const long plane = (long)nx * ny;
    // spectrum columns: nx, or the half spectra of the periodic x pass
    const int hc = half_spectrum_cols(h);
    const int ncol = hc ? hc : nx;
    const long splane = (long)ncol * ny;
    cudaError_t e;
    int t0;
    if (h->rhs_complex || h->opt.z_solver != PP_ZSOLVE_DIRECT) return PP_UNSUPPORTED;
    if (nz > pp_zsolve_max_nz(s_cplx, true)) return PP_UNSUPPORTED;  // FP32 spectra staged beside the tile
    // singular: no Dirichlet end anywhere (the x/y families with a zero mode
    // are N-N or P-P)
    const bool singular = zm && h->bc[4] != 'D' && h->bc[5] != 'D';
    const double* f = h->ext_rhs ? h->ext_rhs : h->rhs.as<double>();
    double* u = reinterpret_cast<double*>(h->bufB.as<char>() + h->bufB.bytes / 2);
    const int tpp = pp_resid_tiles(nx, ny);
    if (zm && !h->psum.p) {
        // zero-mode column (nz) + sum of u + target mean + the planes' sums of u (nz)
        if ((e = h->psum.alloc(sizeof(double) * (2 * nz + 2))) != cudaSuccess)
            return set_cuda_error(h, e, PP_ALLOCATION_FAIL);
        if ((e = h->zero1.alloc(sizeof(double))) != cudaSuccess) return set_cuda_error(h, e, PP_ALLOCATION_FAIL);
        if ((e = cudaMemset(h->zero1.p, 0, sizeof(double))) != cudaSuccess) return set_cuda_error(h, e, PP_CUDA_ERROR);
    }
    const size_t part_bytes = 2 * sizeof(double) * (size_t)nz * tpp;
    if (zm && h->part.bytes < part_bytes && (e = h->part.alloc(part_bytes)) != cudaSuccess)
        return set_cuda_error(h, e, PP_ALLOCATION_FAIL);
    double* part = zm ? h->part.as<double>() : nullptr;
    double* upart = zm ? part + (size_t)nz * tpp : nullptr;
    const double psum_scale = (kx == PP_KIND_DCT2 ? 2.0 : 1.0) * (ky == PP_KIND_DCT2 ? 2.0 : 1.0);
    float* r32 = h->out.as<float>();
    float* A32 = h->bufA.as<float>();
    float* B32 = h->bufB.as<float>();
    int bcode[6];
    for (int q = 0; q < 6; ++q) bcode[q] = h->bc[q] == 'P' ? 2 : (h->bc[q] == 'N' ? 1 : 0);

    PPResidArgs ra{};
    ra.f = f;
    ra.r = r32;
    ra.part = part;
    ra.nx = nx;
    ra.ny = ny;
    ra.nz = nz;
    ra.dz = dz;
    ra.Cx = (dz / dx) * (dz / dx);
    ra.Cy = (dz / dy) * (dz / dy);
    for (int q = 0; q < 6; ++q) ra.bc[q] = bcode[q];
    ra.lift = h->liftv;

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
    ax.dz = dz;
    ax.out_scale = 1.0;
    ax.err = h->errc.as<int>();
    PPLinePassArgs ay = ax;
    ay.n = ny;
    ay.kind = ky;
    ay.nlines = ncol;
    ay.elem_stride = ncol;
    ay.line_stride = 1;
    ay.plane_stride = splane;

    const int zt = z_tile_width(h, s_cplx, ncol);
    PPZArgs z{};
    z.data = reinterpret_cast<double*>(B32);
    z.data_fp32 = 1;
    z.skip_zero = zm ? 1 : 0;
    z.nx = ncol;
    z.ny = ny;
    z.nz = nz;
    int zthreads = 0;
    pp_zsolve_config_p(nz, s_cplx, ncol, h->tune.zsolve_lanes, &z.TS, &zthreads, zt ? zt : h->tune.zsolve_tile, ny);
    z.P = h->tune.zsolve_lanes;
    z.tiled = zt ? 1 : 0;
    z.err = h->errc.as<int>();
    z.tiles_x = (ncol + z.TS - 1) / z.TS;
    z.ax = h->tx.eig.as<double>();
    z.ay = h->ty.eig.as<double>();
    z.Cx = ra.Cx;
    z.Cy = ra.Cy;
    z.zlo = h->bc[4] == 'P' ? PP_Z_PERIODIC : (h->bc[4] == 'N' ? PP_Z_NEUMANN : PP_Z_DIRICHLET);
    z.zhi = h->bc[5] == 'P' ? PP_Z_PERIODIC : (h->bc[5] == 'N' ? PP_Z_NEUMANN : PP_Z_DIRICHLET);
    z.pin_always = 0;  // the true operator; pinned only where singular

    // the kx = ky = 0 column as a 1 x 1 x nz system in FP64 (lambda = -2)
    PPZArgs z0 = z;
    z0.data = h->psum.as<double>();
    z0.data_fp32 = 0;
    z0.skip_zero = 0;
    z0.nx = 1;
    z0.P = 0;
    z0.tiled = 0;
    z0.ny = 1;
    pp_zsolve_config(nz, false, 1, &z0.TS, &zthreads);
    z0.tiles_x = 1;
    z0.ax = h->zero1.as<double>();
    z0.ay = h->zero1.as<double>();

    const int sweeps = h->opt.max_sweeps < 0 ? 0 : h->opt.max_sweeps;
    for (int sw = 0; sw <= sweeps; ++sw) {
        const bool last = sw == sweeps;
        const bool want_usum = singular && sw > 0;
        t0 = stamp(h);
        ra.u = sw == 0 ? nullptr : u;
        ra.upart = want_usum ? upart : nullptr;
        if ((e = pp_launch_resid(ra, h->stream)) != cudaSuccess) return set_cuda_error(h, e, PP_CUDA_ERROR);
        stage_done(h, SLOT_RES, t0);
        PPLinePassArgs a1 = ax;
        a1.src = reinterpret_cast<const double*>(r32);
        a1.dst = reinterpret_cast<double*>(A32);
        if (hc) set_half_out(a1, ncol, splane);
        t0 = stamp(h);
        if ((e = line_pass(a1, h->tx, false, false, false, x_cplx, h->stream, true)) != cudaSuccess)
            return set_cuda_error(h, e, PP_CUFFT_FAIL_X);
        stage_done(h, SLOT_XF, t0);
        if (zm) {
            // the kx = ky = 0 column in FP64: plane sums, its z solve, the anchor
            t0 = stamp(h);
            double* ps = h->psum.as<double>();
            if ((e = pp_launch_zero_mode_sums(part, want_usum ? upart : nullptr, tpp, nz, psum_scale, ps, ps + nz,
                                              ps + nz + 2, h->stream)) != cudaSuccess)
                return set_cuda_error(h, e, PP_CUDA_ERROR);
            if ((e = pp_launch_zsolve(z0, false, h->stream)) != cudaSuccess) return set_cuda_error(h, e, PP_THOMAS_FAIL);
            if (singular &&
                (e = pp_launch_zero_mode_anchor(ps, nz, ps + nz, ps + nz + 1, 1.0 / (psum_scale * (double)nx * ny),
                                                (double)nx * ny * nz, sw == 0, h->stream)) != cudaSuccess)
                return set_cuda_error(h, e, PP_CUDA_ERROR);
            stage_done(h, SLOT_RES, t0);
        }
        PPLinePassArgs a2 = ay;
        a2.src = reinterpret_cast<const double*>(A32);
        a2.dst = reinterpret_cast<double*>(B32);
        if (zt) set_z_tiled_out(a2, ncol, nz, zt);
        t0 = stamp(h);
        if ((e = line_pass(a2, h->ty, false, true, x_cplx, s_cplx, h->stream, true)) != cudaSuccess)
            return set_cuda_error(h, e, PP_CUFFT_FAIL_Y);
        stage_done(h, SLOT_YF, t0);
        t0 = stamp(h);
        if ((e = pp_launch_zsolve(z, s_cplx, h->stream)) != cudaSuccess) return set_cuda_error(h, e, PP_THOMAS_FAIL);
        stage_done(h, SLOT_Z, t0);
        PPLinePassArgs a3 = ay;
        a3.src = reinterpret_cast<const double*>(B32);
        a3.dst = reinterpret_cast<double*>(A32);
        if (zt) set_z_tiled_in(a3, ncol, nz, zt);
        t0 = stamp(h);
        if ((e = line_pass(a3, h->ty, true, true, s_cplx, s_cplx, h->stream, true)) != cudaSuccess)
            return set_cuda_error(h, e, PP_CUFFT_FAIL_INV_Y);
        stage_done(h, SLOT_YI, t0);
        PPLinePassArgs a4 = ax;
        a4.src = reinterpret_cast<const double*>(A32);
        a4.dst = last ? (h->ext_out ? h->ext_out : h->out.as<double>()) : nullptr;
        a4.acc = u;
        a4.acc_read = sw > 0;
        a4.zplane = zm ? h->psum.as<double>() : nullptr;
        a4.zscale = 1.0 / (psum_scale * (double)nx * (double)ny);
        a4.out_scale = 1. / ((double)(nx * ny));
        if (hc) set_half_in(a4, ncol, splane, nx, plane);
        t0 = stamp(h);
        if ((e = line_pass(a4, h->tx, true, false, s_cplx, false, h->stream, true)) != cudaSuccess)
            return set_cuda_error(h, e, PP_CUFFT_FAIL_INV_X);
        stage_done(h, SLOT_XI, t0);
    }
    h->last_sweeps = sweeps;
    return zero_mean(h);
}

}  // namespace

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
static void timing_release(pp_solver_s* h)
{
    for (auto& e : h->tev) cudaEventDestroy(e);
    h->tev.clear();
    h->trec.clear();
    h->tmax = h->tcount = h->tnext = 0;
    h->timing = false;
}

extern "C" {

const char* pp_result_string(int code)
{
    switch (code) {
    case PP_SUCCESS: return "SUCCESS";
    case PP_GPU_INIT_FAILURE: return "GPU_INIT_FAILURE: no usable CUDA device";
    case PP_SOLVER_ARRAY_INCONSISTENT: return "SOLVER_ARRAY_INCONSISTENT";
    case PP_MESH_DIVISIBLE: return "MESH_DIVISIBLE";
    case PP_ALLOCATION_FAIL: return "ALLOCATION_FAIL: not enough device memory";
    case PP_THOMAS_FAIL: return "THOMAS_FAIL: the z-direction tridiagonal solve failed";
    case PP_INPUT_ARGS: return "INPUT_ARGS: invalid sizes, boundary letters or box";
    case PP_CUFFT_FAIL_X: return "CUFFT_FAIL_X: forward x transform failed";
    case PP_CUFFT_FAIL_INV_X: return "CUFFT_FAIL_INV_X: inverse x transform failed";
    case PP_CUFFT_FAIL_Y: return "CUFFT_FAIL_Y: forward y transform failed";
    case PP_CUFFT_FAIL_INV_Y: return "CUFFT_FAIL_INV_Y: inverse y transform failed";
    case PP_INVALID_HANDLE: return "INVALID_HANDLE";
    case PP_NOT_READY: return "NOT_READY: boundary conditions or RHS not assigned";
    case PP_CUDA_ERROR: return "CUDA_ERROR";
    case PP_UNSUPPORTED: return "UNSUPPORTED: size or option outside the GPU kernels";
    case PP_NOALLOC_TOO_LARGE: return "NOALLOC_TOO_LARGE: the grid does not fit the 32 MiB scratch of pp_solve_noalloc";
    default: return "UNKNOWN";
    }
}

int pp_default_options(pp_options* opt)
{
    if (!opt) return PP_INPUT_ARGS;
    opt->precision = PP_PRECISION_FP64;
    opt->max_sweeps = 3;
    opt->tolerance = 1e-10;
    opt->compat_zero_mode = 1;
    opt->dirichlet_lift = 1;
    opt->z_solver = PP_ZSOLVE_DIRECT;
    opt->zero_mean = 0;
    return PP_SUCCESS;
}

int pp_create(int nx, int ny, int nz, pp_handle* out)
{
    if (!out) return PP_INPUT_ARGS;
    *out = nullptr;
    if (nx < 2 || ny < 2 || nz < 3) return PP_INPUT_ARGS;
    if (nz > pp_zsolve_max_nz(false, false)) return PP_UNSUPPORTED;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return PP_GPU_INIT_FAILURE;
    pp_solver_s* h = new (std::nothrow) pp_solver_s;
    if (!h) return PP_ALLOCATION_FAIL;
    h->nx = nx;
    h->ny = ny;
    h->nz = nz;
    cudaGetDevice(&h->device);
    pp_default_options(&h->opt);
    const size_t n = (size_t)nx * ny * nz;
    if (h->rhs.alloc(2 * n * sizeof(double)) != cudaSuccess || h->bufA.alloc(2 * n * sizeof(double)) != cudaSuccess ||
        h->bufB.alloc(2 * n * sizeof(double)) != cudaSuccess || h->out.alloc(2 * n * sizeof(double)) != cudaSuccess ||
        h->errc.alloc(sizeof(int)) != cudaSuccess || cudaMemset(h->errc.p, 0, sizeof(int)) != cudaSuccess) {
        // release what did fit (the buffers have no destructor)
        h->rhs.free();
        h->bufA.free();
        h->bufB.free();
        h->out.free();
        h->errc.free();
        cudaGetLastError();
        delete h;
        return PP_ALLOCATION_FAIL;
    }
    *out = h;
    return PP_SUCCESS;
}

int pp_destroy(pp_handle h)
{
    if (!h) return PP_INVALID_HANDLE;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    else cudaDeviceSynchronize();
    h->rhs.free();
    h->bufA.free();
    h->bufB.free();
    h->out.free();
    for (auto& b : h->lift) b.free();
    timing_release(h);
    h->psum.free();
    h->part.free();
    h->errc.free();
    h->zero1.free();
    h->mgstats.free();
    h->zmean.free();
    h->wlong.free();
    h->tx.free_all();
    h->ty.free_all();
    delete h;
    return PP_SUCCESS;
}

int pp_set_box(pp_handle h, const double X[6])
{
    if (!h) return PP_INVALID_HANDLE;
    if (!X) return PP_INPUT_ARGS;
    for (int d = 0; d < 3; ++d)
        if (!(X[2 * d + 1] > X[2 * d]) || !std::isfinite(X[2 * d]) || !std::isfinite(X[2 * d + 1]))
            return PP_INPUT_ARGS;
    std::lock_guard<std::mutex> g(h->mu);
    std::memcpy(h->box, X, sizeof h->box);
    if (h->have_bc) {
        cudaSetDevice(h->device);
        return build_lift(h);
    }
    return PP_SUCCESS;
}

int pp_assign_boundary(pp_handle h, const char bc[6])
{
    if (!h) return PP_INVALID_HANDLE;
    if (!bc || !valid_bc(bc)) return PP_INPUT_ARGS;
    std::lock_guard<std::mutex> g(h->mu);
    cudaSetDevice(h->device);
    std::memcpy(h->bc, bc, 6);
    int rc = rebuild_tables(h);
    h->have_bc = rc == PP_SUCCESS;
    return rc;
}

int pp_set_face_values(pp_handle h, int face, const double* g)
{
    if (!h) return PP_INVALID_HANDLE;
    if (face < 0 || face > 5) return PP_INPUT_ARGS;
    std::lock_guard<std::mutex> lk(h->mu);
    if (!h->have_bc) return PP_NOT_READY;
    if (h->bc[face] == 'P') return PP_INPUT_ARGS;
    const int d = face / 2;
    const size_t n = d == 0 ? (size_t)h->ny * h->nz : (d == 1 ? (size_t)h->nx * h->nz : (size_t)h->nx * h->ny);
    if (g) {
        for (size_t q = 0; q < n; ++q)
            if (!std::isfinite(g[q])) return PP_INPUT_ARGS;
        h->uface[face].assign(g, g + n);
    } else {
        h->uface[face].clear();
    }
    cudaSetDevice(h->device);
    return build_lift(h);
}

int pp_set_options(pp_handle h, const pp_options* opt)
{
    if (!h) return PP_INVALID_HANDLE;
    if (!opt) return PP_INPUT_ARGS;
    if (opt->precision != PP_PRECISION_FP64 && opt->precision != PP_PRECISION_MIXED) return PP_INPUT_ARGS;
    if (opt->max_sweeps < 0 || opt->max_sweeps > 16) return PP_INPUT_ARGS;
    if (opt->z_solver < PP_ZSOLVE_DIRECT || opt->z_solver > PP_ZSOLVE_REF_CRP) return PP_INPUT_ARGS;
    if (opt->zero_mean != 0 && opt->zero_mean != 1) return PP_INPUT_ARGS;
    std::lock_guard<std::mutex> g(h->mu);
    const bool lift_changed = opt->dirichlet_lift != h->opt.dirichlet_lift;
    if (opt->zero_mean && !h->zmean.p) {
        // allocated here, never inside a solve (which may be captured in a graph)
        cudaSetDevice(h->device);
        if (h->zmean.alloc(pp_zero_mean_scratch_doubles() * sizeof(double)) != cudaSuccess) {
            cudaGetLastError();
            return PP_ALLOCATION_FAIL;
        }
    }
    h->opt = *opt;
    if (lift_changed && h->have_bc) {
        cudaSetDevice(h->device);
        return build_lift(h);
    }
    return PP_SUCCESS;
}

int pp_kernel_timeouts(pp_handle h, int* count)
{
    if (!h) return PP_INVALID_HANDLE;
    if (!count) return PP_INPUT_ARGS;
    std::lock_guard<std::mutex> g(h->mu);
    cudaSetDevice(h->device);
    cudaError_t e = cudaMemcpyAsync(count, h->errc.p, sizeof(int), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    return e == cudaSuccess ? PP_SUCCESS : set_cuda_error(h, e, PP_CUDA_ERROR);
}

int pp_zsolve_stats(pp_handle h, int* max_cycles, int* unconverged)
{
    if (!h) return PP_INVALID_HANDLE;
    if (!max_cycles || !unconverged) return PP_INPUT_ARGS;
    std::lock_guard<std::mutex> g(h->mu);
    *max_cycles = 0;
    *unconverged = 0;
    if (!h->mgstats.p) return PP_SUCCESS;
    cudaSetDevice(h->device);
    int v[2] = {0, 0};
    cudaError_t e = cudaMemcpyAsync(v, h->mgstats.p, sizeof(v), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return set_cuda_error(h, e, PP_CUDA_ERROR);
    *max_cycles = v[0];
    *unconverged = v[1];
    return PP_SUCCESS;
}

int pp_get_options(pp_handle h, pp_options* opt)
{
    if (!h) return PP_INVALID_HANDLE;
    if (!opt) return PP_INPUT_ARGS;
    std::lock_guard<std::mutex> g(h->mu);
    *opt = h->opt;
    return PP_SUCCESS;
}

static int assign_common(pp_handle h, const double* src, bool cplx, cudaMemcpyKind kind)
{
    if (!h) return PP_INVALID_HANDLE;
    if (!src) return PP_INPUT_ARGS;
    std::lock_guard<std::mutex> g(h->mu);
    cudaSetDevice(h->device);
    const size_t n = (size_t)h->nx * h->ny * h->nz;
    cudaError_t e = cudaMemcpyAsync(h->rhs.p, src, (cplx ? 2 : 1) * n * sizeof(double), kind, h->stream);
    if (e != cudaSuccess) return set_cuda_error(h, e, PP_CUDA_ERROR);
    if (kind == cudaMemcpyHostToDevice) {
        // the caller may reuse its buffer once this returns
        if ((e = cudaStreamSynchronize(h->stream)) != cudaSuccess) return set_cuda_error(h, e, PP_CUDA_ERROR);
    }
    h->rhs_complex = cplx;
    h->have_rhs = true;
    h->ext_rhs = nullptr;
    return PP_SUCCESS;
}

int pp_assign_rhs_async(pp_handle h, const double* rhs)
{
    if (!h) return PP_INVALID_HANDLE;
    if (!rhs) return PP_INPUT_ARGS;
    std::lock_guard<std::mutex> g(h->mu);
    cudaSetDevice(h->device);
    const size_t n = (size_t)h->nx * h->ny * h->nz;
    cudaError_t e = cudaMemcpyAsync(h->rhs.p, rhs, n * sizeof(double), cudaMemcpyHostToDevice, h->stream);
    if (e != cudaSuccess) return set_cuda_error(h, e, PP_CUDA_ERROR);
    h->rhs_complex = false;
    h->have_rhs = true;
    h->ext_rhs = nullptr;
    return PP_SUCCESS;
}

int pp_bind_device_buffers(pp_handle h, const double* d_rhs, int is_complex, double* d_P)
{
    if (!h) return PP_INVALID_HANDLE;
    std::lock_guard<std::mutex> g(h->mu);
    if (d_rhs) {
        h->ext_rhs = d_rhs;
        h->rhs_complex = is_complex != 0;
        h->have_rhs = true;
    }
    h->ext_out = d_P;
    return PP_SUCCESS;
}

int pp_assign_rhs(pp_handle h, const double* rhs) { return assign_common(h, rhs, false, cudaMemcpyHostToDevice); }
int pp_assign_rhs_complex(pp_handle h, const double* rhs) { return assign_common(h, rhs, true, cudaMemcpyHostToDevice); }
int pp_assign_rhs_device(pp_handle h, const double* d_rhs, int is_complex)
{
    return assign_common(h, d_rhs, is_complex != 0, cudaMemcpyDeviceToDevice);
}

int pp_solve(pp_handle h)
{
    if (!h) return PP_INVALID_HANDLE;
    std::lock_guard<std::mutex> g(h->mu);
    if (!h->have_bc || !h->have_rhs) return PP_NOT_READY;
    if (h->slab) return PP_UNSUPPORTED;  // a slab solves through the staged entry points
    cudaSetDevice(h->device);
    h->timing = h->tcount < h->tmax;
    if (h->timing) h->tcount++;
    const int rc = h->opt.precision == PP_PRECISION_MIXED ? launch_mixed(h) : launch_solve(h);
    h->timing = false;
    if (rc == PP_SUCCESS) h->solved = true;
    return rc;
}

// ---- staged solve of a z-slab (a grid decomposed over several GPUs) ---------------
int pp_set_slab(pp_handle h, int owns_zmin, int owns_zmax)
{
    if (!h) return PP_INVALID_HANDLE;
    std::lock_guard<std::mutex> g(h->mu);
    h->slab = true;
    h->zface_lo = owns_zmin != 0;
    h->zface_hi = owns_zmax != 0;
    if (!h->have_bc) return PP_SUCCESS;
    cudaSetDevice(h->device);
    return build_lift(h);
}

static int stage_ready(pp_solver_s* h)
{
    if (!h->slab) return PP_INPUT_ARGS;
    if (!h->have_bc) return PP_NOT_READY;
    // the staged solve is the plain FP64 solve with the direct z solve
    if (h->opt.precision != PP_PRECISION_FP64 || h->opt.z_solver != PP_ZSOLVE_DIRECT || h->opt.zero_mean)
        return PP_UNSUPPORTED;
    return PP_SUCCESS;
}

int pp_stage_forward(pp_handle h)
{
    if (!h) return PP_INVALID_HANDLE;
    std::lock_guard<std::mutex> g(h->mu);
    if (const int rc = stage_ready(h)) return rc;
    if (!h->have_rhs) return PP_NOT_READY;
    cudaSetDevice(h->device);
    return launch_solve(h, STAGE_FWD);
}

int pp_stage_spectrum(pp_handle h, double** d_spec, int* ncol, int* parts)
{
    if (!h) return PP_INVALID_HANDLE;
    if (!d_spec || !ncol || !parts) return PP_INPUT_ARGS;
    std::lock_guard<std::mutex> g(h->mu);
    if (const int rc = stage_ready(h)) return rc;
    const int hc = half_spectrum_cols(h);
    *d_spec = h->bufB.as<double>();
    *ncol = hc ? hc : h->nx;
    *parts = h->ty.kind == PP_KIND_FFT ? 2 : 1;
    return PP_SUCCESS;
}

int pp_stage_zsolve(pp_handle h, double* d_cols, int nz_total, int rows, int j0)
{
    if (!h) return PP_INVALID_HANDLE;
    std::lock_guard<std::mutex> g(h->mu);
    if (const int rc = stage_ready(h)) return rc;
    if (!d_cols || nz_total < 3 || rows < 1 || j0 < 0 || j0 + rows > h->ny) return PP_INPUT_ARGS;
    if (nz_total > pp_zsolve_max_nz(h->ty.kind == PP_KIND_FFT, false)) return PP_UNSUPPORTED;
    cudaSetDevice(h->device);
    const StageZ sz{d_cols, nz_total, rows, j0};
    return launch_solve(h, STAGE_Z, &sz);
}

int pp_stage_inverse(pp_handle h)
{
    if (!h) return PP_INVALID_HANDLE;
    std::lock_guard<std::mutex> g(h->mu);
    if (const int rc = stage_ready(h)) return rc;
    cudaSetDevice(h->device);
    const int rc = launch_solve(h, STAGE_INV);
    if (rc == PP_SUCCESS) h->solved = true;
    return rc;
}

int pp_timing_begin(pp_handle h, int max_solves)
{
    if (!h) return PP_INVALID_HANDLE;
    if (max_solves < 1) return PP_INPUT_ARGS;
    std::lock_guard<std::mutex> g(h->mu);
    cudaSetDevice(h->device);
    timing_release(h);
    // two events per stage; a refined solve has 6 stages per sweep
    const int sweeps = h->opt.max_sweeps > 0 ? h->opt.max_sweeps : 0;
    h->tev.resize((size_t)max_solves * 2 * 6 * (sweeps + 1));
    for (auto& e : h->tev)
        if (cudaEventCreate(&e) != cudaSuccess) {
            e = nullptr;
            timing_release(h);
            return PP_CUDA_ERROR;
        }
    h->tmax = max_solves;
    h->tcount = 0;
    return PP_SUCCESS;
}

int pp_timing_end(pp_handle h, double* kernel_ms_total, int n, int* solves)
{
    if (!h) return PP_INVALID_HANDLE;
    if (!kernel_ms_total || n < PP_SOLVE_STAGES || !solves) return PP_INPUT_ARGS;
    std::lock_guard<std::mutex> g(h->mu);
    cudaSetDevice(h->device);
    for (int i = 0; i < PP_SOLVE_STAGES; ++i) kernel_ms_total[i] = 0.0;
    *solves = h->tcount;
    int rc = PP_SUCCESS;
    if (!h->trec.empty()) {
        cudaError_t e = cudaEventSynchronize(h->tev[h->trec.back().e1]);
        if (e != cudaSuccess) rc = set_cuda_error(h, e, PP_CUDA_ERROR);
        for (const auto& r : h->trec) {
            if (rc != PP_SUCCESS) break;
            float ms = 0.f;
            cudaEventElapsedTime(&ms, h->tev[r.e0], h->tev[r.e1]);
            kernel_ms_total[r.slot] += ms;
        }
    }
    timing_release(h);
    return rc;
}

int pp_profile_solve(pp_handle h, double* kernel_ms, int n)
{
    if (!h) return PP_INVALID_HANDLE;
    if (!kernel_ms || n < PP_SOLVE_STAGES) return PP_INPUT_ARGS;
    int rc = pp_timing_begin(h, 1);
    if (rc != PP_SUCCESS) return rc;
    rc = pp_solve(h);
    int solves = 0;
    const int rc2 = pp_timing_end(h, kernel_ms, n, &solves);
    return rc != PP_SUCCESS ? rc : rc2;
}

int pp_get_solution(pp_handle h, double* P)
{
    if (!h) return PP_INVALID_HANDLE;
    if (!P) return PP_INPUT_ARGS;
    std::lock_guard<std::mutex> g(h->mu);
    cudaSetDevice(h->device);
    const size_t n = (size_t)h->nx * h->ny * h->nz;
    const void* src = h->ext_out ? (const void*)h->ext_out : h->out.p;
    cudaError_t e = cudaMemcpyAsync(P, src, 2 * n * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    return e == cudaSuccess ? PP_SUCCESS : set_cuda_error(h, e, PP_CUDA_ERROR);
}

int pp_get_solution_async(pp_handle h, double* P)
{
    if (!h) return PP_INVALID_HANDLE;
    if (!P) return PP_INPUT_ARGS;
    std::lock_guard<std::mutex> g(h->mu);
    cudaSetDevice(h->device);
    const size_t n = (size_t)h->nx * h->ny * h->nz;
    const void* src = h->ext_out ? (const void*)h->ext_out : h->out.p;
    cudaError_t e = cudaMemcpyAsync(P, src, 2 * n * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
    return e == cudaSuccess ? PP_SUCCESS : set_cuda_error(h, e, PP_CUDA_ERROR);
}

// the real part of the solution packed into the (free after the solve)
// workspace A, copied to the host; the caller's next solve on this handle's
// stream starts after the copy
static int get_real(pp_handle h, double* u, bool wait)
{
    if (!h) return PP_INVALID_HANDLE;
    if (!u) return PP_INPUT_ARGS;
    std::lock_guard<std::mutex> g(h->mu);
    cudaSetDevice(h->device);
    const size_t n = (size_t)h->nx * h->ny * h->nz;
    const double* src = h->ext_out ? h->ext_out : h->out.as<double>();
    if (reinterpret_cast<uintptr_t>(src) % 16) return PP_INPUT_ARGS;
    double* pack = h->bufA.as<double>();
    cudaError_t e = pp_launch_real_part(src, pack, (long)n, h->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(u, pack, n * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess && wait) e = cudaStreamSynchronize(h->stream);
    return e == cudaSuccess ? PP_SUCCESS : set_cuda_error(h, e, PP_CUDA_ERROR);
}

int pp_get_solution_real(pp_handle h, double* u) { return get_real(h, u, true); }

int pp_io(pp_handle h, unsigned app, int dir, int aligndir)
{
    if (!h) return PP_INVALID_HANDLE;
    if (dir < 0 || dir > 2 || aligndir < 0 || aligndir > 2) return PP_INPUT_ARGS;
    const int nx = h->nx, ny = h->ny, nz = h->nz;
    double box[6];
    {
        std::lock_guard<std::mutex> g(h->mu);
        if (!h->solved) return PP_NOT_READY;
        std::memcpy(box, h->box, sizeof box);
    }
    std::vector<double> q((size_t)nx * ny * nz);
    const int rc = pp_get_solution_real(h, q.data());
    if (rc != PP_SUCCESS) return rc;
    if (mkdir("soln", 0755) != 0 && errno != EEXIST) return PP_INPUT_ARGS;
    char base[64], path[96];
    std::snprintf(base, sizeof base, "Pxdmf3d%u", app);
    // the attribute values, little-endian float64 (the host's order on x86-64 / aarch64)
    std::snprintf(path, sizeof path, "soln/%s_Q.bin", base);
    FILE* f = std::fopen(path, "wb");
    if (!f) return PP_INPUT_ARGS;
    const size_t wrote = std::fwrite(q.data(), sizeof(double), q.size(), f);
    if (std::fclose(f) != 0 || wrote != q.size()) return PP_INPUT_ARGS;
    std::snprintf(path, sizeof path, "soln/%s.xmf", base);
    f = std::fopen(path, "w");
    if (!f) return PP_INPUT_ARGS;
    const double dx = (box[1] - box[0]) / nx, dy = (box[3] - box[2]) / ny, dz = (box[5] - box[4]) / nz;
    int bad = 0;
    bad |= std::fprintf(f, "<?xml version=\"1.0\" ?>\n<!DOCTYPE Xdmf SYSTEM \"Xdmf.dtd\" []>\n") < 0;
    bad |= std::fprintf(f, "<Xdmf Version=\"2.0\">\n<Domain>\n") < 0;
    bad |= std::fprintf(f, "<Grid Name=\"AMR\" GridType=\"Collection\" CollectionType=\"Spatial\">\n") < 0;
    bad |= std::fprintf(f, "  <Grid Name=\"mesh0\" GridType=\"Uniform\">\n") < 0;
    bad |= std::fprintf(f, "    <Topology TopologyType=\"3DCoRectMesh\" Dimensions=\"%d %d %d\"/>\n", nz + 1, ny + 1,
                        nx + 1) < 0;
    // XDMF lists a CoRectMesh's origin and spacing slowest axis first (z y x)
    bad |= std::fprintf(f, "    <Geometry GeometryType=\"ORIGIN_DXDYDZ\">\n") < 0;
    bad |= std::fprintf(f, "      <DataItem Dimensions=\"3\" NumberType=\"Float\" Precision=\"8\" Format=\"XML\">"
                           "%.17g %.17g %.17g</DataItem>\n", box[4], box[2], box[0]) < 0;
    bad |= std::fprintf(f, "      <DataItem Dimensions=\"3\" NumberType=\"Float\" Precision=\"8\" Format=\"XML\">"
                           "%.17g %.17g %.17g</DataItem>\n", dz, dy, dx) < 0;
    bad |= std::fprintf(f, "    </Geometry>\n") < 0;
    bad |= std::fprintf(f, "    <Attribute Name=\"Q\" AttributeType=\"Scalar\" Center=\"Cell\">\n") < 0;
    bad |= std::fprintf(f, "      <DataItem Dimensions=\"%d %d %d\" NumberType=\"Float\" Precision=\"8\" "
                           "Format=\"Binary\" Endian=\"Little\">%s_Q.bin</DataItem>\n", nz, ny, nx, base) < 0;
    bad |= std::fprintf(f, "    </Attribute>\n  </Grid>\n</Grid>\n</Domain>\n</Xdmf>\n") < 0;
    if (std::fclose(f) != 0 || bad) return PP_INPUT_ARGS;
    return PP_SUCCESS;
}
int pp_get_solution_real_async(pp_handle h, double* u) { return get_real(h, u, false); }

int pp_get_solution_device(pp_handle h, double* d_P)
{
    if (!h) return PP_INVALID_HANDLE;
    if (!d_P) return PP_INPUT_ARGS;
    std::lock_guard<std::mutex> g(h->mu);
    cudaSetDevice(h->device);
    const size_t n = (size_t)h->nx * h->ny * h->nz;
    const void* src = h->ext_out ? (const void*)h->ext_out : h->out.p;
    if (src == (const void*)d_P) return PP_SUCCESS;
    cudaError_t e = cudaMemcpyAsync(d_P, src, 2 * n * sizeof(double), cudaMemcpyDeviceToDevice, h->stream);
    return e == cudaSuccess ? PP_SUCCESS : set_cuda_error(h, e, PP_CUDA_ERROR);
}

int pp_solution_device_ptr(pp_handle h, const double** d_P)
{
    if (!h) return PP_INVALID_HANDLE;
    if (!d_P) return PP_INPUT_ARGS;
    std::lock_guard<std::mutex> g(h->mu);
    *d_P = h->ext_out ? h->ext_out : h->out.as<double>();
    return PP_SUCCESS;
}

int pp_get_error_manufactured(pp_handle h, double* err)
{
    if (!h) return PP_INVALID_HANDLE;
    if (!err) return PP_INPUT_ARGS;
    double box[6];
    char bc[6];
    {
        std::lock_guard<std::mutex> g(h->mu);
        if (!h->have_bc) return PP_NOT_READY;
        std::memcpy(box, h->box, sizeof box);
        std::memcpy(bc, h->bc, sizeof bc);
    }
    const int nx = h->nx, ny = h->ny, nz = h->nz;
    const size_t n = (size_t)nx * ny * nz;
    std::vector<double> P(2 * n);
    int rc = pp_get_solution(h, P.data());
    if (rc != PP_SUCCESS) return rc;
    // getError (src/pencilDcmp.cpp:2040-2208), INITANALYTIC = 1 branch
    const double pi = PP_REF_PI;
    const double Xa = box[0], Ya = box[2], Za = box[4];
    const double c1 = -(box[0] - box[1]) / (nx);
    const double c2 = -(box[2] - box[3]) / (ny);
    const double c3 = -(box[4] - box[5]) / (nz);
    const double omega[3] = {1 * pi, 2 * pi, 3 * pi};
    const int t0 = ref_tag_xy(kind_from_bc(bc[0], bc[1]));
    const int t1 = ref_tag_xy(kind_from_bc(bc[2], bc[3]));
    const int t2 = ref_tag_z(bc);
    const bool pxy = bc[0] == 'P' || bc[2] == 'P';
    const bool pall = bc[0] == 'P' && bc[2] == 'P' && bc[4] == 'P';
    double acc = 0.0;
    for (int k = 0; k < nz; ++k) {
        const double z = Za + k * c3 + 1.0 * c3 * 0.5;
        for (int j = 0; j < ny; ++j) {
            const double y = Ya + j * c2 + 1.0 * c2 * 0.5;
            for (int i = 0; i < nx; ++i) {
                const double x = Xa + i * c1 + 1.0 * c1 * .5;
                const size_t p = i + (size_t)nx * j + (size_t)nx * ny * k;
                double val, val1;
                if (pxy) {
                    val = P[2 * p] - (sin(omega[1] * z) * cos(omega[1] * (x + y)));
                    val1 = P[2 * p + 1] - (sin(omega[1] * z) * sin(omega[1] * (x + y)));
                } else {
                    val = P[2 * p] - pp_exact_value(omega[0], x, t0) * pp_exact_value(omega[1], y, t1) *
                                         pp_exact_value(omega[2], z, t2);
                    val1 = 0.0;
                }
                if (pall) {
                    val = P[2 * p] - cos(omega[1] * (x + y + z));
                    val1 = P[2 * p + 1] - sin(omega[1] * (x + y + z));
                }
                acc += val * val + val1 * val1;
            }
        }
    }
    *err = sqrt(acc / (double)n);
    return PP_SUCCESS;
}

int pp_fill_trigonometric_box(int nx, int ny, int nz, const double X[6], double* rhs)
{
    if (!X || !rhs || nx < 1 || ny < 1 || nz < 1) return PP_INPUT_ARGS;
    for (int d = 0; d < 3; ++d)
        if (!(X[2 * d + 1] > X[2 * d]) || !std::isfinite(X[2 * d]) || !std::isfinite(X[2 * d + 1]))
            return PP_INPUT_ARGS;
    // the reference's SHIFT = 1 branch: cell centres with the cell size
    // dxyz[2] of setDxyz (src/pencilDcmp.cpp:828-830) and pi = 4 atan(1)
    const double pi = 4. * atan(1.0);
    const double c3 = -(X[4] - X[5]) / (nz);
    const double shift = 1.0;
    const size_t plane = (size_t)nx * ny;
    for (int k = 0; k < nz; ++k) {
        const double z = X[4] + k * c3 + shift * c3 * 0.5;
        const double v = -4. * pi * pi * cos(2. * pi * z);
        std::fill(rhs + plane * k, rhs + plane * (k + 1), v);
    }
    return PP_SUCCESS;
}

int pp_fill_trigonometric(pp_handle h, double* rhs)
{
    if (!h) return PP_INVALID_HANDLE;
    double box[6];
    {
        std::lock_guard<std::mutex> g(h->mu);
        std::memcpy(box, h->box, sizeof box);
    }
    return pp_fill_trigonometric_box(h->nx, h->ny, h->nz, box, rhs);
}

int pp_set_stream(pp_handle h, void* stream)
{
    if (!h) return PP_INVALID_HANDLE;
    std::lock_guard<std::mutex> g(h->mu);
    h->stream = (cudaStream_t)stream;
    return PP_SUCCESS;
}

int pp_synchronize(pp_handle h)
{
    if (!h) return PP_INVALID_HANDLE;
    cudaSetDevice(h->device);
    cudaError_t e = cudaStreamSynchronize(h->stream);
    return e == cudaSuccess ? PP_SUCCESS : set_cuda_error(h, e, PP_CUDA_ERROR);
}

int pp_host_alloc(size_t bytes, void** p)
{
    if (!p) return PP_INPUT_ARGS;
    cudaError_t e = cudaHostAlloc(p, bytes, cudaHostAllocDefault);
    return e == cudaSuccess ? PP_SUCCESS : PP_ALLOCATION_FAIL;
}

int pp_host_free(void* p)
{
    cudaError_t e = cudaFreeHost(p);
    return e == cudaSuccess ? PP_SUCCESS : PP_CUDA_ERROR;
}

int pp_workspace_bytes(pp_handle h, size_t* bytes)
{
    if (!h) return PP_INVALID_HANDLE;
    if (!bytes) return PP_INPUT_ARGS;
    std::lock_guard<std::mutex> g(h->mu);
    size_t b = h->rhs.bytes + h->bufA.bytes + h->bufB.bytes + h->out.bytes;
    for (auto& l : h->lift) b += l.bytes;
    for (const DirTables* t : {&h->tx, &h->ty})
        b += t->tw.bytes + t->cs.bytes + t->eig.bytes + t->twf.bytes + t->csf.bytes;
    b += h->psum.bytes + h->part.bytes + h->errc.bytes + h->zero1.bytes + h->mgstats.bytes + h->zmean.bytes;
    b += h->wlong.bytes;
    for (const DirTables* t : {&h->tx, &h->ty}) b += t->long_bytes();
    *bytes = b;
    return PP_SUCCESS;
}

static bool valid_tuning(const pp_solver_s* h, const pp_tuning* t)
{
    if (t->zsolve_lanes != 0 && !pp_zsolve_valid_lanes(h->nz, t->zsolve_lanes)) return false;
    if (t->line_tile < 0 || t->line_tile > 32) return false;
    if (t->zsolve_tile != 0 && (t->zsolve_tile < 1 || t->zsolve_tile > 32 || (t->zsolve_tile & (t->zsolve_tile - 1))))
        return false;
    return true;
}

int pp_set_tuning(pp_handle h, const pp_tuning* t)
{
    if (!h) return PP_INVALID_HANDLE;
    if (!t || !valid_tuning(h, t)) return PP_INPUT_ARGS;
    std::lock_guard<std::mutex> g(h->mu);
    h->tune = *t;
    return PP_SUCCESS;
}

int pp_get_tuning(pp_handle h, pp_tuning* t)
{
    if (!h) return PP_INVALID_HANDLE;
    if (!t) return PP_INPUT_ARGS;
    std::lock_guard<std::mutex> g(h->mu);
    *t = h->tune;
    return PP_SUCCESS;
}

// milliseconds per solve of one launch shape: one untimed solve, then reps
// solves between two events on the handle's stream
static int time_config(pp_handle h, const pp_tuning& t, int reps, cudaEvent_t e0, cudaEvent_t e1, double* ms)
{
    {
        std::lock_guard<std::mutex> g(h->mu);
        h->tune = t;
    }
    int rc = pp_solve(h);
    if (rc != PP_SUCCESS) return rc;
    cudaError_t e = cudaEventRecord(e0, h->stream);
    if (e != cudaSuccess) return set_cuda_error(h, e, PP_CUDA_ERROR);
    for (int r = 0; r < reps && rc == PP_SUCCESS; ++r) rc = pp_solve(h);
    if (rc != PP_SUCCESS) return rc;
    if ((e = cudaEventRecord(e1, h->stream)) == cudaSuccess) e = cudaEventSynchronize(e1);
    if (e != cudaSuccess) return set_cuda_error(h, e, PP_CUDA_ERROR);
    float f = 0.f;
    if ((e = cudaEventElapsedTime(&f, e0, e1)) != cudaSuccess) return set_cuda_error(h, e, PP_CUDA_ERROR);
    *ms = f / reps;
    return PP_SUCCESS;
}

int pp_autotune(pp_handle h, int reps, pp_tuning* chosen, double* best_ms)
{
    if (!h) return PP_INVALID_HANDLE;
    if (reps < 1 || reps > 100) return PP_INPUT_ARGS;
    pp_tuning start;
    {
        std::lock_guard<std::mutex> g(h->mu);
        if (!h->have_bc || !h->have_rhs) return PP_NOT_READY;
        start = h->tune;
    }
    cudaSetDevice(h->device);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
        if (e0) cudaEventDestroy(e0);
        return PP_CUDA_ERROR;
    }
    pp_tuning best{0, 0, 0};
    double bms = 0.0;
    int rc = time_config(h, best, reps, e0, e1, &bms);
    // z solve: lane counts around the default
    for (int P = 1; P <= 32 && rc == PP_SUCCESS; P *= 2) {
        if (!pp_zsolve_valid_lanes(h->nz, P)) continue;
        pp_tuning t = best;
        t.zsolve_lanes = P;
        double ms = 0.0;
        rc = time_config(h, t, reps, e0, e1, &ms);
        if (rc == PP_SUCCESS && ms < bms) {
            bms = ms;
            best = t;
        }
    }
    // z solve: systems per CTA with the chosen lane count
    for (int T = 2; T <= 32 && rc == PP_SUCCESS; T *= 2) {
        pp_tuning t = best;
        t.zsolve_tile = T;
        double ms = 0.0;
        rc = time_config(h, t, reps, e0, e1, &ms);
        if (rc == PP_SUCCESS && ms < bms) {
            bms = ms;
            best = t;
        }
    }
    // generic transform kernel: lines per tile, only where it runs
    const bool generic = reg_lines(h->nx) == 0 || reg_lines(h->ny) == 0;
    for (int L = 1; generic && L <= 32 && rc == PP_SUCCESS; L *= 2) {
        pp_tuning t = best;
        t.line_tile = L;
        double ms = 0.0;
        rc = time_config(h, t, reps, e0, e1, &ms);
        if (rc == PP_SUCCESS && ms < bms) {
            bms = ms;
            best = t;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    std::lock_guard<std::mutex> g(h->mu);
    h->tune = rc == PP_SUCCESS ? best : start;
    if (rc != PP_SUCCESS) return rc;
    if (chosen) *chosen = best;
    if (best_ms) *best_ms = bms;
    return PP_SUCCESS;
}

}  // extern "C"
