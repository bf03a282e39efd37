// Restatement of FFTW's published transform definitions for the single-rank
// reference build.  TEST INFRASTRUCTURE ONLY (oracle/_ref).  See fftw3.h.
#include "fftw3.h"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

struct pp_shim_fftw_plan_s {
    int n;
    int sign;
    int kind;  // -1: complex DFT, else r2r kind
    void* in;
    void* out;
};

static int shim_fast()
{
    static int mode = -1;
    if (mode < 0) {
        const char* e = std::getenv("PP_SHIM_FFT");
        mode = (e && std::strcmp(e, "fast") == 0) ? 1 : 0;
    }
    return mode;
}

extern "C" void* fftw_malloc(size_t n) { return std::malloc(n); }
extern "C" void fftw_free(void* p) { std::free(p); }

extern "C" fftw_plan fftw_plan_dft_1d(int n, fftw_complex* in, fftw_complex* out, int sign, unsigned)
{
    fftw_plan p = new pp_shim_fftw_plan_s;
    p->n = n;
    p->sign = sign;
    p->kind = -1;
    p->in = in;
    p->out = out;
    return p;
}

extern "C" fftw_plan fftw_plan_r2r_1d(int n, double* in, double* out, fftw_r2r_kind kind, unsigned)
{
    fftw_plan p = new pp_shim_fftw_plan_s;
    p->n = n;
    p->sign = 0;
    p->kind = kind;
    p->in = in;
    p->out = out;
    return p;
}

extern "C" void fftw_destroy_plan(fftw_plan p) { delete p; }
extern "C" void fftw_cleanup(void) {}

// ---- long double mixed-radix DFT (decimation in time on the smallest factor)
template <typename R>
static void dft_rec(const R* wr, const R* wi, int N, const R* xr, const R* xi, int stride, int n, R* yr, R* yi)
{
    if (n == 1) {
        yr[0] = xr[0];
        yi[0] = xi[0];
        return;
    }
    int p = n;
    for (int f = 2; f * f <= n; ++f)
        if (n % f == 0) {
            p = f;
            break;
        }
    int m = n / p;
    if (p == n) {
        for (int k = 0; k < n; ++k) {
            R ar = 0, ai = 0;
            for (int j = 0; j < n; ++j) {
                long long e = ((long long)j * k) % n * (N / n);
                R vr = xr[(long)j * stride], vi = xi[(long)j * stride];
                ar += vr * wr[e] - vi * wi[e];
                ai += vr * wi[e] + vi * wr[e];
            }
            yr[k] = ar;
            yi[k] = ai;
        }
        return;
    }
    std::vector<R> s(2 * (size_t)n);
    R* sr = s.data();
    R* si = sr + n;
    for (int r = 0; r < p; ++r)
        dft_rec<R>(wr, wi, N, xr + (long)r * stride, xi + (long)r * stride, stride * p, m, sr + r * m, si + r * m);
    for (int k = 0; k < n; ++k) {
        int kk = k % m;
        R ar = 0, ai = 0;
        for (int r = 0; r < p; ++r) {
            long long e = ((long long)r * k) % n * (N / n);
            R vr = sr[r * m + kk], vi = si[r * m + kk];
            ar += vr * wr[e] - vi * wi[e];
            ai += vr * wi[e] + vi * wr[e];
        }
        yr[k] = ar;
        yi[k] = ai;
    }
}

template <typename R>
static void dft_complex(int n, int sign, const double* in, double* out)
{
    std::vector<R> w(2 * (size_t)n), x(2 * (size_t)n), y(2 * (size_t)n);
    const R two_pi = (R)6.283185307179586476925286766559005768L;
    for (int m = 0; m < n; ++m) {
        R a = two_pi * (R)m / (R)n;
        w[m] = std::cos(a);
        w[n + m] = (sign < 0 ? -1 : 1) * std::sin(a);
    }
    for (int j = 0; j < n; ++j) {
        x[j] = in[2 * j];
        x[n + j] = in[2 * j + 1];
    }
    dft_rec<R>(w.data(), w.data() + n, n, x.data(), x.data() + n, 1, n, y.data(), y.data() + n);
    for (int k = 0; k < n; ++k) {
        out[2 * k] = (double)y[k];
        out[2 * k + 1] = (double)y[n + k];
    }
}

// FFTW manual, "1d Real-even DFTs (DCTs)" / "1d Real-odd DFTs (DSTs)"
static void r2r_direct(int n, int kind, const double* in, double* out)
{
    const long double pi = 3.141592653589793238462643383279502884L;
    std::vector<long double> y(n);
    for (int k = 0; k < n; ++k) {
        long double acc = 0.0L;
        switch (kind) {
        case FFTW_REDFT10:
            for (int j = 0; j < n; ++j) acc += 2.0L * in[j] * cosl(pi * (2 * j + 1) * k / (2.0L * n));
            break;
        case FFTW_REDFT01:
            acc = in[0];
            for (int j = 1; j < n; ++j) acc += 2.0L * in[j] * cosl(pi * j * (2 * k + 1) / (2.0L * n));
            break;
        case FFTW_RODFT10:
            for (int j = 0; j < n; ++j) acc += 2.0L * in[j] * sinl(pi * (2 * j + 1) * (k + 1) / (2.0L * n));
            break;
        case FFTW_RODFT01:
            acc = ((k % 2) ? -1.0L : 1.0L) * in[n - 1];
            for (int j = 0; j < n - 1; ++j) acc += 2.0L * in[j] * sinl(pi * (j + 1) * (2 * k + 1) / (2.0L * n));
            break;
        default:
            std::fprintf(stderr, "fftw shim: r2r kind %d not provided\n", kind);
            std::abort();
        }
        y[k] = acc;
    }
    for (int k = 0; k < n; ++k) out[k] = (double)y[k];
}

extern "C" void fftw_execute(const fftw_plan p)
{
    if (p->kind >= 0) {
        r2r_direct(p->n, p->kind, (const double*)p->in, (double*)p->out);
        return;
    }
    if (shim_fast())
        dft_complex<double>(p->n, p->sign, (const double*)p->in, (double*)p->out);
    else
        dft_complex<long double>(p->n, p->sign, (const double*)p->in, (double*)p->out);
}
