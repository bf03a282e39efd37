/*
 * pp_oracle.c -- CPU restatement of PittPack's single-rank FFT-FFT-tridiagonal
 * Poisson solve.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: it is loaded by the
 * tests, by the smoke check and by the CPU-baseline leg of bench.py.  The
 * product (pittpack_b200/) never links, loads or calls it.
 *
 * Every step below restates the reference algorithm in plain C, step by step,
 * in double precision as the reference computes it.  The only arithmetic that
 * is not the reference's own is the 1-D DFT: the reference calls FFTW 3.3.x
 * (fftw_plan_dft_1d, FFTW_FORWARD = exp(-2*pi*i*jk/N), unnormalised;
 * src/poissonCPU.cpp:40-234) or cuFFT Z2Z (src/poissonGPU.cpp:5-97).  Neither
 * library is part of the reference tree; the published definition of that DFT
 * is restated here as a mixed-radix FFT carried out in long double and rounded
 * to double, i.e. an (almost) exactly rounded DFT.
 *
 * Paths are relative to the PittPack source tree.
 *   step order ........ src/pencilDcmp.cpp:5801-6430 (PencilDcmp::pittPack)
 *   BC -> transforms .. src/pencilDcmp.cpp:3578-3732 (assignBoundary, extractTag,
 *                       detectTransforms), eigen parameters 3533-3576, scale 3670-3683
 *   RHS scaling ....... src/pencilDcmp.cpp:5591-5647 (assignRhs)
 *   Dirichlet lift .... src/pencilDcmp.cpp:4623-4835 (modifyRhsDirichlet),
 *                       exactValue 1837-1866
 *   DCT/DST pre/post .. src/signalProc.cpp:32-265
 *   eigenvalue ........ src/pencilDcmp.cpp:4393-4417 (getEigenVal)
 *   z-solve ........... src/pencilDcmp.cpp:5066-5105 (solveThmBatch),
 *                       src/triDiag.cpp:1629-1886 (thomasLowMem*),
 *                       src/triDiag.cpp:1961-2255 (shermanMorrisonThomas*)
 *   rescale ........... src/pencilDcmp.cpp:3503-3531
 *   layout ............ src/chunkedArray.cpp:100-199: P[2*(i+nx*j+nx*ny*k)+{0,1}]
 *   manufactured sol .. src/pencilDcmp.cpp:1871-2208, params COEFF0..2 = 1,2,3
 *
 * Extensions that the reference does not have (marked EXT below):
 *   - the N-D / D-N x or y families (DCT-IV / DST-IV).  The reference maps an
 *     N-D pair to transform 'U' and leaves its eigen parameters unset
 *     (src/pencilDcmp.cpp:3685-3732, 3533-3570), so these have no reference
 *     result; the oracle states them from the mathematics.
 *   - exact zero mode (compat_zero_mode = 0): the reference replaces row 0 of
 *     the kx=ky=0 z-system by x0 = r0 whatever the z boundary is
 *     (src/triDiag.cpp:1753-1776).  With compat_zero_mode = 0 that pin is kept
 *     only where the true system is singular (no Dirichlet end in z).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "pp_oracle.h"

/* the constant of src/include/params.h (const double pi) */
static const double REF_PI = 3.1415926535897932384;

/* ------------------------------------------------------------------------- */
/* transform kinds per direction                                              */
/* ------------------------------------------------------------------------- */
/* DST = tag 0, DCT = tag 1, FFT = tag 2 in the reference (extractTag,
 * src/pencilDcmp.cpp:3636-3668); ND/DN are EXT. */
int ppo_kind_from_bc(char lo, char hi)
{
    if (lo == 'D' && hi == 'D') return PPO_DST2;
    if (lo == 'N' && hi == 'N') return PPO_DCT2;
    if (lo == 'P' && hi == 'P') return PPO_FFT;
    if (lo == 'N' && hi == 'D') return PPO_DCT4;
    if (lo == 'D' && hi == 'N') return PPO_DST4;
    return PPO_BAD;
}

/* the reference's tag as used by exactValue (tags[] of extractTag): DST 0,
 * DCT 1, FFT 2, anything else -1 */
static int ref_tag_xy(int kind)
{
    switch (kind) {
    case PPO_DST2: return 0;
    case PPO_DCT2: return 1;
    case PPO_FFT: return 2;
    default: return -1;
    }
}

/* tags[2] of extractTag: z transform from detectTransforms (only 'F' survives
 * when x or y has no transform; with all three directions transformable the
 * z transform is reset to 'U'), then overwritten by bc[4] == 'D' -> -1,
 * bc[4] == 'N' -> -2 */
static int ref_tag_z(const char* bc)
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

/* ------------------------------------------------------------------------- */
/* exactly rounded DFT (FFTW's unnormalised definition) in long double        */
/* ------------------------------------------------------------------------- */
typedef struct {
    int n;
    long double* wr; /* exp(sign 2 pi i m / n), m < n */
    long double* wi;
} dft_plan;

static void dft_plan_init(dft_plan* p, int n, int sign)
{
    p->n = n;
    p->wr = (long double*)malloc(sizeof(long double) * n);
    p->wi = (long double*)malloc(sizeof(long double) * n);
    const long double two_pi = 6.283185307179586476925286766559005768L;
    for (int m = 0; m < n; ++m) {
        long double a = two_pi * (long double)m / (long double)n;
        p->wr[m] = cosl(a);
        p->wi[m] = (sign < 0 ? -1.0L : 1.0L) * sinl(a);
    }
}

static void dft_plan_free(dft_plan* p)
{
    free(p->wr);
    free(p->wi);
}

static int smallest_factor(int n)
{
    for (int p = 2; p * p <= n; ++p)
        if (n % p == 0) return p;
    return n;
}

/* y[k] = sum_j x[j*stride] w^(j*k*(N/n)), n | N; x and y do not alias.
 * Recursive mixed-radix Cooley-Tukey on the smallest prime factor; prime
 * lengths fall back to the direct sum.  Each level owns its scratch. */
static void dft_rec(const dft_plan* P, const long double* xr, const long double* xi, int stride, int n,
                         long double* yr, long double* yi)
{
    if (n == 1) {
        yr[0] = xr[0];
        yi[0] = xi[0];
        return;
    }
    int p = smallest_factor(n);
    int m = n / p;
    int N = P->n;
    if (p == n) {
        for (int k = 0; k < n; ++k) {
            long double ar = 0.0L, ai = 0.0L;
            for (int j = 0; j < n; ++j) {
                long long e = ((long long)j * k) % n * (N / n);
                long double vr = xr[(long)j * stride], vi = xi[(long)j * stride];
                ar += vr * P->wr[e] - vi * P->wi[e];
                ai += vr * P->wi[e] + vi * P->wr[e];
            }
            yr[k] = ar;
            yi[k] = ai;
        }
        return;
    }
    long double* sr = (long double*)malloc(sizeof(long double) * 2 * n);
    long double* si = sr + n;
    for (int r = 0; r < p; ++r)
        dft_rec(P, xr + (long)r * stride, xi + (long)r * stride, stride * p, m, sr + r * m, si + r * m);
    for (int k = 0; k < n; ++k) {
        int kk = k % m;
        long double ar = 0.0L, ai = 0.0L;
        for (int r = 0; r < p; ++r) {
            long long e = ((long long)r * k) % n * (N / n);
            long double vr = sr[r * m + kk], vi = si[r * m + kk];
            ar += vr * P->wr[e] - vi * P->wi[e];
            ai += vr * P->wi[e] + vi * P->wr[e];
        }
        yr[k] = ar;
        yi[k] = ai;
    }
    free(sr);
}

static void dft_line(const dft_plan* P, double* re, double* im)
{
    int n = P->n;
    long double* xr = (long double*)malloc(sizeof(long double) * n * 4);
    long double* xi = xr + n;
    long double* yr = xi + n;
    long double* yi = yr + n;
    for (int j = 0; j < n; ++j) {
        xr[j] = re[j];
        xi[j] = im[j];
    }
    dft_rec(P, xr, xi, 1, n, yr, yi);
    for (int j = 0; j < n; ++j) {
        re[j] = (double)yr[j];
        im[j] = (double)yi[j];
    }
    free(xr);
}

/* public: one unnormalised DFT, sign -1 forward / +1 backward */
void ppo_dft(int n, int sign, double* re, double* im)
{
    dft_plan P;
    dft_plan_init(&P, n, sign);
    dft_line(&P, re, im);
    dft_plan_free(&P);
}

/* ------------------------------------------------------------------------- */
/* DCT/DST pre- and post-processing, src/signalProc.cpp                        */
/* ------------------------------------------------------------------------- */
/* swap: x'[j] = (-1)^j x[N-1-j], imaginary part cleared (signalProc.cpp:242-265) */
static void sp_swap(double* re, double* im, int n, double* t)
{
    for (int j = 0; j < n; ++j) {
        t[j] = re[n - j - 1];
        if (j % 2 == 1) t[j] = -t[j];
    }
    for (int j = 0; j < n; ++j) {
        re[j] = t[j];
        im[j] = 0.0;
    }
}

/* Makhoul even/odd reorder (signalProc.cpp:160-195) */
static void sp_dct10_pre(double* re, double* im, int n, double* t)
{
    int upper = (n - 1) / 2 + 1;
    int odd = n % 2;
    for (int j = 0; j < upper; ++j) t[j] = re[2 * j];
    for (int j = upper; j < n; ++j) t[j] = re[n - 2 * (j - upper) - 1 - odd];
    for (int j = 0; j < n; ++j) {
        re[j] = t[j];
        im[j] = 0.0;
    }
}

/* Hermitian fill, then X_j = 2 (Re V_j cos th + Im V_j sin th), th = (pi/2/N) j
 * (signalProc.cpp:32-71) */
static void sp_dct10_post(double* re, double* im, int n)
{
    int idx = (n % 2 == 1) ? 0 : 1;
    for (int j = 0; j < n / 2 - idx; ++j) {
        re[j + n / 2 + 1] = re[n / 2 - j - idx];
        im[j + n / 2 + 1] = -im[n / 2 - j - idx];
    }
    for (int j = 0; j < n; ++j) {
        double theta = (REF_PI / 2. / n) * j;
        re[j] = 2. * (re[j] * cos(theta) + im[j] * sin(theta));
        im[j] = 0.0;
    }
}

/* V_0 = X_0/2, V_j = (1/2) e^{i th}(X_j - i X_{N-j}) for 1 <= j <= N/2, conjugate
 * upper half (signalProc.cpp:112-154) */
static void sp_dct01_pre(double* re, double* im, int n, double* t)
{
    double theta0 = REF_PI / 2. / n;
    for (int j = 0; j < n; ++j) t[j] = re[j];
    re[0] = 0.5 * cos(0.0) * t[0];
    im[0] = 0.0;
    for (int j = 1; j < n / 2 + 1; ++j) {
        double theta = theta0 * j;
        im[j] = 0.5 * (sin(theta) * t[j] - cos(theta) * t[n - j]);
        re[j] = 0.5 * (cos(theta) * t[j] + sin(theta) * t[n - j]);
    }
    for (int j = n / 2 + 1; j < n; ++j) {
        re[j] = re[n - j];
        im[j] = -im[n - j];
    }
}

/* x[2i] = Re v[i], x[2i+1] = Re v[N-1-i], imaginary part cleared
 * (signalProc.cpp:76-108) */
static void sp_dct01_post(double* re, double* im, int n, double* t)
{
    int upper = (n - 1) / 2 + 1;
    for (int i = 0; i < upper; ++i) t[2 * i] = re[i];
    for (int i = 0; i < n / 2; ++i) t[2 * i + 1] = re[n - i - 1];
    for (int i = 0; i < n; ++i) {
        re[i] = t[i];
        im[i] = 0.0;
    }
}

/* EXT: DCT-IV / DST-IV (FFTW REDFT11 / RODFT11 convention, factor 2):
 *   X_k = 2 sum_n x_n cos(pi (2n+1)(2k+1) / (4N)).
 * Even N: with a_m = x_{2m}, b_m = x_{N-1-2m},
 *   z_m = (a_m + i b_m) e^{-i pi m / N},  Z = DFT_{N/2}(z),
 *   w_p = e^{-i pi (4p+1) / (4N)} Z_p,   X_{2p} = 2 Re w_p,  X_{N-1-2p} = -2 Im w_p.
 * Odd N: the direct sum.  Both in long double.  'scale' is 2 for the forward
 * and 1 for the inverse, so the round trip is N like every other family.
 * DST-IV(x)_k = (-1)^k DCT-IV(reverse(x))_k. */
static void ext_dct4(const dft_plan* Ph, double* re, double* im, int n, int is_sine, long double scale)
{
    const long double pi = 3.141592653589793238462643383279502884L;
    long double* x = (long double*)malloc(sizeof(long double) * n * 2);
    long double* y = x + n;
    for (int j = 0; j < n; ++j) x[j] = is_sine ? re[n - 1 - j] : re[j];
    if (n % 2 == 0) {
        int h = n / 2;
        long double* zr = (long double*)malloc(sizeof(long double) * h * 4);
        long double* zi = zr + h;
        long double* Zr = zi + h;
        long double* Zi = Zr + h;
        for (int m = 0; m < h; ++m) {
            long double a = x[2 * m], b = x[n - 1 - 2 * m];
            long double t = -pi * (long double)m / (long double)n;
            zr[m] = a * cosl(t) - b * sinl(t);
            zi[m] = a * sinl(t) + b * cosl(t);
        }
        dft_rec(Ph, zr, zi, 1, h, Zr, Zi);
        for (int p = 0; p < h; ++p) {
            long double t = -pi * (long double)(4 * p + 1) / (4.0L * n);
            long double wr = Zr[p] * cosl(t) - Zi[p] * sinl(t);
            long double wi = Zr[p] * sinl(t) + Zi[p] * cosl(t);
            y[2 * p] = wr;
            y[n - 1 - 2 * p] = -wi;
        }
        free(zr);
    } else {
        for (int k = 0; k < n; ++k) {
            long double acc = 0.0L;
            for (int j = 0; j < n; ++j) {
                long long e = ((long long)(2 * j + 1) * (2 * k + 1)) % (8LL * n);
                acc += x[j] * cosl(pi * (long double)e / (4.0L * n));
            }
            y[k] = acc;
        }
    }
    for (int k = 0; k < n; ++k) {
        long double v = scale * y[k];
        if (is_sine && (k % 2 == 1)) v = -v;
        re[k] = (double)v;
        im[k] = 0.0;
    }
    free(x);
}

/* forward transform of one line according to the family (pittPack steps
 * pre(d) -> FFT -> post(d), src/pencilDcmp.cpp:5945-5966, 6034-6050) */
static void line_forward(int kind, const dft_plan* Pf, const dft_plan* Ph, double* re, double* im, int n, double* t)
{
    switch (kind) {
    case PPO_DCT2:
        sp_dct10_pre(re, im, n, t);
        dft_line(Pf, re, im);
        sp_dct10_post(re, im, n);
        break;
    case PPO_DST2:
        sp_swap(re, im, n, t);
        sp_dct10_pre(re, im, n, t);
        dft_line(Pf, re, im);
        sp_dct10_post(re, im, n);
        sp_swap(re, im, n, t);
        break;
    case PPO_FFT:
        dft_line(Pf, re, im);
        break;
    case PPO_DCT4:
        ext_dct4(Ph, re, im, n, 0, 2.0L);
        break;
    case PPO_DST4:
        ext_dct4(Ph, re, im, n, 1, 2.0L);
        break;
    }
}

/* inverse transform of one line (pre-rev -> IFFT -> post-rev,
 * src/pencilDcmp.cpp:6206-6215, 6285-6294) */
static void line_inverse(int kind, const dft_plan* Ph, const dft_plan* Pb, double* re, double* im, int n,
                         double* t)
{
    switch (kind) {
    case PPO_DCT2:
        sp_dct01_pre(re, im, n, t);
        dft_line(Pb, re, im);
        sp_dct01_post(re, im, n, t);
        break;
    case PPO_DST2:
        sp_swap(re, im, n, t);
        sp_dct01_pre(re, im, n, t);
        dft_line(Pb, re, im);
        sp_dct01_post(re, im, n, t);
        sp_swap(re, im, n, t);
        break;
    case PPO_FFT:
        dft_line(Pb, re, im);
        break;
    case PPO_DCT4:
        ext_dct4(Ph, re, im, n, 0, 1.0L);
        break;
    case PPO_DST4:
        ext_dct4(Ph, re, im, n, 1, 1.0L);
        break;
    }
}

/* ------------------------------------------------------------------------- */
/* eigenvalues (setEigenVal + getEigenVal)                                    */
/* ------------------------------------------------------------------------- */
/* num / denum / freq per family: DST (1,0,pi), DCT (0,0,pi), FFT (0,0,2pi);
 * EXT ND/DN (1/2, 0, pi). */
static void eig_params(int kind, double* num, double* den, double* freq)
{
    *den = 0.0;
    *freq = REF_PI;
    switch (kind) {
    case PPO_DST2: *num = 1.0; break;
    case PPO_DCT2: *num = 0.0; break;
    case PPO_FFT: *num = 0.0; *freq = 2. * REF_PI; break;
    default: *num = 0.5; break;
    }
}

/* lambda(i = ky, j = kx), src/pencilDcmp.cpp:4393-4417 (p0 = 1: no offsets) */
double ppo_eigenvalue(const ppo_problem* pb, int kx, int ky)
{
    int kindx = ppo_kind_from_bc(pb->bc[0], pb->bc[1]);
    int kindy = ppo_kind_from_bc(pb->bc[2], pb->bc[3]);
    double num0, den0, f0, num1, den1, f1;
    eig_params(kindx, &num0, &den0, &f0);
    eig_params(kindy, &num1, &den1, &f1);
    double dx = -(pb->box[0] - pb->box[1]) / (pb->nx);
    double dy = -(pb->box[2] - pb->box[3]) / (pb->ny);
    double dz = -(pb->box[4] - pb->box[5]) / (pb->nz);
    double Cx = (dz / dx) * (dz / dx);
    double Cy = (dz / dy) * (dz / dy);
    return (-2.0 + (-2.0 + 2. * cos((kx + num0) * f0 / (pb->nx + den0))) * Cx
            + (-2.0 + 2. * cos((ky + num1) * f1 / (pb->ny + den1))) * Cy);
}

/* ------------------------------------------------------------------------- */
/* tridiagonal solvers, src/triDiag.cpp (sub = {0,1,1}, sup = {1,1,0})         */
/* ------------------------------------------------------------------------- */
static const double SUB[3] = {0.0, 1.0, 1.0};
static const double SUP[3] = {1.0, 1.0, 0.0};

/* thomasLowMemNoBC, triDiag.cpp:1828-1886 */
static void thomas_nobc(double* g, double* rh, const double* b, int N)
{
    double bet;
    rh[0] = rh[0] / (bet = b[0]);
    int j = 1;
    g[j] = SUP[j - 1] / bet;
    bet = b[1] - SUB[1] * g[j];
    rh[1] = (rh[1] - SUB[1] * rh[j - 1]) / bet;
    for (j = 2; j < N - 1; ++j) {
        g[j] = SUP[1] / bet;
        bet = b[1] - SUB[1] * g[j];
        rh[j] = (rh[j] - SUB[1] * rh[j - 1]) / bet;
    }
    j = N - 1;
    g[j] = SUP[1] / bet;
    bet = b[2] - SUB[2] * g[j];
    rh[j] = (rh[j] - SUB[2] * rh[j - 1]) / bet;
    for (j = N - 2; j >= 0; --j) rh[j] -= g[j + 1] * rh[j + 1];
}

/* thomasLowMemNoBCV1, triDiag.cpp:1629-1687: row 0 decoupled from row 1 */
static void thomas_nobc_v1(double* g, double* rh, const double* b, int N)
{
    double bet;
    rh[0] = rh[0] / (bet = b[0]);
    int j = 1;
    g[j] = 0.0;
    bet = b[1] - SUB[1] * g[j];
    rh[1] = (rh[1] - SUB[1] * rh[j - 1]) / bet;
    for (j = 2; j < N - 1; ++j) {
        g[j] = SUP[1] / bet;
        bet = b[1] - SUB[1] * g[j];
        rh[j] = (rh[j] - SUB[1] * rh[j - 1]) / bet;
    }
    j = N - 1;
    g[j] = SUP[1] / bet;
    bet = b[2] - SUB[2] * g[j];
    rh[j] = (rh[j] - SUB[2] * rh[j - 1]) / bet;
    for (j = N - 2; j >= 0; --j) rh[j] -= g[j + 1] * rh[j + 1];
}

/* thomasLowMem, triDiag.cpp:1693-1822.  'pin' says whether the zero-mode row
 * replacement is applied when |diag + 2| < 1e-10 (always, in the reference). */
static void thomas_low_mem(double* g, double* rh, double diag, int N, char bc0, char bc1, int pin)
{
    double b[3] = {diag, diag, diag};
    if (bc0 == 'D') b[0] = b[1] - 1.;
    if (bc1 == 'D') b[2] = b[1] - 1.;
    if (bc0 == 'N') b[0] = b[1] + 1.;
    if (bc1 == 'N') b[2] = b[1] + 1.0;
    if (fabs(diag + 2.) < 1.e-10 && pin) {
        b[0] = 1.0;
        thomas_nobc_v1(g, rh, b, N);
        return;
    }
    thomas_nobc(g, rh, b, N);
}

/* shermanMorrisonThomasV1, triDiag.cpp:2112-2255 */
static void sherman_morrison_v1(double* g, double* rh, double* rh1, double diag, double alpha, double beta, int N)
{
    double b[3] = {1.0, diag, diag};
    double bb[3];
    double gamma = -b[0];
    bb[0] = b[0] - gamma;
    bb[1] = b[1];
    bb[2] = b[2] - alpha * beta / gamma;
    rh[0] = (rh[0] + rh[N - 1]) * 0.5;
    thomas_nobc_v1(g, rh, bb, N);
    rh1[0] = gamma;
    rh1[N - 1] = alpha;
    for (int i = 1; i < N - 1; ++i) rh1[i] = 0.0;
    thomas_nobc_v1(g, rh1, bb, N);
    double part1 = (rh[0] + beta * rh[N - 1] / gamma);
    double part2 = (1. + rh1[0] + beta * rh1[N - 1] / gamma);
    double fact = part1 / part2;
    for (int i = 0; i < N; ++i) rh[i] -= fact * rh1[i];
}

/* shermanMorrisonThomas, triDiag.cpp:1961-2108 */
static void sherman_morrison(double* g, double* rh, double* rh1, double diag, double alpha, double beta, int N)
{
    double b[3] = {diag, diag, diag};
    double bb[3];
    double gamma = -b[0];
    bb[0] = b[0] - gamma;
    bb[1] = b[1];
    bb[2] = b[2] - alpha * beta / gamma;
    if (fabs(diag + 2.) < 1.e-10) {
        sherman_morrison_v1(g, rh, rh1, diag, 1.0, 1.0, N);
        return;
    }
    thomas_nobc(g, rh, bb, N);
    rh1[0] = gamma;
    rh1[N - 1] = alpha;
    for (int i = 1; i < N - 1; ++i) rh1[i] = 0.0;
    thomas_nobc(g, rh1, bb, N);
    double part1 = (rh[0] + beta * rh[N - 1] / gamma);
    double part2 = (1. + rh1[0] + beta * rh1[N - 1] / gamma);
    double fact = part1 / part2;
    for (int i = 0; i < N; ++i) rh[i] -= fact * rh1[i];
}

/* ------------------------------------------------------------------------- */
/* manufactured solution pieces                                                */
/* ------------------------------------------------------------------------- */
/* exactValue, src/pencilDcmp.cpp:1837-1866 */
static double exact_value(double omega, double x, int tg)
{
    double ans = 0.0;
    if (fabs(omega) < 1.0e-6) return 1.0;
    if (tg == 0) ans = sin(omega * x);
    else if (tg == 1) ans = cos(omega * x);
    else if (tg == -1) ans = sin(omega * x);
    else if (tg == -2) ans = sin(omega * x);
    return ans;
}

/* ------------------------------------------------------------------------- */
/* validation                                                                  */
/* ------------------------------------------------------------------------- */
/* ------------------------------------------------------------------------- */
/* the reference's alternate z solvers as its CPU build computes them          */
/* ------------------------------------------------------------------------- */
/* myLog2 (src/mathFunction.cpp:36): log2 truncated to int */
static int ref_log2(int x) { return (int)(log2((double)x)); }

/* TriDiag::pcr (src/triDiag.cpp:1442-1542) is written for OpenACC, where each
 * vector lane keeps its own copy of the gathered a0..d2; compiled for the CPU
 * those are arrays of 20 entries indexed by i / VECLENGTH (256), so the first
 * loop leaves in entry b the neighbours of the LAST row of block b, and the
 * second loop updates every row of the block with them.  Defined (every read
 * in bounds, every entry within the 20) for Dirichlet or Neumann ends and
 * nz <= 256 not a power of two: one block, whose last row n - 1 always has
 * both i - s >= 0 and i + s >= n. */
int ppo_ref_pcr_defined(int nz, char z0, char z1)
{
    if ((z0 != 'D' && z0 != 'N') || (z1 != 'D' && z1 != 'N')) return 0;
    return nz >= 3 && nz <= 256 && (nz & (nz - 1)) != 0;
}

static void ref_pcr(int n, double* a, double* c, double* d)
{
    const int level = ref_log2(n) + 1;
    const int m = 256; /* VECLENGTH, src/include/params.h:56 */
    double a0[20], a1[20], a2[20], c0[20], c1[20], c2[20], d0[20], d1[20], d2[20];
    for (int p = 0; p < level; p++) {
        const int s = 1 << p;
        for (int i = 0; i < n; i++) {
            const int index = i / m;
            if (i - s < 0 && i + s < n) {
                a0[index] = a[i]; a1[index] = 0.0; a2[index] = a[i + s];
                c0[index] = c[i]; c1[index] = 0.0; c2[index] = c[i + s];
                d0[index] = d[i]; d1[index] = 0.0; d2[index] = d[i + s];
            } else if (i + s >= n && i - s >= 0) {
                a0[index] = a[i]; a1[index] = a[i - s]; a2[index] = 0.0;
                c0[index] = c[i]; c1[index] = c[i - s]; c2[index] = 0.0;
                d0[index] = d[i]; d1[index] = d[i - s]; d2[index] = 0.0;
            } else {
                a0[index] = a[i]; a1[index] = a[i - s]; a2[index] = a[i + s];
                c0[index] = c[i]; c1[index] = c[i - s]; c2[index] = c[i + s];
                d0[index] = d[i]; d1[index] = d[i - s]; d2[index] = d[i + s];
            }
        }
        for (int i = 0; i < n; i++) {
            const int index = i / m;
            const double r = 1. / (1. - a0[index] * c1[index] - c0[index] * a2[index]);
            a[i] = -r * a0[index] * a1[index];
            c[i] = -r * c0[index] * c2[index];
            d[i] = r * (d0[index] - a0[index] * d1[index] - c0[index] * d2[index]);
        }
    }
}

/* solvePCR (src/pencilDcmp.cpp:5239-5270): the system divided by eig
 * (fillInArrayContigNormalize :5320-5345, imposeBoundaryonContainer
 * :5372-5401, offDiagNormalize :5406-5452, imposeBoundaryonOffDiag
 * :5457-5481), then pcr; r in, solution out */
static void ref_solve_pcr(double* r, double eig, int nz, char z0, char z1, double* lower, double* upper)
{
    const double eigInv = 1. / eig;
    const double r0 = r[0], rn = r[nz - 1];
    for (int k = 1; k < nz - 1; k++) r[k] = r[k] * eigInv;
    if (z0 == 'D') r[0] = r0 / (eig - 1.);
    if (z1 == 'D') r[nz - 1] = rn / (eig - 1.);
    if (z0 == 'N') r[0] = r0 / (eig + 1.);
    if (z1 == 'N') r[nz - 1] = rn / (eig + 1.);
    for (int k = 1; k < nz; k++) lower[k] = eigInv;
    for (int k = 0; k < nz - 1; k++) upper[k] = eigInv;
    lower[0] = 0.0;
    upper[nz - 1] = 0.0;
    if (z0 == 'D') upper[0] = 1. / (eig - 1.);
    if (z1 == 'D') lower[nz - 1] = 1. / (eig - 1.);
    if (z0 == 'N') upper[0] = 1. / (eig + 1.);
    if (z1 == 'N') lower[nz - 1] = 1. / (eig + 1.);
    ref_pcr(nz, lower, upper, r);
}

/* TriDiag::crp (src/triDiag.cpp:1285-1437): cyclic reduction of the
 * constant-coefficient system (diagonal 1, off-diagonals 1/eig) down to a
 * 3 x 3 system, solved by the three-row Thomas (thomasLowMem
 * src/triDiag.cpp:1891-1950 with b = 1), and back-substitution.  Defined for
 * nz = 2^L - 1 with Dirichlet ends (the only ends solveCRP treats), L >= 2. */
int ppo_ref_crp_defined(int nz, char z0, char z1)
{
    if (z0 != 'D' || z1 != 'D') return 0;
    return nz >= 3 && nz <= 32767 && ((nz + 1) & nz) == 0;
}

static void ref_thomas3(const double* a, const double* b, const double* c, double* r)
{
    double gam[3], bet;
    r[0] = r[0] / (bet = b[0]);
    gam[1] = c[0] / bet;
    bet = b[1] - a[1] * gam[1];
    r[1] = (r[1] - a[1] * r[0]) / bet;
    gam[2] = c[1] / bet;
    bet = b[2] - a[2] * gam[2];
    r[2] = (r[2] - a[2] * r[1]) / bet;
    for (int j = 1; j >= 0; j--) r[j] -= gam[j + 1] * r[j + 1];
}

static void ref_crp(int n, double offdiag, double* rhs)
{
    const int level = ref_log2(n);
    double tmpA[16], tmpC[16];
    int m = n;
    tmpA[0] = offdiag;
    tmpC[0] = offdiag;
    for (int i = 0; i < level - 1; i++) {
        const int d1 = 1 << (i + 1);
        m = m >> 1;
        const double a0 = tmpA[i], c0 = tmpC[i];
        const double cte = 1. - (2. * a0 * c0);
        for (int j = 0; j < m; j++) {
            const int ind0 = d1 * j + (d1 - 1);
            const int im1 = d1 * j + (d1 - 1) - d1 / 2;
            const int ip1 = d1 * j + (d1 - 1) + d1 / 2;
            rhs[ind0] = (rhs[im1] * (-a0) + rhs[ind0] + rhs[ip1] * (-c0)) / cte;
        }
        tmpA[i + 1] = -a0 * a0 / cte;
        tmpC[i + 1] = -c0 * c0 / cte;
    }
    {
        const int d1 = 1 << level;
        const int ind0 = d1 - 1, im1 = (d1 - 1) - d1 / 2, ip1 = (d1 - 1) + d1 / 2;
        double t[3] = {rhs[im1], rhs[ind0], rhs[ip1]};
        const double A[3] = {0.0, tmpA[level - 1], tmpA[level - 1]};
        const double B[3] = {1.0, 1.0, 1.0};
        const double C[3] = {tmpC[level - 1], tmpC[level - 1], 0.0};
        ref_thomas3(A, B, C, t);
        rhs[ind0] = t[1];
        rhs[im1] = t[0];
        rhs[ip1] = t[2];
    }
    m = 3;
    for (int i = level - 1; i > 0; i--) {
        const int d0 = 1 << i;
        for (int j = 0; j < m; j++)
            rhs[d0 * j + (d0 - 1) - d0 / 2] = rhs[d0 * j + (d0 - 1) - d0 / 2] - tmpA[i - 1] * rhs[d0 * j + (d0 - 1)];
        for (int j = 0; j < m; j++)
            rhs[d0 * j + (d0 - 1) + d0 / 2] = rhs[d0 * j + (d0 - 1) + d0 / 2] - tmpC[i - 1] * rhs[d0 * j + (d0 - 1)];
        m = (1 << (level - i + 2)) - 1;
    }
}

/* solveCRP (src/pencilDcmp.cpp:5275-5315): interior rows times 1/eig
 * (fillInArrayContigNormalize), the Dirichlet end rows divided by eig
 * (imposeBoundaryonCRPTmp :5350-5369), then crp with off-diagonal 1/eig */
static void ref_solve_crp(double* r, double eig, int nz)
{
    const double eigInv = 1. / eig;
    const double r0 = r[0], rn = r[nz - 1];
    for (int k = 1; k < nz - 1; k++) r[k] = r[k] * eigInv;
    r[0] = r0 / (eig);
    r[nz - 1] = rn / (eig);
    ref_crp(nz, 1. / eig, r);
}

int ppo_check(const ppo_problem* pb)
{
    if (pb->nx < 2 || pb->ny < 2 || pb->nz < 3) return PPO_ERR_INPUT;
    int kx = ppo_kind_from_bc(pb->bc[0], pb->bc[1]);
    int ky = ppo_kind_from_bc(pb->bc[2], pb->bc[3]);
    if (kx == PPO_BAD || ky == PPO_BAD) return PPO_ERR_INPUT;
    char z0 = pb->bc[4], z1 = pb->bc[5];
    if (z0 == 'P' || z1 == 'P') {
        if (z0 != 'P' || z1 != 'P') return PPO_ERR_INPUT;
    } else if ((z0 != 'D' && z0 != 'N') || (z1 != 'D' && z1 != 'N')) {
        return PPO_ERR_INPUT;
    }
    for (int d = 0; d < 3; ++d)
        if (!(pb->box[2 * d + 1] > pb->box[2 * d])) return PPO_ERR_INPUT;
    if (pb->z_method == 1 && !ppo_ref_pcr_defined(pb->nz, z0, z1)) return PPO_ERR_INPUT;
    if (pb->z_method == 2 && !ppo_ref_crp_defined(pb->nz, z0, z1)) return PPO_ERR_INPUT;
    if (pb->z_method < 0 || pb->z_method > 2) return PPO_ERR_INPUT;
    return 0;
}

/* ------------------------------------------------------------------------- */
/* the solve                                                                   */
/* ------------------------------------------------------------------------- */
/* modifyRhsDirichlet, src/pencilDcmp.cpp:4623-4835, on the real part of P */
static void modify_rhs_dirichlet(const ppo_problem* pb, double* P)
{
    int nx = pb->nx, ny = pb->ny, nz = pb->nz;
    double pi = 4. * atan(1.0);
    double Xa = pb->box[0], Ya = pb->box[2], Za = pb->box[4];
    double c1 = -(pb->box[0] - pb->box[1]) / (nx);
    double c2 = -(pb->box[2] - pb->box[3]) / (ny);
    double c3 = -(pb->box[4] - pb->box[5]) / (nz);
    double shift = 1.0;
    double omega[3] = {1 * pi, 2 * pi, 3 * pi};
    int t0 = ref_tag_xy(ppo_kind_from_bc(pb->bc[0], pb->bc[1]));
    int t1 = ref_tag_xy(ppo_kind_from_bc(pb->bc[2], pb->bc[3]));
    int t2 = ref_tag_z(pb->bc);
    double x, y, z;
#define PRE(i, j, k) P[2 * ((long)(i) + (long)nx * (j) + (long)nx * ny * (k))]
    if (pb->bc[4] == 'D' && !pb->face[4]) {
        z = Za;
        int k = 0;
        for (int i = 0; i < nx; ++i) {
            x = Xa + i * c1 + shift * c1 * .5;
            for (int j = 0; j < ny; ++j) {
                y = Ya + j * c2 + shift * c2 * 0.5;
                PRE(i, j, k) = PRE(i, j, k)
                               - 2. * exact_value(omega[0], x, t0) * exact_value(omega[1], y, t1)
                                     * exact_value(omega[2], z, t2);
            }
        }
    }
    if (pb->bc[5] == 'D' && !pb->face[5]) {
        z = Za + (nz - 1) * c3 + c3;
        int k = nz - 1;
        for (int i = 0; i < nx; ++i) {
            x = Xa + i * c1 + shift * c1 * .5;
            for (int j = 0; j < ny; ++j) {
                y = Ya + j * c2 + shift * c2 * 0.5;
                PRE(i, j, k) = PRE(i, j, k)
                               - 2 * exact_value(omega[0], x, t0) * exact_value(omega[1], y, t1)
                                     * exact_value(omega[2], z, t2);
            }
        }
    }
    if (pb->bc[0] == 'D' && !pb->face[0]) {
        x = Xa;
        int i = 0;
        for (int k = 0; k < nz; ++k) {
            z = Za + k * c3 + shift * c3 * .5;
            for (int j = 0; j < ny; ++j) {
                y = Ya + j * c2 + shift * c2 * 0.5;
                PRE(i, j, k) = PRE(i, j, k)
                               - 2. * exact_value(omega[0], x, t0) * exact_value(omega[1], y, t1)
                                     * exact_value(omega[2], z, t2);
            }
        }
    }
    if (pb->bc[1] == 'D' && !pb->face[1]) {
        int i = nx - 1;
        x = Xa + (i + 1) * c1;
        for (int k = 0; k < nz; ++k) {
            z = Za + k * c3 + shift * c3 * .5;
            for (int j = 0; j < ny; ++j) {
                y = Ya + j * c2 + shift * c2 * 0.5;
                PRE(i, j, k) = PRE(i, j, k)
                               - 2. * exact_value(omega[0], x, t0) * exact_value(omega[1], y, t1)
                                     * exact_value(omega[2], z, t2);
            }
        }
    }
    if (pb->bc[2] == 'D' && !pb->face[2]) {
        y = Ya;
        int j = 0;
        for (int k = 0; k < nz; ++k) {
            z = Za + k * c3 + shift * c3 * .5;
            for (int i = 0; i < nx; ++i) {
                x = Xa + i * c1 + shift * c1 * 0.5;
                PRE(i, j, k) = PRE(i, j, k)
                               - 2. * exact_value(omega[0], x, t0) * exact_value(omega[1], y, t1)
                                     * exact_value(omega[2], z, t2);
            }
        }
    }
    if (pb->bc[3] == 'D' && !pb->face[3]) {
        int j = ny - 1;
        y = Ya + (j + 1) * c2;
        for (int k = 0; k < nz; ++k) {
            z = Za + k * c3 + shift * c3 * .5;
            for (int i = 0; i < nx; ++i) {
                x = Xa + i * c1 + shift * c1 * 0.5;
                PRE(i, j, k) = PRE(i, j, k)
                               - 2. * exact_value(omega[0], x, t0) * exact_value(omega[1], y, t1)
                                     * exact_value(omega[2], z, t2);
            }
        }
    }
#undef PRE
}

/* the caller's boundary data (ppo_problem.face): the right-hand-side share of
 * each face's ghost cells, subtracted from the dz^2-scaled RHS on the first
 * cell layer */
static void user_faces(const ppo_problem* pb, double* P)
{
    int nx = pb->nx, ny = pb->ny, nz = pb->nz;
    double h[3] = {-(pb->box[0] - pb->box[1]) / nx, -(pb->box[2] - pb->box[3]) / ny,
                   -(pb->box[4] - pb->box[5]) / nz};
    double w[3] = {(h[2] / h[0]) * (h[2] / h[0]), (h[2] / h[1]) * (h[2] / h[1]), 1.0};
#define PRE(i, j, k) P[2 * ((long)(i) + (long)nx * (j) + (long)nx * ny * (k))]
    for (int f = 0; f < 6; ++f) {
        const double* g = pb->face[f];
        if (!g || pb->bc[f] == 'P') continue;
        int d = f / 2;
        double c = pb->bc[f] == 'D' ? 2.0 * w[d] : w[d] * h[d];
        if (d == 0) {
            int i = (f & 1) ? nx - 1 : 0;
            for (int k = 0; k < nz; ++k)
                for (int j = 0; j < ny; ++j) PRE(i, j, k) -= c * g[j + (long)ny * k];
        } else if (d == 1) {
            int j = (f & 1) ? ny - 1 : 0;
            for (int k = 0; k < nz; ++k)
                for (int i = 0; i < nx; ++i) PRE(i, j, k) -= c * g[i + (long)nx * k];
        } else {
            int k = (f & 1) ? nz - 1 : 0;
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < nx; ++i) PRE(i, j, k) -= c * g[i + (long)nx * j];
        }
    }
#undef PRE
}

/* public: the Dirichlet lift as a standalone correction (what modifyRhsDirichlet
 * subtracts from the scaled RHS), written into an n-sized real array */
void ppo_dirichlet_lift(const ppo_problem* pb, double* lift)
{
    long n = (long)pb->nx * pb->ny * pb->nz;
    double* P = (double*)calloc(2 * n, sizeof(double));
    modify_rhs_dirichlet(pb, P);
    for (long p = 0; p < n; ++p) lift[p] = -P[2 * p];
    free(P);
}

int ppo_solve(const ppo_problem* pb, const double* rhs_re, const double* rhs_im, double* P)
{
    int err = ppo_check(pb);
    if (err) return err;
    int nx = pb->nx, ny = pb->ny, nz = pb->nz;
    long n = (long)nx * ny * nz;
    int kindx = ppo_kind_from_bc(pb->bc[0], pb->bc[1]);
    int kindy = ppo_kind_from_bc(pb->bc[2], pb->bc[3]);
    double c3 = -(pb->box[4] - pb->box[5]) / (nz);

    /* assignRhs: P.re = f dz dz, P.im = 0 (the complex variant also scales im) */
    for (long p = 0; p < n; ++p) {
        P[2 * p] = rhs_re[p] * c3 * c3;
        P[2 * p + 1] = rhs_im ? rhs_im[p] * c3 * c3 : 0.0;
    }
    if (pb->dirichlet_lift) modify_rhs_dirichlet(pb, P);
    user_faces(pb, P);

    int nmax = nx > ny ? nx : ny;
    if (nz > nmax) nmax = nz;
    double* re = (double*)malloc(sizeof(double) * nmax);
    double* im = (double*)malloc(sizeof(double) * nmax);
    double* t = (double*)malloc(sizeof(double) * nmax);
    dft_plan fx, bx, fy, by, hx, hy;
    dft_plan_init(&fx, nx, -1);
    dft_plan_init(&bx, nx, +1);
    dft_plan_init(&fy, ny, -1);
    dft_plan_init(&by, ny, +1);
    dft_plan_init(&hx, nx / 2 > 0 ? nx / 2 : 1, -1); /* half-length plans for DCT-IV */
    dft_plan_init(&hy, ny / 2 > 0 ? ny / 2 : 1, -1);

#define AT(i, j, k, c) P[2 * ((long)(i) + (long)nx * (j) + (long)nx * ny * (k)) + (c)]
    /* x forward */
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j) {
            for (int i = 0; i < nx; ++i) { re[i] = AT(i, j, k, 0); im[i] = AT(i, j, k, 1); }
            line_forward(kindx, &fx, &hx, re, im, nx, t);
            for (int i = 0; i < nx; ++i) { AT(i, j, k, 0) = re[i]; AT(i, j, k, 1) = im[i]; }
        }
    /* y forward (the reference first transposes each z-plane; the arithmetic
     * per y-line is the same) */
    for (int k = 0; k < nz; ++k)
        for (int i = 0; i < nx; ++i) {
            for (int j = 0; j < ny; ++j) { re[j] = AT(i, j, k, 0); im[j] = AT(i, j, k, 1); }
            line_forward(kindy, &fy, &hy, re, im, ny, t);
            for (int j = 0; j < ny; ++j) { AT(i, j, k, 0) = re[j]; AT(i, j, k, 1) = im[j]; }
        }
    /* z solve: real part always, imaginary part when x or y is periodic */
    {
        double* g = (double*)malloc(sizeof(double) * nz);
        double* r = (double*)malloc(sizeof(double) * nz);
        double* r1 = (double*)malloc(sizeof(double) * nz);
        int nidx = (pb->bc[0] == 'P' || pb->bc[2] == 'P') ? 2 : 1;
        int has_d = (pb->bc[4] == 'D' || pb->bc[5] == 'D');
        int pin = pb->compat_zero_mode ? 1 : !has_d;
        for (int jx = 0; jx < nx; ++jx)
            for (int iy = 0; iy < ny; ++iy) {
                double eig = ppo_eigenvalue(pb, jx, iy);
                for (int c = 0; c < nidx; ++c) {
                    for (int k = 0; k < nz; ++k) r[k] = AT(jx, iy, k, c);
                    if (pb->z_method == 1)
                        ref_solve_pcr(r, eig, nz, pb->bc[4], pb->bc[5], g, r1);
                    else if (pb->z_method == 2)
                        ref_solve_crp(r, eig, nz);
                    else if (pb->bc[4] != 'P')
                        thomas_low_mem(g, r, eig, nz, pb->bc[4], pb->bc[5], pin);
                    else
                        sherman_morrison(g, r, r1, eig, 1.0, 1.0, nz);
                    for (int k = 0; k < nz; ++k) AT(jx, iy, k, c) = r[k];
                }
            }
        free(g); free(r); free(r1);
    }
    /* y inverse */
    for (int k = 0; k < nz; ++k)
        for (int i = 0; i < nx; ++i) {
            for (int j = 0; j < ny; ++j) { re[j] = AT(i, j, k, 0); im[j] = AT(i, j, k, 1); }
            line_inverse(kindy, &hy, &by, re, im, ny, t);
            for (int j = 0; j < ny; ++j) { AT(i, j, k, 0) = re[j]; AT(i, j, k, 1) = im[j]; }
        }
    /* x inverse */
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j) {
            for (int i = 0; i < nx; ++i) { re[i] = AT(i, j, k, 0); im[i] = AT(i, j, k, 1); }
            line_inverse(kindx, &hx, &bx, re, im, nx, t);
            for (int i = 0; i < nx; ++i) { AT(i, j, k, 0) = re[i]; AT(i, j, k, 1) = im[i]; }
        }
#undef AT
    /* rescale by 1/(nx ny) */
    double scale = (double)nx * (double)ny;
    for (long p = 0; p < 2 * n; ++p) P[p] = 1. / (scale)*P[p];

    dft_plan_free(&fx);
    dft_plan_free(&bx);
    dft_plan_free(&fy);
    dft_plan_free(&by);
    dft_plan_free(&hx);
    dft_plan_free(&hy);
    free(re); free(im); free(t);
    if (pb->zero_mean) {
        /* subtractMeanValue (src/pencilDcmp.cpp:5649-5683) */
        long double sum = 0.0L;
        for (long p = 0; p < n; ++p) sum += P[2 * p];
        double mean = (double)(sum / n);
        for (long p = 0; p < n; ++p) P[2 * p] -= mean;
    }
    return 0;
}

/* ------------------------------------------------------------------------- */
/* manufactured solution (initializeTrigonometric / getError)                  */
/* ------------------------------------------------------------------------- */
/* f (unscaled: the solve multiplies by dz^2 as assignRhs does) and the
 * analytic u.  src/pencilDcmp.cpp:1871-2034 (RHS) and 2040-2208 (exact). */
void ppo_manufactured(const ppo_problem* pb, double* f_re, double* f_im, double* u_re, double* u_im)
{
    int nx = pb->nx, ny = pb->ny, nz = pb->nz;
    double pi = 4. * atan(1.0);
    double Xa = pb->box[0], Ya = pb->box[2], Za = pb->box[4];
    double c1 = -(pb->box[0] - pb->box[1]) / (nx);
    double c2 = -(pb->box[2] - pb->box[3]) / (ny);
    double c3 = -(pb->box[4] - pb->box[5]) / (nz);
    double omega[3] = {1 * pi, 2 * pi, 3 * pi};
    int t0 = ref_tag_xy(ppo_kind_from_bc(pb->bc[0], pb->bc[1]));
    int t1 = ref_tag_xy(ppo_kind_from_bc(pb->bc[2], pb->bc[3]));
    int t2 = ref_tag_z(pb->bc);
    int periodic_xy = (pb->bc[0] == 'P' || pb->bc[2] == 'P');
    int periodic_all = (pb->bc[0] == 'P' && pb->bc[2] == 'P' && pb->bc[4] == 'P');
    for (int k = 0; k < nz; ++k) {
        double z = Za + k * c3 + 1.0 * c3 * 0.5;
        for (int j = 0; j < ny; ++j) {
            double y = Ya + j * c2 + 1.0 * c2 * 0.5;
            for (int i = 0; i < nx; ++i) {
                double x = Xa + i * c1 + 1.0 * c1 * .5;
                long p = (long)i + (long)nx * j + (long)nx * ny * k;
                double fr, fi, ur, ui;
                if (periodic_all) {
                    fr = -3. * omega[1] * omega[1] * (cos(omega[1] * (x + y + z)));
                    fi = -3. * omega[1] * omega[1] * (sin(omega[1] * (x + y + z)));
                    ur = cos(omega[1] * (x + y + z));
                    ui = sin(omega[1] * (x + y + z));
                } else if (periodic_xy) {
                    fr = -3. * omega[1] * omega[1] * (sin(omega[1] * z) * cos(omega[1] * (x + y)));
                    fi = -3. * omega[1] * omega[1] * (sin(omega[1] * z) * sin(omega[1] * (x + y)));
                    ur = sin(omega[1] * z) * cos(omega[1] * (x + y));
                    ui = sin(omega[1] * z) * sin(omega[1] * (x + y));
                } else {
                    double e = exact_value(omega[0], x, t0) * exact_value(omega[1], y, t1)
                               * exact_value(omega[2], z, t2);
                    fr = -((omega[0] * omega[0]) * exact_value(omega[0], x, t0) * exact_value(omega[1], y, t1)
                               * exact_value(omega[2], z, t2)
                           + (omega[1] * omega[1]) * exact_value(omega[0], x, t0) * exact_value(omega[1], y, t1)
                                 * exact_value(omega[2], z, t2)
                           + (omega[2] * omega[2]) * exact_value(omega[0], x, t0) * exact_value(omega[1], y, t1)
                                 * exact_value(omega[2], z, t2));
                    fi = 0.0;
                    ur = e;
                    ui = 0.0;
                }
                if (f_re) f_re[p] = fr;
                if (f_im) f_im[p] = fi;
                if (u_re) u_re[p] = ur;
                if (u_im) u_im[p] = ui;
            }
        }
    }
}

/* ------------------------------------------------------------------------- */
/* math oracle: 7-point residual of the exact (non-compat) discrete problem   */
/* ------------------------------------------------------------------------- */
/* r = b - A u in the dz^2-scaled system, with ghost cells D: -u, N: +u,
 * P: wrap (the operator whose eigen-decomposition the transforms realise).
 * u and b are n-sized real arrays; long double accumulation. */
void ppo_residual(const ppo_problem* pb, const double* u, const double* b, double* r)
{
    int nx = pb->nx, ny = pb->ny, nz = pb->nz;
    double dx = -(pb->box[0] - pb->box[1]) / (nx);
    double dy = -(pb->box[2] - pb->box[3]) / (ny);
    double dz = -(pb->box[4] - pb->box[5]) / (nz);
    long double Cx = ((long double)dz / dx) * ((long double)dz / dx);
    long double Cy = ((long double)dz / dy) * ((long double)dz / dy);
#define U(i, j, k) ((long double)u[(long)(i) + (long)nx * (j) + (long)nx * ny * (k)])
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                long double c = U(i, j, k);
                long double nb[6];
                /* x */
                if (i > 0) nb[0] = U(i - 1, j, k);
                else nb[0] = pb->bc[0] == 'P' ? U(nx - 1, j, k) : (pb->bc[0] == 'N' ? c : -c);
                if (i < nx - 1) nb[1] = U(i + 1, j, k);
                else nb[1] = pb->bc[1] == 'P' ? U(0, j, k) : (pb->bc[1] == 'N' ? c : -c);
                if (j > 0) nb[2] = U(i, j - 1, k);
                else nb[2] = pb->bc[2] == 'P' ? U(i, ny - 1, k) : (pb->bc[2] == 'N' ? c : -c);
                if (j < ny - 1) nb[3] = U(i, j + 1, k);
                else nb[3] = pb->bc[3] == 'P' ? U(i, 0, k) : (pb->bc[3] == 'N' ? c : -c);
                if (k > 0) nb[4] = U(i, j, k - 1);
                else nb[4] = pb->bc[4] == 'P' ? U(i, j, nz - 1) : (pb->bc[4] == 'N' ? c : -c);
                if (k < nz - 1) nb[5] = U(i, j, k + 1);
                else nb[5] = pb->bc[5] == 'P' ? U(i, j, 0) : (pb->bc[5] == 'N' ? c : -c);
                long double au = Cx * (nb[0] - 2 * c + nb[1]) + Cy * (nb[2] - 2 * c + nb[3]) + (nb[4] - 2 * c + nb[5]);
                long p = (long)i + (long)nx * j + (long)nx * ny * k;
                r[p] = (double)((long double)b[p] - au);
            }
#undef U
}
