// Batched mixed-radix (2,3,4,5,8) Stockham FFT on lines held in shared memory.
//
// The reference hands every line to FFTW or cuFFT (src/poissonCPU.cpp:40-234,
// src/poissonGPU.cpp:5-97: unnormalised, exp(-2 pi i jk/N) forward and
// exp(+2 pi i jk/N) backward).  Here the lines of one CTA tile sit in shared
// memory, line-major (line l, element e at buf[l * N + e]), and are
// transformed in place by log_r(N) Stockham passes that ping-pong between two
// buffers.  Pass p with radix r and span Ns (product of the earlier radices):
// butterfly j of a line reads r inputs at j + q N/r, multiplies input q by
// W_N^{q (j mod Ns) N/(Ns r)}, takes an r-point DFT and writes output q to
// (j / Ns) Ns r + (j mod Ns) + q Ns.  The output ends in natural order.
#pragma once

#include "pp_common.cuh"

#define PP_FFT_MAXPASS 16

struct PPFftPlan {
    int n;                       // line length
    int npass;                   // number of passes
    int radix[PP_FFT_MAXPASS];   // radix of every pass, product = n
    const double2* tw;           // W_n^m = exp(-2 pi i m / n), m < n
};

// r-point DFT in registers; SIGN = -1 forward, +1 backward
template <int SIGN>
PP_D void dft2(double2* v)
{
    double2 a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
}

template <int SIGN>
PP_D void dft3(double2* v)
{
    const double h = 0.86602540378443864676372317075293618;  // sin(2 pi / 3)
    double2 t1 = cadd(v[1], v[2]);
    double2 t2 = csub(v[1], v[2]);
    double2 m = make_double2(v[0].x - 0.5 * t1.x, v[0].y - 0.5 * t1.y);
    double2 r = cmul_i(cscale(t2, h), (double)SIGN);
    v[0] = cadd(v[0], t1);
    v[1] = cadd(m, r);
    v[2] = csub(m, r);
}

template <int SIGN>
PP_D void dft4(double2* v)
{
    double2 a = cadd(v[0], v[2]);
    double2 b = csub(v[0], v[2]);
    double2 c = cadd(v[1], v[3]);
    double2 d = cmul_i(csub(v[1], v[3]), (double)SIGN);
    v[0] = cadd(a, c);
    v[2] = csub(a, c);
    v[1] = cadd(b, d);
    v[3] = csub(b, d);
}

template <int SIGN>
PP_D void dft5(double2* v)
{
    const double c1 = 0.30901699437494742410229341718281906;   // cos(2 pi / 5)
    const double c2 = -0.80901699437494742410229341718281906;  // cos(4 pi / 5)
    const double s1 = 0.95105651629515357211643933337938214;   // sin(2 pi / 5)
    const double s2 = 0.58778525229247312916870595463907277;   // sin(4 pi / 5)
    double2 t1 = cadd(v[1], v[4]);
    double2 t2 = cadd(v[2], v[3]);
    double2 t3 = csub(v[1], v[4]);
    double2 t4 = csub(v[2], v[3]);
    double2 a1 = make_double2(v[0].x + c1 * t1.x + c2 * t2.x, v[0].y + c1 * t1.y + c2 * t2.y);
    double2 a2 = make_double2(v[0].x + c2 * t1.x + c1 * t2.x, v[0].y + c2 * t1.y + c1 * t2.y);
    double2 b1 = cmul_i(make_double2(s1 * t3.x + s2 * t4.x, s1 * t3.y + s2 * t4.y), (double)SIGN);
    double2 b2 = cmul_i(make_double2(s2 * t3.x - s1 * t4.x, s2 * t3.y - s1 * t4.y), (double)SIGN);
    v[0] = cadd(v[0], cadd(t1, t2));
    v[1] = cadd(a1, b1);
    v[4] = csub(a1, b1);
    v[2] = cadd(a2, b2);
    v[3] = csub(a2, b2);
}

template <int SIGN>
PP_D void dft8(double2* v)
{
    const double h = 0.70710678118654752440084436210484904;  // sqrt(2) / 2
    double2 e[4] = {v[0], v[2], v[4], v[6]};
    double2 o[4] = {v[1], v[3], v[5], v[7]};
    dft4<SIGN>(e);
    dft4<SIGN>(o);
    // o[k] *= exp(SIGN 2 pi i k / 8)
    double2 o1 = make_double2(h * (o[1].x - SIGN * o[1].y), h * (o[1].y + SIGN * o[1].x));
    double2 o2 = cmul_i(o[2], (double)SIGN);
    double2 o3 = make_double2(h * (-o[3].x - SIGN * o[3].y), h * (-o[3].y + SIGN * o[3].x));
    v[0] = cadd(e[0], o[0]);
    v[4] = csub(e[0], o[0]);
    v[1] = cadd(e[1], o1);
    v[5] = csub(e[1], o1);
    v[2] = cadd(e[2], o2);
    v[6] = csub(e[2], o2);
    v[3] = cadd(e[3], o3);
    v[7] = csub(e[3], o3);
}

template <int R, int SIGN>
PP_D void stockham_pass(const double2* __restrict__ src, double2* __restrict__ dst, int n, int nlines, int ns,
                        const double2* __restrict__ tw, int tid, int nthreads)
{
    const int nb = n / R;         // butterflies per line
    const int tstride = n / (ns * R);
    const int total = nb * nlines;
    for (int t = tid; t < total; t += nthreads) {
        const int l = t / nb;
        const int j = t - l * nb;
        const int k = j % ns;
        const double2* in = src + l * n;
        double2* out = dst + l * n;
        double2 v[R];
#pragma unroll
        for (int q = 0; q < R; ++q) v[q] = in[j + q * nb];
        if (ns > 1) {
#pragma unroll
            for (int q = 1; q < R; ++q) {
                double2 w = __ldg(&tw[q * k * tstride]);
                if (SIGN > 0) w.y = -w.y;
                v[q] = cmul(v[q], w);
            }
        }
        if (R == 2) dft2<SIGN>(v);
        if (R == 3) dft3<SIGN>(v);
        if (R == 4) dft4<SIGN>(v);
        if (R == 5) dft5<SIGN>(v);
        if (R == 8) dft8<SIGN>(v);
        const int base = (j / ns) * ns * R + k;
#pragma unroll
        for (int q = 0; q < R; ++q) out[base + q * ns] = v[q];
    }
}

// Transform nlines lines of plan.n points held in a (line-major); b is scratch
// of the same size.  Returns the buffer that holds the result.  Ends with a
// __syncthreads(); must be entered by every thread of the block after the
// data in 'a' is complete (the caller synchronises before the call).
template <int SIGN>
__device__ double2* fft_lines(double2* a, double2* b, int nlines, const PPFftPlan& P, int tid, int nthreads)
{
    double2* src = a;
    double2* dst = b;
    int ns = 1;
    for (int p = 0; p < P.npass; ++p) {
        const int r = P.radix[p];
        switch (r) {
        case 2: stockham_pass<2, SIGN>(src, dst, P.n, nlines, ns, P.tw, tid, nthreads); break;
        case 3: stockham_pass<3, SIGN>(src, dst, P.n, nlines, ns, P.tw, tid, nthreads); break;
        case 4: stockham_pass<4, SIGN>(src, dst, P.n, nlines, ns, P.tw, tid, nthreads); break;
        case 5: stockham_pass<5, SIGN>(src, dst, P.n, nlines, ns, P.tw, tid, nthreads); break;
        default: stockham_pass<8, SIGN>(src, dst, P.n, nlines, ns, P.tw, tid, nthreads); break;
        }
        __syncthreads();
        double2* t = src;
        src = dst;
        dst = t;
        ns *= r;
    }
    return src;
}
