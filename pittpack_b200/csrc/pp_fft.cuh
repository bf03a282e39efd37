// Batched mixed-radix Stockham FFT on lines held in shared memory, in FP64
// (double2) or FP32 (float2): register butterflies of radix 2, 3, 4, 5, 7
// and 8, and one pass per remaining prime factor p, whose p-point DFTs are
// summed directly (p^2 multiplies, twiddles from the line's own table), so
// that every line length has a plan.
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

// the passes of a length: radix 8 while 8 divides, then 4, 2, 3, 5, 7, then
// the remaining prime factors in increasing order; false if n < 1
PP_HD bool pp_fft_plan(int n, PPFftPlan* P)
{
    int m = n, k = 0;
    if (n < 1) return false;
    const int small[6] = {8, 4, 2, 3, 5, 7};
    for (int q = 0; q < 6; ++q)
        while (m % small[q] == 0 && k < PP_FFT_MAXPASS) {
            P->radix[k++] = small[q];
            m /= small[q];
        }
    for (int p = 11; p * p <= m && k < PP_FFT_MAXPASS; p += 2)
        while (m % p == 0 && k < PP_FFT_MAXPASS) {
            P->radix[k++] = p;
            m /= p;
        }
    if (m > 1 && k < PP_FFT_MAXPASS) {
        P->radix[k++] = m;
        m = 1;
    }
    P->n = n;
    P->npass = k;
    return m == 1;
}

// r-point DFTs in registers; SIGN = -1 forward, +1 backward
template <int SIGN, typename C>
PP_D void dft2(C* v)
{
    C a = v[0], b = v[1];
    v[0] = c_add(a, b);
    v[1] = c_sub(a, b);
}

template <int SIGN, typename C>
PP_D void dft3(C* v)
{
    using R = typename CReal<C>::type;
    const R h = (R)0.86602540378443864676372317075293618;  // sin(2 pi / 3)
    C t1 = c_add(v[1], v[2]);
    C t2 = c_sub(v[1], v[2]);
    C m = mkc<C>(v[0].x - (R)0.5 * t1.x, v[0].y - (R)0.5 * t1.y);
    C r = c_mul_si<SIGN>(c_scale(t2, h));
    v[0] = c_add(v[0], t1);
    v[1] = c_add(m, r);
    v[2] = c_sub(m, r);
}

template <int SIGN, typename C>
PP_D void dft4(C* v)
{
    C a = c_add(v[0], v[2]);
    C b = c_sub(v[0], v[2]);
    C c = c_add(v[1], v[3]);
    C d = c_mul_si<SIGN>(c_sub(v[1], v[3]));
    v[0] = c_add(a, c);
    v[2] = c_sub(a, c);
    v[1] = c_add(b, d);
    v[3] = c_sub(b, d);
}

template <int SIGN, typename C>
PP_D void dft5(C* v)
{
    using R = typename CReal<C>::type;
    const R c1 = (R)0.30901699437494742410229341718281906;   // cos(2 pi / 5)
    const R c2 = (R)-0.80901699437494742410229341718281906;  // cos(4 pi / 5)
    const R s1 = (R)0.95105651629515357211643933337938214;   // sin(2 pi / 5)
    const R s2 = (R)0.58778525229247312916870595463907277;   // sin(4 pi / 5)
    C t1 = c_add(v[1], v[4]);
    C t2 = c_add(v[2], v[3]);
    C t3 = c_sub(v[1], v[4]);
    C t4 = c_sub(v[2], v[3]);
    C a1 = mkc<C>(v[0].x + c1 * t1.x + c2 * t2.x, v[0].y + c1 * t1.y + c2 * t2.y);
    C a2 = mkc<C>(v[0].x + c2 * t1.x + c1 * t2.x, v[0].y + c2 * t1.y + c1 * t2.y);
    C b1 = c_mul_si<SIGN>(mkc<C>(s1 * t3.x + s2 * t4.x, s1 * t3.y + s2 * t4.y));
    C b2 = c_mul_si<SIGN>(mkc<C>(s2 * t3.x - s1 * t4.x, s2 * t3.y - s1 * t4.y));
    v[0] = c_add(v[0], c_add(t1, t2));
    v[1] = c_add(a1, b1);
    v[4] = c_sub(a1, b1);
    v[2] = c_add(a2, b2);
    v[3] = c_sub(a2, b2);
}

template <int SIGN, typename C>
PP_D void dft8(C* v)
{
    using R = typename CReal<C>::type;
    const R h = (R)0.70710678118654752440084436210484904;  // sqrt(2) / 2
    C e[4] = {v[0], v[2], v[4], v[6]};
    C o[4] = {v[1], v[3], v[5], v[7]};
    dft4<SIGN>(e);
    dft4<SIGN>(o);
    // o[k] *= exp(SIGN 2 pi i k / 8)
    const R s = (R)SIGN;
    C o1 = mkc<C>(h * (o[1].x - s * o[1].y), h * (o[1].y + s * o[1].x));
    C o2 = c_mul_si<SIGN>(o[2]);
    C o3 = mkc<C>(h * (-o[3].x - s * o[3].y), h * (-o[3].y + s * o[3].x));
    v[0] = c_add(e[0], o[0]);
    v[4] = c_sub(e[0], o[0]);
    v[1] = c_add(e[1], o1);
    v[5] = c_sub(e[1], o1);
    v[2] = c_add(e[2], o2);
    v[6] = c_sub(e[2], o2);
    v[3] = c_add(e[3], o3);
    v[7] = c_sub(e[3], o3);
}

// R-point DFT in registers by direct summation, W_R^m = tw[m * rstride]
// (the line's own table, W_n^{n/R} = W_R)
template <int R, int SIGN, typename C>
PP_D void dft_direct(C* v, const C* __restrict__ tw, int rstride)
{
    C out[R];
#pragma unroll
    for (int k = 0; k < R; ++k) {
        C acc = v[0];
#pragma unroll
        for (int q = 1; q < R; ++q) {
            C w = __ldg(&tw[((q * k) % R) * rstride]);
            if (SIGN > 0) w.y = -w.y;
            acc = c_add(acc, c_mul(v[q], w));
        }
        out[k] = acc;
    }
#pragma unroll
    for (int k = 0; k < R; ++k) v[k] = out[k];
}

// a pass of any radix r (a prime factor above 7): one thread per butterfly,
// each output summed directly from the r inputs in shared memory
template <int SIGN, typename C>
PP_D void stockham_pass_any(const C* __restrict__ src, C* __restrict__ dst, int n, int nlines, int ns, int r,
                            const C* __restrict__ tw, int tid, int nthreads)
{
    const int nb = n / r;
    const int tstride = n / (ns * r);
    const int total = nb * nlines;
    for (int t = tid; t < total; t += nthreads) {
        const int l = t / nb;
        const int j = t - l * nb;
        const int k = j % ns;
        const C* in = src + l * n;
        C* out = dst + l * n;
        const int base = (j / ns) * ns * r + k;
        for (int ko = 0; ko < r; ++ko) {
            C acc = in[j];
            int m = 0;  // q ko mod r
            for (int q = 1; q < r; ++q) {
                m += ko;
                if (m >= r) m -= r;
                C v = in[j + q * nb];
                if (ns > 1) {
                    C w = __ldg(&tw[q * k * tstride]);
                    if (SIGN > 0) w.y = -w.y;
                    v = c_mul(v, w);
                }
                C w = __ldg(&tw[m * nb]);
                if (SIGN > 0) w.y = -w.y;
                acc = c_add(acc, c_mul(v, w));
            }
            out[base + ko * ns] = acc;
        }
    }
}

template <int R, int SIGN, typename C>
PP_D void stockham_pass(const C* __restrict__ src, C* __restrict__ dst, int n, int nlines, int ns,
                        const C* __restrict__ tw, int tid, int nthreads)
{
    const int nb = n / R;         // butterflies per line
    const int tstride = n / (ns * R);
    const int total = nb * nlines;
    for (int t = tid; t < total; t += nthreads) {
        const int l = t / nb;
        const int j = t - l * nb;
        const int k = j % ns;
        const C* in = src + l * n;
        C* out = dst + l * n;
        C v[R];
#pragma unroll
        for (int q = 0; q < R; ++q) v[q] = in[j + q * nb];
        if (ns > 1) {
#pragma unroll
            for (int q = 1; q < R; ++q) {
                C w = __ldg(&tw[q * k * tstride]);
                if (SIGN > 0) w.y = -w.y;
                v[q] = c_mul(v[q], w);
            }
        }
        if (R == 2) dft2<SIGN>(v);
        if (R == 3) dft3<SIGN>(v);
        if (R == 4) dft4<SIGN>(v);
        if (R == 5) dft5<SIGN>(v);
        if (R == 7) dft_direct<7, SIGN>(v, tw, nb);
        if (R == 8) dft8<SIGN>(v);
        const int base = (j / ns) * ns * R + k;
#pragma unroll
        for (int q = 0; q < R; ++q) out[base + q * ns] = v[q];
    }
}

// Transform nlines lines of plan.n points held in a (line-major); b is scratch
// of the same size; tw is the plan's twiddle table in the precision of C.
// Returns the buffer that holds the result.  Ends with a __syncthreads(); must
// be entered by every thread of the block after the data in 'a' is complete
// (the caller synchronises before the call).
template <int SIGN, typename C>
__device__ C* fft_lines(C* a, C* b, int nlines, const PPFftPlan& P, const C* tw, int tid, int nthreads)
{
    C* src = a;
    C* dst = b;
    int ns = 1;
    for (int p = 0; p < P.npass; ++p) {
        const int r = P.radix[p];
        switch (r) {
        case 2: stockham_pass<2, SIGN>(src, dst, P.n, nlines, ns, tw, tid, nthreads); break;
        case 3: stockham_pass<3, SIGN>(src, dst, P.n, nlines, ns, tw, tid, nthreads); break;
        case 4: stockham_pass<4, SIGN>(src, dst, P.n, nlines, ns, tw, tid, nthreads); break;
        case 5: stockham_pass<5, SIGN>(src, dst, P.n, nlines, ns, tw, tid, nthreads); break;
        case 7: stockham_pass<7, SIGN>(src, dst, P.n, nlines, ns, tw, tid, nthreads); break;
        case 8: stockham_pass<8, SIGN>(src, dst, P.n, nlines, ns, tw, tid, nthreads); break;
        default: stockham_pass_any<SIGN>(src, dst, P.n, nlines, ns, r, tw, tid, nthreads); break;
        }
        __syncthreads();
        C* t = src;
        src = dst;
        dst = t;
        ns *= r;
    }
    return src;
}
