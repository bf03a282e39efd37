// Register-resident power-of-two FFT for a CTA tile of lines.
//
// Every line of N points is owned by N/8 threads; each thread holds 8 points
// in registers.  A pass of radix R (8, or 4 / 2 for the last pass) performs
// 8/R butterflies per thread in registers; between passes the points are
// exchanged through a padded shared-memory line (one slot of padding per 8
// points, odd line pitch) -- the Stockham autosort order, so the result comes
// out in natural order with no bit reversal.  Pass p with span Ns: butterfly
// b = t + g N/8 reads points b + q N/R, multiplies point q by W_N^{q (b mod Ns) N/(Ns R)}
// and writes output q to (b / Ns) Ns R + (b mod Ns) + q Ns.
//
// After the last pass, register v[g R + q] holds X[t + (g + q 8/R) N/8].
#pragma once

#include "pp_common.cuh"

// ---- compile-time pass plan ------------------------------------------------------
constexpr int rp_npass(int n)
{
    int p = 0;
    while (n >= 8) {
        n /= 8;
        ++p;
    }
    return n > 1 ? p + 1 : p;
}
constexpr int rp_radix(int n, int pass)
{
    int i = 0;
    while (n >= 8) {
        if (i == pass) return 8;
        n /= 8;
        ++i;
    }
    return n;
}
constexpr int rp_ns(int n, int pass)
{
    int ns = 1;
    for (int i = 0; i < pass; ++i) ns *= rp_radix(n, i);
    return ns;
}
constexpr int rp_log2(int n)
{
    int l = 0;
    while ((1 << l) < n) ++l;
    return l;
}
// padded slot of point i, and an odd line pitch
PP_HD constexpr int rp_pad(int i) { return i + (i >> 3); }
PP_HD constexpr int rp_pitch(int n) { return ((rp_pad(n - 1) + 1) | 1); }

// ---- small DFTs ----------------------------------------------------------------------
template <int SIGN, typename C>
PP_D void rdft2(C* v)
{
    C a = v[0], b = v[1];
    v[0] = c_add(a, b);
    v[1] = c_sub(a, b);
}

template <int SIGN, typename C>
PP_D void rdft4(C* v)
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
PP_D void rdft8(C* v)
{
    using R = typename CReal<C>::type;
    const R h = (R)0.70710678118654752440084436210484904;
    C e[4] = {v[0], v[2], v[4], v[6]};
    C o[4] = {v[1], v[3], v[5], v[7]};
    rdft4<SIGN>(e);
    rdft4<SIGN>(o);
    // o[k] *= exp(SIGN 2 pi i k / 8)
    C o1 = mkc<C>(h * (o[1].x - SIGN * o[1].y), h * (o[1].y + SIGN * o[1].x));
    C o2 = c_mul_si<SIGN>(o[2]);
    C o3 = mkc<C>(h * (-o[3].x - SIGN * o[3].y), h * (-o[3].y + SIGN * o[3].x));
    v[0] = c_add(e[0], o[0]);
    v[4] = c_sub(e[0], o[0]);
    v[1] = c_add(e[1], o1);
    v[5] = c_sub(e[1], o1);
    v[2] = c_add(e[2], o2);
    v[6] = c_sub(e[2], o2);
    v[3] = c_add(e[3], o3);
    v[7] = c_sub(e[3], o3);
}

template <int SIGN, int R, typename C>
PP_D void rdft(C* v)
{
    if (R == 8) rdft8<SIGN>(v);
    if (R == 4) rdft4<SIGN>(v);
    if (R == 2) rdft2<SIGN>(v);
}

// ---- one pass ------------------------------------------------------------------------
template <int N, int R, typename C>
PP_D void rp_gather(C* v, const C* line, int t)
{
#pragma unroll
    for (int g = 0; g < 8 / R; ++g)
#pragma unroll
        for (int q = 0; q < R; ++q) v[g * R + q] = line[rp_pad(t + g * (N / 8) + q * (N / R))];
}

template <int N, int R, int NS, typename C>
PP_D void rp_scatter(const C* v, C* line, int t)
{
#pragma unroll
    for (int g = 0; g < 8 / R; ++g) {
        const int b = t + g * (N / 8);
        const int base = (b / NS) * NS * R + (b % NS);
#pragma unroll
        for (int q = 0; q < R; ++q) line[rp_pad(base + q * NS)] = v[g * R + q];
    }
}

// tw[m] = exp(-2 pi i m / N) for m < N
template <int SIGN, int N, int R, int NS, typename C>
PP_D void rp_butterflies(C* v, int t, const C* __restrict__ tw)
{
#pragma unroll
    for (int g = 0; g < 8 / R; ++g) {
        C* u = v + g * R;
        if (NS > 1) {
            const int b = t + g * (N / 8);
            const int k = b % NS;
            const int s = N / (NS * R);
            C w1 = __ldg(&tw[k * s]);
            if (SIGN > 0) w1.y = -w1.y;
            if (R == 2) {
                u[1] = c_mul(u[1], w1);
            } else {
                C w2 = __ldg(&tw[2 * k * s]);
                if (SIGN > 0) w2.y = -w2.y;
                const C w3 = c_mul(w1, w2);
                u[1] = c_mul(u[1], w1);
                u[2] = c_mul(u[2], w2);
                u[3] = c_mul(u[3], w3);
                if (R == 8) {
                    C w4 = __ldg(&tw[4 * k * s]);
                    if (SIGN > 0) w4.y = -w4.y;
                    u[4] = c_mul(u[4], w4);
                    u[5] = c_mul(u[5], c_mul(w1, w4));
                    u[6] = c_mul(u[6], c_mul(w2, w4));
                    u[7] = c_mul(u[7], c_mul(w3, w4));
                }
            }
        }
        rdft<SIGN, R>(u);
    }
}

// passes 1..npass-1 of the power-of-two factor MF of the line length N (pass 0
// is done by the caller-facing entry below)
template <int SIGN, int N, int MF, int P, int NP = rp_npass(MF)>
struct RpRest {
    template <typename C>
    static PP_D void run(C* v, C* line, int t, const C* tw)
    {
        constexpr int RP = rp_radix(MF, P - 1), NSP = rp_ns(MF, P - 1);
        constexpr int R = rp_radix(MF, P), NS = rp_ns(MF, P);
        __syncthreads();  // everybody finished reading the previous contents
        rp_scatter<N, RP, NSP>(v, line, t);
        __syncthreads();
        rp_gather<N, R>(v, line, t);
        rp_butterflies<SIGN, N, R, NS>(v, t, tw);
        RpRest<SIGN, N, MF, P + 1, NP>::run(v, line, t, tw);
    }
};
template <int SIGN, int N, int MF, int NP>
struct RpRest<SIGN, N, MF, NP, NP> {
    template <typename C>
    static PP_D void run(C*, C*, int, const C*)
    {
    }
};

// Point index of register v[g R0 + q] at the input of pass 0.
template <int N>
PP_D int rp_in_index(int t, int g, int q)
{
    constexpr int R0 = rp_radix(N, 0);
    return t + g * (N / 8) + q * (N / R0);
}
// Point index of register j at the output of the last pass.
template <int N>
PP_D int rp_out_index(int t, int j)
{
    constexpr int RL = rp_radix(N, rp_npass(N) - 1);
    const int g = j / RL, q = j % RL;
    return t + (g + q * (8 / RL)) * (N / 8);
}

// The FFT of one line per thread group.  On entry v[g R0 + q] holds the
// point rp_in_index(t, g, q); 'line' is this line's padded shared-memory
// scratch (contents may still be read by other threads on entry: the first
// exchange starts with a barrier).  On exit v[j] holds X[rp_out_index(t, j)].
// Every thread of the block must call it (it contains __syncthreads()).
// MF < N (N = m MF, m odd): only the Stockham passes of the power-of-two
// factor MF run (spans 1 .. MF/R_last); the caller scatters the last one and
// finishes with the radix-m pass of span MF.
template <int SIGN, int N, int MF = N, typename C>
PP_D void rp_fft(C* v, C* line, int t, const C* __restrict__ tw)
{
    static_assert(MF >= 8 && (MF & (MF - 1)) == 0 && N % MF == 0, "power-of-two factor >= 8");
    rp_butterflies<SIGN, N, rp_radix(MF, 0), 1>(v, t, tw);
    RpRest<SIGN, N, MF, 1>::run(v, line, t, tw);
}
// the largest power of two dividing n
constexpr int rp_pow2_part(int n) { return n & -n; }
