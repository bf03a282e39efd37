// Shared device helpers for the PittPack B200 solver.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#define PP_HD __host__ __device__ __forceinline__
#define PP_D __device__ __forceinline__

// transform kind of one direction (x or y).  The first three are the
// reference's tags (extractTag, src/pencilDcmp.cpp:3636-3668: DST 0, DCT 1,
// FFT 2); the N-D and D-N families are not in the reference.
enum PPKind : int {
    PP_KIND_DST2 = 0,  // D-D: DST-II forward, DST-III inverse
    PP_KIND_DCT2 = 1,  // N-N: DCT-II forward, DCT-III inverse
    PP_KIND_FFT = 2,   // P-P: complex DFT
    PP_KIND_DCT4 = 3,  // N-D: DCT-IV both ways
    PP_KIND_DST4 = 4,  // D-N: DST-IV both ways
};

PP_HD bool pp_kind_is_fft(int k) { return k == PP_KIND_FFT; }
PP_HD bool pp_kind_is_quarter(int k) { return k == PP_KIND_DCT4 || k == PP_KIND_DST4; }

PP_D double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
PP_D double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
PP_D double2 cmul(double2 a, double2 b) { return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
PP_D double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
PP_D double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
// multiply by i*s (s = +1 or -1)
PP_D double2 cmul_i(double2 a, double s) { return make_double2(-s * a.y, s * a.x); }

// ---- complex helpers for float2 / double2 ------------------------------------
template <typename C>
struct CReal;
template <>
struct CReal<double2> {
    using type = double;
};
template <>
struct CReal<float2> {
    using type = float;
};

template <typename C>
PP_D C mkc(typename CReal<C>::type x, typename CReal<C>::type y)
{
    C r;
    r.x = x;
    r.y = y;
    return r;
}
template <typename C>
PP_D C c_add(C a, C b) { return mkc<C>(a.x + b.x, a.y + b.y); }
template <typename C>
PP_D C c_sub(C a, C b) { return mkc<C>(a.x - b.x, a.y - b.y); }
template <typename C>
PP_D C c_mul(C a, C b) { return mkc<C>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
template <typename C>
PP_D C c_scale(C a, typename CReal<C>::type s) { return mkc<C>(a.x * s, a.y * s); }
// multiply by SIGN * i
template <int SIGN, typename C>
PP_D C c_mul_si(C a) { return SIGN > 0 ? mkc<C>(-a.y, a.x) : mkc<C>(a.y, -a.x); }
