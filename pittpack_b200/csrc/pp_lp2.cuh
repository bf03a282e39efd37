// Transform pass for line lengths N = m 2^k (m = 1, 3, 5, 9, 15; the FFT's
// power-of-two factor at least 8): the same four passes and the same
// per-family pre/post-processing as pp_linepass.cu (see the reference
// citations there), built on the register-resident FFT of pp_fftreg.cuh and
// specialised at compile time on the length and the boundary family, so that
// reorders, signs and twiddle selection cost no run-time branches.  The
// power-of-two factor runs as register passes; an odd factor m > 1 as one
// final Stockham pass of radix m and span 2^k in shared memory.
//
//   FFT family (P-P): LPC complex lines per CTA, one FFT of N each.
//   DCT-II/III, DST-II/III (N-N, D-D): 2 LPC real lines per CTA, packed two
//     to a complex FFT of N (z = v1 + i v2) and separated exactly afterwards:
//     V1_k = (Z_k + conj Z_{N-k}) / 2, V2_k = (Z_k - conj Z_{N-k}) / (2i);
//     inverse: Z = V1 + i V2 of two Hermitian spectra, z = v1 + i v2.
//   DCT-IV, DST-IV (N-D, D-N): 2 LPC real lines per CTA, one complex FFT of
//     N/2 each.
//
// Phases: (1) the raw tile is copied into shared memory by cp.async, 16-byte
// chunks where the layout allows (a line of N elements, or for the strided y
// pass a row segment of the tile's lines); (2) each thread gathers its pass-0
// FFT inputs from the raw tile with the family's reorder folded into the
// addresses (radix 8 first, so which half a register falls in is known at
// compile time); (3) FFT, ending with the radix-m pass where m > 1;
// (4) post-processing of pairs (k, N-k), each Z read once, and stores.  The
// forward x pass's dz^2 scaling is applied to the
// outputs (a linear factor), the Dirichlet lift is subtracted (divided by
// dz^2) from the few raw elements on a Dirichlet face.
#pragma once

#include <type_traits>

#include "pp_common.cuh"
#include "pp_fft.cuh"
#include "pp_fftreg.cuh"
#include "pp_kernels.h"

namespace pp_lp2 {

// F_R2C / F_C2R: the periodic x pass of a real RHS on half spectra (k <= N/2,
// the other half is the conjugate mirror): two real lines per complex FFT
enum Fam : int { F_DST2 = 0, F_DCT2 = 1, F_FFT = 2, F_Q4 = 3, F_R2C = 4, F_C2R = 5 };

// raw tile of a family: complex elements (FFT, half-spectrum input) or real;
// elements per line in the contiguous pass (half spectra: N/2 + 1)
template <int FAM>
constexpr bool raw_cplx() { return FAM == F_FFT || FAM == F_C2R; }
template <int FAM, int N>
constexpr int raw_len() { return FAM == F_C2R ? N / 2 + 1 : N; }

template <typename T>
struct Vec2;
template <>
struct Vec2<double> {
    using type = double2;
};
template <>
struct Vec2<float> {
    using type = float2;
};

PP_D int mk_pos(int e, int n) { return (e & 1) ? (n - 1 - (e >> 1)) : (e >> 1); }

// R-point DFT in registers, R = 3 or 5 (pp_fft.cuh)
template <int SIGN, int R, typename C>
PP_D void small_dft(C* v)
{
    if constexpr (R == 3) dft3<SIGN>(v);
    else dft5<SIGN>(v);
}

// MM = A B point DFT by one Cooley-Tukey step: n = B n1 + n2, k = k1 + A k2;
// A-point DFTs over n1, twiddles W_MM^{n2 k1}, B-point DFTs over n2.  W_MM^x
// is taken from the FFT's own table as tw[x * stride] (stride = NF / MM).
template <int SIGN, int A, int B, typename C>
PP_D void dft_ct(C* v, const C* __restrict__ tw, int stride)
{
    C y[B][A];
#pragma unroll
    for (int n2 = 0; n2 < B; ++n2) {
#pragma unroll
        for (int n1 = 0; n1 < A; ++n1) y[n2][n1] = v[B * n1 + n2];
        small_dft<SIGN, A>(y[n2]);
    }
#pragma unroll
    for (int n2 = 1; n2 < B; ++n2)
#pragma unroll
        for (int k1 = 1; k1 < A; ++k1) {
            C w = __ldg(&tw[n2 * k1 * stride]);
            if (SIGN > 0) w.y = -w.y;
            y[n2][k1] = c_mul(y[n2][k1], w);
        }
#pragma unroll
    for (int k1 = 0; k1 < A; ++k1) {
        C z[B];
#pragma unroll
        for (int n2 = 0; n2 < B; ++n2) z[n2] = y[n2][k1];
        small_dft<SIGN, B>(z);
#pragma unroll
        for (int k2 = 0; k2 < B; ++k2) v[k1 + A * k2] = z[k2];
    }
}

PP_D double lift_at(const PPLift& L, int i, int j, int k, int nx, int ny, int nz)
{
    double s = 0.0;
    // same order as the reference: z-min, z-max, x-min, x-max, y-min, y-max
    if (L.z0 && k == 0) s += L.z0[i + (long)nx * j];
    if (L.z1 && k == nz - 1) s += L.z1[i + (long)nx * j];
    if (L.x0 && i == 0) s += L.x0[j + (long)ny * k];
    if (L.x1 && i == nx - 1) s += L.x1[j + (long)ny * k];
    if (L.y0 && j == 0) s += L.y0[i + (long)nx * k];
    if (L.y1 && j == ny - 1) s += L.y1[i + (long)nx * k];
    return s;
}

// asynchronous global -> shared copy of BYTES (4, 8 or 16)
template <int BYTES>
PP_D void cp_async(void* smem, const void* gmem)
{
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    if (BYTES == 16) asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
    if (BYTES == 8) asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem) : "memory");
    if (BYTES == 4) asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(gmem) : "memory");
}

// bulk-copy staging: smem_u32, mbar_*, bulk_g2s (pp_common.cuh)

// row pitch (elements) of the strided pass's raw tile [element][line]: the
// smallest pitch above the tile's line count whose rows start on 16-byte
// boundaries and are an odd number of 16-byte units apart, so that threads
// reading consecutive rows fall in different banks
template <int FAM, int LPC>
constexpr int raw_row_pitch(int elem_bytes)
{
    const int dl = FAM == F_FFT ? LPC : 2 * LPC;
    int rp = dl + 1;
    while ((rp * elem_bytes) % 16 != 0 || ((rp * elem_bytes / 16) & 1) == 0) ++rp;
    return rp;
}

// The forward DCT-II / DST-II passes (Makhoul's reorder) and both DCT-IV /
// DST-IV passes (x[2m], x[N-1-2m]) read the rows of a strided tile two apart.
// Their raw tile keeps the even rows first and the odd rows from row
// split_odd_base on, so that the reads fall on consecutive rows; the base is
// 4 mod 8 rows so that a row and the next one still land in different banks
// while the tile is copied in.  (The contiguous passes keep their 16-byte
// copies: an even/odd split there needs 8-byte ones, which cost more than the
// two-way conflicts they remove.)
template <int FAM, bool INVERSE, bool STRIDED>
constexpr bool split_rows()
{
    return STRIDED && ((!INVERSE && (FAM == F_DCT2 || FAM == F_DST2)) || FAM == F_Q4);
}
template <int N>
constexpr int split_odd_base() { return (N / 2 + 7 - 4) / 8 * 8 + 4; }
template <int FAM, bool INVERSE, bool STRIDED, int N>
constexpr int raw_rows()
{
    return split_rows<FAM, INVERSE, STRIDED>() ? split_odd_base<N>() + N / 2 : raw_len<FAM, N>();
}
template <int FAM, bool INVERSE, bool STRIDED, int N>
PP_HD constexpr int raw_row(int e)
{
    return split_rows<FAM, INVERSE, STRIDED>() ? ((e & 1) ? split_odd_base<N>() + (e >> 1) : (e >> 1)) : e;
}

// pitch (complex elements) of an FFT line buffer.  The strided pass reads the
// lines' spectra four lines by two indices per 8-thread phase: a pitch of
// 2 mod 8 sixteen-byte units puts them in 8 distinct banks.
template <int N, bool STRIDED>
constexpr int line_pitch()
{
    if (!STRIDED || N < 64) return rp_pitch(N);
    int p = rp_pad(N - 1) + 1;
    while (p % 8 != 2) ++p;
    return p;
}

// shared memory of one CTA: the FFT line buffers, or the raw tile that
// aliases them if that is larger (the padded strided tile)
template <typename Real, int N, int LPC, int FAM, bool INVERSE, bool STRIDED>
constexpr size_t smem_bytes()
{
    using C = typename Vec2<Real>::type;
    constexpr size_t a1 = (size_t)LPC * line_pitch<N, STRIDED>() * sizeof(C);
    constexpr size_t a4 = (size_t)2 * LPC * rp_pitch(N / 2) * sizeof(C);
    constexpr size_t lines = a1 > a4 ? a1 : a4;
    constexpr size_t re = raw_cplx<FAM>() ? sizeof(C) : sizeof(Real);
    constexpr size_t raw = (size_t)raw_rows<FAM, INVERSE, STRIDED, N>() *
                           (STRIDED ? raw_row_pitch<FAM, LPC>((int)re) : (FAM == F_FFT ? LPC : 2 * LPC)) * re;
    return lines > raw ? lines : raw;
}

// one output element (line l of the tile, element e): the refinement
// epilogue (acc set) or a scaled store
template <typename Real>
PP_D void put(const PPLinePassArgs& a, long off, int plane, Real re, Real im, Real sc)
{
    using C = typename Vec2<Real>::type;
    if (a.acc) {
        // u = u_prev + scale * correction + zero-mode constant, in FP64
        const double u = (a.acc_read ? a.acc[off] : 0.0) + a.out_scale * (double)re +
                         (a.zplane ? a.zscale * a.zplane[plane] : 0.0);
        if (a.dst) reinterpret_cast<double2*>(a.dst)[off] = make_double2(u, 0.0);
        else a.acc[off] = u;
        return;
    }
    if (a.out_cplx) reinterpret_cast<C*>(a.dst)[off] = mkc<C>(sc * re, sc * im);
    else reinterpret_cast<Real*>(a.dst)[off] = sc * re;
}

template <typename Real, int N, int LPC, int FAM, bool INVERSE, bool STRIDED>
__device__ __forceinline__ void lp2_body(const PPLinePassArgs& a)
{
    using C = typename Vec2<Real>::type;
    constexpr bool FFTK = FAM == F_FFT;
    constexpr bool Q4 = FAM == F_Q4;
    constexpr bool R2C = FAM == F_R2C;
    constexpr bool C2R = FAM == F_C2R;
    constexpr bool RAWC = raw_cplx<FAM>();
    constexpr int LLEN = raw_len<FAM, N>();  // raw elements per line
    constexpr int NT = LPC * N / 8;
    constexpr int DL = FFTK ? LPC : 2 * LPC;  // data lines per tile
    constexpr int LDL = rp_log2(DL);
    // raw tile elements: complex for the FFT family, real otherwise
    using RE = typename std::conditional<RAWC, C, Real>::type;
    extern __shared__ __align__(16) unsigned char lp2_smem[];
    C* sb = reinterpret_cast<C*>(lp2_smem);
    RE* raw = reinterpret_cast<RE*>(lp2_smem);

    const int tid = threadIdx.x;
    const int tile = blockIdx.x;
    const int plane = tile / a.tiles_per_plane;
    const int l0 = (tile - plane * a.tiles_per_plane) * DL;
    const int nl = min(DL, a.nlines - l0);
    const long base = (long)plane * a.plane_stride + (long)l0 * (a.tile_stride ? a.tile_stride : a.line_stride);
    const C* tw = reinterpret_cast<const C*>(a.tw);
    const C* cs = reinterpret_cast<const C*>(a.cs2);
    // raw position of (line l, element e)
    constexpr int RP = raw_row_pitch<FAM, LPC>((int)sizeof(RE));
    auto ridx = [](int l, int e) -> int {
        return STRIDED ? raw_row<FAM, INVERSE, STRIDED, N>(e) * RP + l : l * LLEN + e;
    };

    // ---- 1. load the raw tile ----------------------------------------------------------
    // full tiles whose global element type equals the raw one go in 16-byte
    // chunks (a line of N elements, or a row segment of DL elements); the
    // rest element by element (real <-> complex conversion, partial tiles)
    const bool same = RAWC ? (a.in_cplx != 0) : (a.in_cplx == 0);
    constexpr int RUN = STRIDED ? DL : LLEN;         // elements per contiguous run
    constexpr int PER = 16 / (int)sizeof(RE);        // elements per 16-byte chunk
    constexpr bool VOK = (RUN * (int)sizeof(RE)) % 16 == 0;  // runs are whole chunks
    if (!STRIDED && VOK && same && a.vec16 && nl == DL) {
        // contiguous pass, full tile of whole 16-byte lines: one bulk copy per
        // line, issued by one thread and counted on an mbarrier, so that the
        // staged bytes skip the LSU pipe the rest of the pass is bound by
        __shared__ __align__(8) unsigned long long bulk_bar;
        const unsigned bar = smem_u32(&bulk_bar);
        constexpr unsigned LB = (unsigned)(LLEN * sizeof(RE));
        if (tid == 0) mbar_init(bar);
        __syncthreads();
        if (tid == 0) {
            mbar_expect(bar, LB * DL);
            const RE* src = reinterpret_cast<const RE*>(a.src);
            for (int r = 0; r < DL; ++r) bulk_g2s(raw + r * LLEN, src + base + (long)r * a.line_stride, LB, bar);
        }
        // a bounded wait (about a second of polls): a CTA whose copies never
        // land counts itself and leaves without output, with every thread
        const bool landed = mbar_wait0(bar, 1L << 22);
        if (__syncthreads_or(!landed)) {
            if (tid == 0 && a.err) atomicAdd(a.err, 1);
            return;
        }
    } else if (VOK && same && a.vec16 && nl == DL) {
        constexpr int CPR = VOK ? RUN / PER : 1;     // chunks per run
        constexpr int TOT = (STRIDED ? LLEN : DL) * CPR;
        const RE* src = reinterpret_cast<const RE*>(a.src);
        for (int c = tid; c < TOT; c += NT) {
            int r = c / CPR;  // run: element row (strided) or line
            int k = (c - r * CPR) * PER;
            if (STRIDED && CPR == 4 && !split_rows<FAM, INVERSE, STRIDED>()) {
                // an 8-thread phase copies rows r and r + 4 (odd row pitch in
                // 16-byte units: 8 distinct banks); a warp still covers 8 rows
                const int j = c & 31;
                r = (c >> 5) * 8 + ((j >> 3) & 3) + 4 * ((j >> 2) & 1);
                k = (j & 3) * PER;
            }
            const long goff = base + (STRIDED ? (long)r * a.elem_stride : (long)r * a.line_stride) + k;
            cp_async<16>(raw + (STRIDED ? raw_row<FAM, INVERSE, STRIDED, N>(r) * RP : r * LLEN) + k, src + goff);
        }
    } else {
        for (int idx = tid; idx < DL * LLEN; idx += NT) {
            int l, e;
            if (STRIDED) {
                l = idx & (DL - 1);
                e = idx >> LDL;
            } else if (C2R) {
                l = idx / LLEN;
                e = idx - l * LLEN;
            } else {
                l = idx / N;
                e = idx - l * N;
            }
            Real* d = reinterpret_cast<Real*>(raw + ridx(l, e));
            if (l < nl) {
                const long off = base + (long)l * a.line_stride + (long)e * a.elem_stride;
                const Real* s = reinterpret_cast<const Real*>(a.src);
                if (RAWC) {
                    if (a.in_cplx) {
                        cp_async<2 * sizeof(Real)>(d, s + 2 * off);
                    } else {
                        cp_async<sizeof(Real)>(d, s + off);
                        d[1] = (Real)0;
                    }
                } else {
                    // the DCT/DST families read the real part only
                    cp_async<sizeof(Real)>(d, s + (a.in_cplx ? 2 * off : off));
                }
            } else {
                d[0] = (Real)0;
                if (RAWC) d[1] = (Real)0;
            }
        }
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    __syncthreads();

    // ---- 1b. Dirichlet lift (forward x pass of the plain solve) ---------------------
    // b = f dz^2 - lift; the dz^2 factor is applied to the outputs, so the
    // raw elements on a Dirichlet face lose lift / dz^2 here
    if (a.rhs_scale && a.lift.any) {
        const double inv = 1.0 / (a.dz * a.dz);
        const PPLift& L = a.lift;
        const bool whole = (L.z0 && plane == 0) || (L.z1 && plane == a.nz - 1) || (L.y0 && l0 == 0) ||
                           (L.y1 && l0 + nl >= a.ny);
        if (whole) {
            for (int idx = tid; idx < nl * N; idx += NT) {
                const int l = idx / N, e = idx - (idx / N) * N;
                Real* d = reinterpret_cast<Real*>(raw + ridx(l, e));
                d[0] = d[0] - (Real)(lift_at(L, e, l0 + l, plane, a.nx, a.ny, a.nz) * inv);
            }
        } else if (L.x0 || L.x1) {
            for (int idx = tid; idx < 2 * nl; idx += NT) {
                const int l = idx >> 1, e = (idx & 1) ? N - 1 : 0;
                Real* d = reinterpret_cast<Real*>(raw + ridx(l, e));
                d[0] = d[0] - (Real)(lift_at(L, e, l0 + l, plane, a.nx, a.ny, a.nz) * inv);
            }
        }
        __syncthreads();
    }

    // ---- 2. pass-0 registers: the family's pre-processing, from the raw tile ----------
    // radix 8 first: register q holds point m = t + q N/8 (t < N/8), so the
    // half of the line it falls in is known from q at compile time
    constexpr int NF = Q4 ? N / 2 : N;  // FFT length
    constexpr int MF = rp_pow2_part(NF);  // its power-of-two factor (register passes)
    constexpr int MM = NF / MF;           // and its odd factor (one radix-MM pass)
    static_assert(MM == 1 || MM == 3 || MM == 5 || MM == 9 || MM == 15, "FFT length 2^k, 3 2^k, 5 2^k, 9 2^k or 15 2^k");
    constexpr int TPL = NF / 8;         // threads per FFT line
    static_assert(rp_radix(MF, 0) == 8, "the first pass is radix 8");
    static_assert(!(FAM == F_DST2 && INVERSE) || TPL % 2 == 0, "the DST-III sign uses the parity of t");
    const int fl = tid / TPL;           // FFT line of this thread
    const int t = tid - fl * TPL;
    C* line = sb + fl * (Q4 ? rp_pitch(N / 2) : line_pitch<N, STRIDED>());
    C v[8];
    if constexpr (FFTK) {
#pragma unroll
        for (int q = 0; q < 8; ++q) v[q] = raw[ridx(fl, t + q * (N / 8))];
    } else if constexpr (R2C) {
        // two real lines as one complex line z = x_a + i x_b
        const int la = 2 * fl, lb = la + 1;
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int m = t + q * (N / 8);
            if (STRIDED) v[q] = *reinterpret_cast<const C*>(raw + ridx(la, m));
            else v[q] = mkc<C>(raw[ridx(la, m)], raw[ridx(lb, m)]);
        }
    } else if constexpr (C2R) {
        // Z_m = X_a,m + i X_b,m with the upper half rebuilt as the conjugate
        // mirror X_m = conj X_{N-m} of the stored half spectra
        const int la = 2 * fl, lb = la + 1;
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int m = t + q * (N / 8);
            C xa, xb;
            if (q < 4 || (q == 4 && t == 0)) {
                xa = raw[ridx(la, m)];
                xb = raw[ridx(lb, m)];
            } else {
                const C ya = raw[ridx(la, N - m)], yb = raw[ridx(lb, N - m)];
                xa = mkc<C>(ya.x, -ya.y);
                xb = mkc<C>(yb.x, -yb.y);
            }
            v[q] = mkc<C>(xa.x - xb.y, xa.y + xb.x);
        }
    } else if constexpr (Q4) {
        // z_m = (x[2m] + i x[N-1-2m]) e^{-i pi m / N}; DST-IV reverses its input
        const bool rev = a.kind == PP_KIND_DST4;
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int m = t + q * (NF / 8);
            const int ea = 2 * m, eb = N - 1 - 2 * m;
            const Real xa = raw[ridx(fl, rev ? N - 1 - ea : ea)];
            const Real xb = raw[ridx(fl, rev ? N - 1 - eb : eb)];
            const C w = __ldg(&cs[m]);
            v[q] = mkc<C>(xa * w.x - xb * w.y, xa * w.y + xb * w.x);
        }
    } else if constexpr (!INVERSE) {
        // DCT-II: Makhoul reorder v[m] = x[2m] (m < N/2), x[2N-1-2m] (m >= N/2);
        // DST-II first swaps x'[j] = (-1)^j x[N-1-j]: v[m] = x[N-1-2m] or -x[2m-N]
        const int la = 2 * fl, lb = la + 1;
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int m = t + q * (N / 8);
            int e;
            if (FAM == F_DCT2) e = q < 4 ? 2 * m : 2 * N - 1 - 2 * m;
            else e = q < 4 ? N - 1 - 2 * m : 2 * m - N;
            const Real s = (FAM == F_DST2 && q >= 4) ? (Real)-1 : (Real)1;
            if (STRIDED) {
                // lines la, lb are adjacent in a row: one 16-byte read
                const C z = *reinterpret_cast<const C*>(raw + ridx(la, e));
                v[q] = mkc<C>(s * z.x, s * z.y);
            } else {
                v[q] = mkc<C>(s * raw[ridx(la, e)], s * raw[ridx(lb, e)]);
            }
        }
    } else {
        // DCT-III pre-processing of both packed spectra; Z = V1 + i V2.  DST-III
        // reads the reversed line and carries (-1)^m
        const int la = 2 * fl, lb = la + 1;
        auto X = [&](int k) -> C {
            const int e = FAM == F_DCT2 ? k : N - 1 - k;
            if (STRIDED) return *reinterpret_cast<const C*>(raw + ridx(la, e));
            return mkc<C>(raw[ridx(la, e)], raw[ridx(lb, e)]);
        };
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int m = t + q * (N / 8);
            const C Xm = X(m);
            C V1, V2;
            if (q == 0 && t == 0) {
                V1 = mkc<C>((Real)0.5 * Xm.x, 0);
                V2 = mkc<C>((Real)0.5 * Xm.y, 0);
            } else {
                const C Xn = X(N - m);
                if (q < 4 || (q == 4 && t == 0)) {
                    const C w = __ldg(&cs[m]);
                    V1 = mkc<C>((Real)0.5 * (w.x * Xm.x + w.y * Xn.x), (Real)0.5 * (w.y * Xm.x - w.x * Xn.x));
                    V2 = mkc<C>((Real)0.5 * (w.x * Xm.y + w.y * Xn.y), (Real)0.5 * (w.y * Xm.y - w.x * Xn.y));
                } else {
                    const C w = __ldg(&cs[N - m]);
                    V1 = mkc<C>((Real)0.5 * (w.x * Xn.x + w.y * Xm.x), -((Real)0.5 * (w.y * Xn.x - w.x * Xm.x)));
                    V2 = mkc<C>((Real)0.5 * (w.x * Xn.y + w.y * Xm.y), -((Real)0.5 * (w.y * Xn.y - w.x * Xm.y)));
                }
            }
            C Z = mkc<C>(V1.x - V2.y, V1.y + V2.x);
            if (FAM == F_DST2 && (t & 1)) Z = mkc<C>(-Z.x, -Z.y);  // m and t have the same parity
            v[q] = Z;
        }
    }

    // ---- 3. FFT (its first exchange starts with a barrier, so the raw tile
    //         that aliases the line buffers is no longer needed) ----------------------
    constexpr int FS = (INVERSE && !Q4) ? +1 : -1;
    rp_fft<FS, NF, MF>(v, line, t, tw);
    __syncthreads();  // all reads of the last exchange are done
    if constexpr (MM == 1) {
#pragma unroll
        for (int j = 0; j < 8; ++j) line[rp_pad(rp_out_index<NF>(t, j))] = v[j];
    } else {
        // Stockham output of the last register pass, then the final pass of
        // radix MM and span MF, in place: butterfly j < MF reads points
        // j + q MF, multiplies point q by W_NF^{q j} and writes output q to
        // j + q MF (natural order)
        constexpr int NPM = rp_npass(MF);
        rp_scatter<NF, rp_radix(MF, NPM - 1), rp_ns(MF, NPM - 1)>(v, line, t);
        __syncthreads();
        constexpr int NB = (MF + TPL - 1) / TPL;  // butterflies of this thread, at most
        C u[NB][MM];
#pragma unroll
        for (int b = 0; b < NB; ++b) {
            const int j = t + b * TPL;
            if (j < MF) {
#pragma unroll
                for (int q = 0; q < MM; ++q) u[b][q] = line[rp_pad(j + q * MF)];
            }
        }
        __syncthreads();
#pragma unroll
        for (int b = 0; b < NB; ++b) {
            const int j = t + b * TPL;
            if (j < MF) {
#pragma unroll
                for (int q = 1; q < MM; ++q) {
                    C w = __ldg(&tw[q * j]);
                    if (FS > 0) w.y = -w.y;
                    u[b][q] = c_mul(u[b][q], w);
                }
                if constexpr (MM == 3 || MM == 5) small_dft<FS, MM>(u[b]);
                else if constexpr (MM == 9) dft_ct<FS, 3, 3>(u[b], tw, MF);
                else dft_ct<FS, 5, 3>(u[b], tw, MF);
#pragma unroll
                for (int q = 0; q < MM; ++q) line[rp_pad(j + q * MF)] = u[b][q];
            }
        }
    }
    __syncthreads();

    // ---- 4. post-processing and stores ------------------------------------------------
    // thread -> (line, index): the strided pass runs the line fastest, so that
    // a warp writes row segments; the contiguous pass runs the index fastest
    const Real sc = (Real)(a.out_scale * (a.rhs_scale ? a.dz * a.dz : 1.0));
    // output strides (computed here, after the FFT, so that they hold no
    // registers through it): their own (z-tiled spectrum, half spectra) or,
    // when unset, the input's
    const bool own = a.o_elem_stride != 0;
    const long oes = own ? a.o_elem_stride : a.elem_stride;
    const long ols = own ? a.o_line_stride : a.line_stride;
    const long ops = own ? a.o_plane_stride : a.plane_stride;
    const long ots = own ? a.o_tile_stride : a.tile_stride;
    const long obase = (long)plane * ops + (long)l0 * (ots ? ots : ols);
    auto goff = [&](int l, int e) -> long { return obase + (long)l * ols + (long)e * oes; };
    constexpr int P1 = line_pitch<N, STRIDED>();
    // the two packed real lines of a strided pass are adjacent in the output:
    // one 16-byte store for both where the layout allows
    const bool pair = !a.acc && !a.out_cplx && ols == 1 && ((oes | ops | obase) & 1) == 0 &&
                      (reinterpret_cast<unsigned long>(a.dst) & 15) == 0;
    auto put2 = [&](int la, int e, Real va, Real vb) {
        if (STRIDED && pair && la + 1 < nl) {
            reinterpret_cast<C*>(reinterpret_cast<Real*>(a.dst) + goff(la, e))[0] = mkc<C>(sc * va, sc * vb);
        } else {
            if (la < nl) put<Real>(a, goff(la, e), plane, va, (Real)0, sc);
            if (la + 1 < nl) put<Real>(a, goff(la + 1, e), plane, vb, (Real)0, sc);
        }
    };
    if constexpr (FFTK) {
        for (int idx = tid; idx < LPC * N; idx += NT) {
            int l, e;
            if (STRIDED) {
                l = idx & (LPC - 1);
                e = idx >> rp_log2(LPC);
            } else {
                l = idx / N;
                e = idx - l * N;
            }
            if (l >= nl) continue;
            const C z = sb[l * P1 + rp_pad(e)];
            put<Real>(a, goff(l, e), plane, z.x, z.y, sc);
        }
    } else if constexpr (R2C) {
        // half spectra k = 0..N/2 of both packed lines:
        // X_a,k = (Z_k + conj Z_{N-k}) / 2, X_b,k = (Z_k - conj Z_{N-k}) / (2i)
        constexpr int LL = rp_log2(LPC);
        for (int idx = tid; idx < LPC * (N / 2); idx += NT) {
            int cl, kk;
            if (STRIDED) {
                cl = idx & (LPC - 1);
                kk = idx >> LL;
            } else {
                cl = idx / (N / 2);
                kk = idx - cl * (N / 2);
            }
            const int la = 2 * cl, lb = la + 1;
            const C* ln = sb + cl * P1;
            auto emit = [&](int k, C Zk, C Zn) {
                if (la < nl)
                    put<Real>(a, goff(la, k), plane, (Real)0.5 * (Zk.x + Zn.x), (Real)0.5 * (Zk.y - Zn.y), sc);
                if (lb < nl)
                    put<Real>(a, goff(lb, k), plane, (Real)0.5 * (Zk.y + Zn.y), -(Real)0.5 * (Zk.x - Zn.x), sc);
            };
            const C Zk = ln[rp_pad(kk)];
            if (kk == 0) {
                const C Zh = ln[rp_pad(N / 2)];
                emit(0, Zk, Zk);
                emit(N / 2, Zh, Zh);
            } else {
                emit(kk, Zk, ln[rp_pad(N - kk)]);
            }
        }
        // the rows of the half spectra are padded to the y pass's tile width:
        // the padding columns are zeroed, since the y pass of a real family
        // transforms two columns as one complex line and a column's partner
        // must not carry stale values into it
        const int npad = (int)ols - (N / 2 + 1);
        for (int idx = tid; idx < DL * npad; idx += NT) {
            const int l = idx / npad, e = N / 2 + 1 + (idx - (idx / npad) * npad);
            if (l < nl) put<Real>(a, goff(l, e), plane, (Real)0, (Real)0, sc);
        }
    } else if constexpr (C2R) {
        // z = x_a + i x_b: both real lines at once
        constexpr int LL = rp_log2(LPC);
        for (int idx = tid; idx < LPC * N; idx += NT) {
            int cl, e;
            if (STRIDED) {
                cl = idx & (LPC - 1);
                e = idx >> LL;
            } else {
                cl = idx / N;
                e = idx - cl * N;
            }
            const int la = 2 * cl, lb = la + 1;
            const C z = sb[cl * P1 + rp_pad(e)];
            if (la < nl) put<Real>(a, goff(la, e), plane, z.x, (Real)0, sc);
            if (lb < nl) put<Real>(a, goff(lb, e), plane, z.y, (Real)0, sc);
        }
    } else if constexpr (Q4) {
        // w_p = e^{-i pi (4p+1)/(4N)} Z_p: X[2p] = c Re w_p, X[N-1-2p] = -c Im w_p
        // (c = 2 forward, 1 inverse); DST-IV flips the sign of the odd outputs
        constexpr int NH = N / 2, P4 = rp_pitch(N / 2);
        const Real c = INVERSE ? (Real)1 : (Real)2;
        const Real so = a.kind == PP_KIND_DST4 ? c : -c;
        for (int idx = tid; idx < DL * NH; idx += NT) {
            int l, p;
            if (STRIDED) {
                l = idx & (DL - 1);
                p = idx >> LDL;
            } else {
                l = idx / NH;
                p = idx - l * NH;
            }
            if (l >= nl) continue;
            const C z = sb[l * P4 + rp_pad(p)];
            const C w = __ldg(&cs[NH + p]);
            const Real wr = z.x * w.x - z.y * w.y;
            const Real wi = z.x * w.y + z.y * w.x;
            put<Real>(a, goff(l, 2 * p), plane, c * wr, (Real)0, sc);
            put<Real>(a, goff(l, N - 1 - 2 * p), plane, so * wi, (Real)0, sc);
        }
    } else if constexpr (!INVERSE) {
        // pairs (k, N-k) of both packed lines: X_k = 2 (Re V_k cos t_k + Im V_k sin t_k),
        // output e = k (DCT-II) or e = N-1-k with sign (-1)^e (DST-II)
        constexpr int LL = rp_log2(LPC);
        for (int idx = tid; idx < LPC * (N / 2); idx += NT) {
            int cl, kk;
            if (STRIDED) {
                cl = idx & (LPC - 1);
                kk = idx >> LL;
            } else {
                cl = idx / (N / 2);
                kk = idx - cl * (N / 2);
            }
            const int la = 2 * cl;
            const C* ln = sb + cl * P1;
            const int k1 = kk == 0 ? 0 : kk;
            const int k2 = kk == 0 ? N / 2 : N - kk;
            const C Z1 = ln[rp_pad(k1)];
            const C Z2 = ln[rp_pad(k2)];
            // partners: Z_{N-k1} = Z2 and Z_{N-k2} = Z1, except at k = 0 and N/2
            const C P1z = kk == 0 ? Z1 : Z2;
            const C P2z = kk == 0 ? Z2 : Z1;
            const C w1 = __ldg(&cs[k1]);
            const C w2 = __ldg(&cs[k2]);
            auto emit = [&](int k, C Zk, C Zn, C w) {
                // V1 (line a) and V2 (line b) at k
                const Real v1x = (Real)0.5 * (Zk.x + Zn.x), v1y = (Real)0.5 * (Zk.y - Zn.y);
                const Real v2x = (Real)0.5 * (Zk.y + Zn.y), v2y = -(Real)0.5 * (Zk.x - Zn.x);
                int e = k;
                Real sg = (Real)2;
                if (FAM == F_DST2) {
                    e = N - 1 - k;
                    if (e & 1) sg = (Real)-2;
                }
                put2(la, e, sg * (v1x * w.x + v1y * w.y), sg * (v2x * w.x + v2y * w.y));
            };
            emit(k1, Z1, P1z, w1);
            emit(k2, Z2, P2z, w2);
        }
    } else {
        // DCT-III output reorder x[2i] = Re v[i], x[2i+1] = Re v[N-1-i] of both
        // packed lines; DST-III reverses with sign (-1)^e
        constexpr int LL = rp_log2(LPC);
        for (int idx = tid; idx < LPC * N; idx += NT) {
            int cl, e;
            if (STRIDED && LPC == 4) {
                // an 8-thread phase takes outputs e, e + 2 of four lines: their
                // spectrum slots are adjacent (8 distinct banks)
                cl = idx & 3;
                const int rest = idx >> 3;
                e = 4 * (rest >> 1) + (rest & 1) + 2 * ((idx >> 2) & 1);
            } else if (STRIDED) {
                cl = idx & (LPC - 1);
                e = idx >> LL;
            } else {
                cl = idx / N;
                e = idx - cl * N;
            }
            const int la = 2 * cl;
            int j = e;
            Real sg = (Real)1;
            if (FAM == F_DST2) {
                j = N - 1 - e;
                if (e & 1) sg = (Real)-1;
            }
            const C z = sb[cl * P1 + rp_pad(mk_pos(j, N))];
            put2(la, e, sg * z.x, sg * z.y);
        }
    }
}

// the power-of-two lengths, and (with a register bound that leaves room for
// one more CTA per SM) the lengths with an odd factor, whose final radix-m
// pass holds up to three butterflies per thread.  The second argument of
// __launch_bounds__ is what bounds the registers.
constexpr int lpm_min_blocks(int nt) { return 65536 / (84 * nt) > 1 ? 65536 / (84 * nt) : 1; }
template <typename Real, int N, int LPC, int FAM, bool INVERSE, bool STRIDED>
__global__ void __launch_bounds__(LPC * N / 8) lp2_kernel(PPLinePassArgs a)
{
    lp2_body<Real, N, LPC, FAM, INVERSE, STRIDED>(a);
}
template <typename Real, int N, int LPC, int FAM, bool INVERSE, bool STRIDED>
__global__ void __launch_bounds__(LPC * N / 8, lpm_min_blocks(LPC * N / 8)) lpm_kernel(PPLinePassArgs a)
{
    lp2_body<Real, N, LPC, FAM, INVERSE, STRIDED>(a);
}
// the periodic family's 512-point FP64 instances (complex lines, half
// spectra): bounded to 48 registers, five CTAs of 256 threads per SM
// (measured faster; the real families' instances spill under the same bound
// and are not)
template <typename Real, int N, int LPC, int FAM, bool INVERSE, bool STRIDED>
__global__ void __launch_bounds__(LPC * N / 8, 5) lp2b_kernel(PPLinePassArgs a)
{
    lp2_body<Real, N, LPC, FAM, INVERSE, STRIDED>(a);
}
template <typename Real, int N, int LPC, int FAM, bool INVERSE, bool STRIDED>
constexpr auto pass_kernel()
{
    if constexpr (N == 512 && (FAM == F_FFT || FAM == F_R2C || FAM == F_C2R) && std::is_same<Real, double>::value)
        return lp2b_kernel<Real, N, LPC, FAM, INVERSE, STRIDED>;
    else if constexpr ((N & (N - 1)) == 0) return lp2_kernel<Real, N, LPC, FAM, INVERSE, STRIDED>;
    else return lpm_kernel<Real, N, LPC, FAM, INVERSE, STRIDED>;
}

template <typename Real, int N, int LPC, int FAM>
cudaError_t launch_fam(const PPLinePassArgs& a, bool inverse, bool strided, cudaStream_t st)
{
    dim3 grid(a.nplanes * a.tiles_per_plane), block(LPC * N / 8);
#define PP_LP2(INV, STR)                                                                                    \
    do {                                                                                                    \
        constexpr size_t smem = smem_bytes<Real, N, LPC, FAM, INV, STR>();                                  \
        auto kfn = pass_kernel<Real, N, LPC, FAM, INV, STR>();                                              \
        cudaError_t e = cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem); \
        if (e != cudaSuccess) return e;                                                                     \
        kfn<<<grid, block, smem, st>>>(a);                                                                  \
        return cudaGetLastError();                                                                          \
    } while (0)
    if (inverse && strided) PP_LP2(true, true);
    if (inverse && !strided) PP_LP2(true, false);
    if (!inverse && strided) PP_LP2(false, true);
    PP_LP2(false, false);
#undef PP_LP2
}

template <typename Real, int N, int LPC, int FAM>
cudaError_t launch_half(const PPLinePassArgs& a, cudaStream_t st)
{
    // the contiguous x pass only: forward real -> half spectra, inverse back
    constexpr size_t smem = smem_bytes<Real, N, LPC, FAM, FAM == F_C2R, false>();
    auto kfn = pass_kernel<Real, N, LPC, FAM, FAM == F_C2R, false>();
    cudaError_t e = cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    kfn<<<a.nplanes * a.tiles_per_plane, LPC * N / 8, smem, st>>>(a);
    return cudaGetLastError();
}

template <typename Real, int N, int LPC>
cudaError_t launch_n(const PPLinePassArgs& a, bool inverse, bool strided, cudaStream_t st)
{
    if (a.half && a.kind == PP_KIND_FFT) {
        if (strided) return cudaErrorInvalidValue;
        return inverse ? launch_half<Real, N, LPC, F_C2R>(a, st) : launch_half<Real, N, LPC, F_R2C>(a, st);
    }
    switch (a.kind) {
    case PP_KIND_DST2: return launch_fam<Real, N, LPC, F_DST2>(a, inverse, strided, st);
    case PP_KIND_DCT2: return launch_fam<Real, N, LPC, F_DCT2>(a, inverse, strided, st);
    case PP_KIND_FFT: return launch_fam<Real, N, LPC, F_FFT>(a, inverse, strided, st);
    default: return launch_fam<Real, N, LPC, F_Q4>(a, inverse, strided, st);
    }
}

// lines per CTA (complex FFT lines) for a power-of-two length; 0 if the
// length has no specialised kernel
inline int lpc_of(int n)
{
    switch (n) {
    case 16: return 16;
    case 32: return 16;
    case 64: return 8;
    case 128: return 8;
    case 256: return 4;
    case 512: return 4;
    case 1024: return 2;
    case 2048: return 1;
    default: return 0;
    }
}

template <typename Real>
cudaError_t launch(const PPLinePassArgs& a, bool inverse, bool strided, cudaStream_t st)
{
    switch (a.n) {
    case 16: return launch_n<Real, 16, 16>(a, inverse, strided, st);
    case 32: return launch_n<Real, 32, 16>(a, inverse, strided, st);
    case 64: return launch_n<Real, 64, 8>(a, inverse, strided, st);
    case 128: return launch_n<Real, 128, 8>(a, inverse, strided, st);
    case 256: return launch_n<Real, 256, 4>(a, inverse, strided, st);
    case 512: return launch_n<Real, 512, 4>(a, inverse, strided, st);
    case 1024: return launch_n<Real, 1024, 2>(a, inverse, strided, st);
    case 2048: return launch_n<Real, 2048, 1>(a, inverse, strided, st);
    default: return cudaErrorInvalidValue;
    }
}

// lines per CTA for the lengths m 2^k, m = 3, 5, 9, 15, with 2^k >= 16 so
// that the quarter-wave families' half-length FFT still starts with a
// radix-8 register pass (the register passes take the power-of-two factor,
// one shared-memory pass the odd one); 0 if the length has no such kernel
inline int lpm_of(int n)
{
    switch (n) {
    case 48: return 8;
    case 80: return 8;
    case 96: return 8;
    case 144: return 8;
    case 160: return 4;
    case 192: return 4;
    case 240: return 4;
    case 288: return 4;
    case 320: return 4;
    case 384: return 4;
    case 480: return 2;
    case 576: return 2;
    case 640: return 2;
    case 768: return 2;
    case 960: return 1;
    case 1152: return 1;
    case 1280: return 1;
    case 1536: return 1;
    default: return 0;
    }
}
inline bool lpm_odd9or15(int n) { return n == 144 || n == 240 || n == 288 || n == 480 || n == 576 || n == 960 || n == 1152; }

// the odd factors 9 and 15 (their own translation units)
template <typename Real>
cudaError_t launch_mixed915(const PPLinePassArgs& a, bool inverse, bool strided, cudaStream_t st)
{
    switch (a.n) {
    case 144: return launch_n<Real, 144, 8>(a, inverse, strided, st);
    case 240: return launch_n<Real, 240, 4>(a, inverse, strided, st);
    case 288: return launch_n<Real, 288, 4>(a, inverse, strided, st);
    case 480: return launch_n<Real, 480, 2>(a, inverse, strided, st);
    case 576: return launch_n<Real, 576, 2>(a, inverse, strided, st);
    case 960: return launch_n<Real, 960, 1>(a, inverse, strided, st);
    case 1152: return launch_n<Real, 1152, 1>(a, inverse, strided, st);
    default: return cudaErrorInvalidValue;
    }
}

template <typename Real>
cudaError_t launch_mixed(const PPLinePassArgs& a, bool inverse, bool strided, cudaStream_t st)
{
    switch (a.n) {
    case 48: return launch_n<Real, 48, 8>(a, inverse, strided, st);
    case 80: return launch_n<Real, 80, 8>(a, inverse, strided, st);
    case 96: return launch_n<Real, 96, 8>(a, inverse, strided, st);
    case 160: return launch_n<Real, 160, 4>(a, inverse, strided, st);
    case 192: return launch_n<Real, 192, 4>(a, inverse, strided, st);
    case 320: return launch_n<Real, 320, 4>(a, inverse, strided, st);
    case 384: return launch_n<Real, 384, 4>(a, inverse, strided, st);
    case 640: return launch_n<Real, 640, 2>(a, inverse, strided, st);
    case 768: return launch_n<Real, 768, 2>(a, inverse, strided, st);
    case 1280: return launch_n<Real, 1280, 1>(a, inverse, strided, st);
    case 1536: return launch_n<Real, 1536, 1>(a, inverse, strided, st);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace pp_lp2
