// Transform pass for power-of-two line lengths: the same four passes and the
// same per-family pre/post-processing as pp_linepass.cu (see the reference
// citations there), built on the register-resident FFT of pp_fftreg.cuh.
//
//   FFT family (P-P): LPC complex lines per CTA, one FFT of N each.
//   DCT-II/III, DST-II/III (N-N, D-D): 2 LPC real lines per CTA, packed two
//     to a complex FFT of N (z = v1 + i v2) and separated exactly afterwards:
//     V1_k = (Z_k + conj Z_{N-k}) / 2, V2_k = (Z_k - conj Z_{N-k}) / (2i);
//     inverse: Z = V1 + i V2 of two Hermitian spectra, z = v1 + i v2.
//   DCT-IV, DST-IV (N-D, D-N): 2 LPC real lines per CTA, one complex FFT of
//     N/2 each.
//
// Phases: cooperative coalesced load of the raw tile into shared memory
// (scaling / lift / reorders folded in) -> pass-0 inputs into registers with
// the family's pre-processing -> FFT -> results back to shared memory ->
// cooperative coalesced store with the post-processing folded in.
#include "pp_common.cuh"
#include "pp_fftreg.cuh"
#include "pp_kernels.h"

namespace {

PP_D int mk_pos(int e, int n) { return (e & 1) ? (n - 1 - (e >> 1)) : (e >> 1); }

PP_D double lift2(const PPLift& L, int i, int j, int k, int nx, int ny, int nz)
{
    double s = 0.0;
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

// global element read as (re, im); real arrays give im = 0
template <typename TG, typename Real>
PP_D void gload(const void* base, long off, bool cplx, Real& re, Real& im)
{
    if (cplx) {
        const typename Vec2<TG>::type v = reinterpret_cast<const typename Vec2<TG>::type*>(base)[off];
        re = (Real)v.x;
        im = (Real)v.y;
    } else {
        re = (Real) reinterpret_cast<const TG*>(base)[off];
        im = (Real)0;
    }
}

template <typename TG, typename Real>
PP_D void gstore(void* base, long off, bool cplx, Real re, Real im)
{
    if (cplx) {
        typename Vec2<TG>::type v;
        v.x = (TG)re;
        v.y = (TG)im;
        reinterpret_cast<typename Vec2<TG>::type*>(base)[off] = v;
    } else {
        reinterpret_cast<TG*>(base)[off] = (TG)re;
    }
}

template <typename Real, typename TI, typename TO, int N, int LPC, bool INVERSE, bool STRIDED>
__global__ void __launch_bounds__(LPC * N / 8) lp2_kernel(PPLinePassArgs a)
{
    using C = typename Vec2<Real>::type;
    constexpr int NT = LPC * N / 8;
    constexpr int P1 = rp_pitch(N);
    constexpr int P4 = rp_pitch(N / 2);
    extern __shared__ __align__(16) unsigned char lp2_smem[];
    C* sb = reinterpret_cast<C*>(lp2_smem);
    Real* sr = reinterpret_cast<Real*>(lp2_smem);

    const int kind = a.kind;
    const bool fftk = kind == PP_KIND_FFT;
    const bool quarter = pp_kind_is_quarter(kind);
    const int DL = fftk ? LPC : 2 * LPC;  // data lines per tile
    const int tid = threadIdx.x;

    const int tile = blockIdx.x;
    const int plane = tile / a.tiles_per_plane;
    const int l0 = (tile - plane * a.tiles_per_plane) * DL;
    const int nl = min(DL, a.nlines - l0);
    const long base = (long)plane * a.plane_stride + (long)l0 * a.line_stride;
    const C* tw = reinterpret_cast<const C*>(a.tw);
    const C* cs = reinterpret_cast<const C*>(a.cs2);

    // ---- 1. load the raw tile ---------------------------------------------------------
    // Every element is copied asynchronously (cp.async, no register staging)
    // straight to its slot in the FFT buffer: the family's reorder / reversal
    // is the slot; signs and the RHS scaling are applied later.  Lines beyond
    // nl (last tile of a plane) are zero-filled.
    const int ldl = __ffs(DL) - 1;
    constexpr int LN = rp_log2(N);
    const int total = DL * N;
    // slot (in Real units) of element e of data line l
    auto slot = [&](int l, int e) -> int {
        if (fftk) return 2 * (l * P1 + rp_pad(e));
        if (quarter) return l * 2 * P4 + ((kind == PP_KIND_DST4) ? (N - 1 - e) : e);
        int pos;
        if (!INVERSE) pos = mk_pos(kind == PP_KIND_DCT2 ? e : N - 1 - e, N);
        else pos = (kind == PP_KIND_DCT2) ? e : N - 1 - e;
        return 2 * ((l >> 1) * P1 + rp_pad(pos)) + (l & 1);
    };
    for (int idx = tid; idx < total; idx += NT) {
        int l, e;
        if (STRIDED) {
            l = idx & (DL - 1);
            e = idx >> ldl;
        } else {
            l = idx >> LN;
            e = idx & (N - 1);
        }
        Real* d = sr + slot(l, e);
        if (l < nl) {
            const long off = base + (long)l * a.line_stride + (long)e * a.elem_stride;
            if (sizeof(TI) == sizeof(Real) && fftk && a.in_cplx) {
                cp_async<2 * sizeof(TI)>(d, reinterpret_cast<const TI*>(a.src) + 2 * off);
            } else if (sizeof(TI) == sizeof(Real)) {
                cp_async<sizeof(TI)>(d, reinterpret_cast<const TI*>(a.src) + (a.in_cplx ? 2 * off : off));
                if (fftk) d[1] = (Real)0;
            } else {
                // precision change on the way in: plain loads
                Real re, im;
                gload<TI, Real>(a.src, off, a.in_cplx, re, im);
                d[0] = re;
                if (fftk) d[1] = im;
            }
        } else {
            d[0] = (Real)0;
            if (fftk) d[1] = (Real)0;
        }
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    __syncthreads();
    if (a.rhs_scale) {
        // forward x pass: f dz dz minus the Dirichlet lift (assignRhs, modifyRhsDirichlet)
        for (int idx = tid; idx < nl * N; idx += NT) {
            const int l = idx >> LN;
            const int e = idx & (N - 1);
            Real* d = sr + slot(l, e);
            Real re = d[0] * (Real)a.dz * (Real)a.dz;
            if (a.lift.any) re = re - (Real)lift2(a.lift, e, l0 + l, plane, a.nx, a.ny, a.nz);
            d[0] = re;
            if (fftk) d[1] = d[1] * (Real)a.dz * (Real)a.dz;
        }
        __syncthreads();
    }

    // ---- 2. pre-processing into the pass-0 registers and 3. FFT --------------------
    C v[8];
    if (!quarter) {
        const int l = tid / (N / 8);
        const int t = tid - l * (N / 8);
        C* line = sb + l * P1;
        constexpr int R0 = rp_radix(N, 0);
#pragma unroll
        for (int g = 0; g < 8 / R0; ++g)
#pragma unroll
            for (int q = 0; q < R0; ++q) {
                const int m = rp_in_index<N>(t, g, q);
                if (fftk) {
                    v[g * R0 + q] = line[rp_pad(m)];
                } else if (!INVERSE) {
                    // DST-II: x'[j] = (-1)^j x[N-1-j]; odd j land in the upper half
                    const C z = line[rp_pad(m)];
                    v[g * R0 + q] = (kind == PP_KIND_DST2 && m >= N / 2) ? mkc<C>(-z.x, -z.y) : z;
                } else {
                    // DCT-III pre-processing of both packed spectra; Z = V1 + i V2
                    const C Xm = line[rp_pad(m)];
                    C V1, V2;
                    if (m == 0) {
                        V1 = mkc<C>((Real)0.5 * Xm.x, 0);
                        V2 = mkc<C>((Real)0.5 * Xm.y, 0);
                    } else {
                        const C Xn = line[rp_pad(N - m)];
                        if (m <= N / 2) {
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
                    // DST-III: the swapped input carries (-1)^m at slots m and N-m
                    if (kind == PP_KIND_DST2 && (m & 1)) Z = mkc<C>(-Z.x, -Z.y);
                    v[g * R0 + q] = Z;
                }
            }
        if (INVERSE && !fftk) rp_fft<+1, N>(v, line, t, tw);
        else if (INVERSE) rp_fft<+1, N>(v, line, t, tw);
        else rp_fft<-1, N>(v, line, t, tw);
        __syncthreads();  // all reads of the last exchange are done
#pragma unroll
        for (int j = 0; j < 8; ++j) line[rp_pad(rp_out_index<N>(t, j))] = v[j];
    } else {
        constexpr int NH = N / 2;
        const int l = tid / (NH / 8);
        const int t = tid - l * (NH / 8);
        C* line = sb + l * P4;
        const Real* raw = sr + l * 2 * P4;
        constexpr int R0 = rp_radix(NH, 0);
#pragma unroll
        for (int g = 0; g < 8 / R0; ++g)
#pragma unroll
            for (int q = 0; q < R0; ++q) {
                const int m = rp_in_index<NH>(t, g, q);
                const Real xa = raw[2 * m], xb = raw[N - 1 - 2 * m];
                const C w = __ldg(&cs[m]);  // e^{-i pi m / N}
                v[g * R0 + q] = mkc<C>(xa * w.x - xb * w.y, xa * w.y + xb * w.x);
            }
        rp_fft<-1, NH>(v, line, t, tw);
        __syncthreads();
        const Real c = INVERSE ? (Real)1 : (Real)2;
        Real* out = sr + l * 2 * P4;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const int p = rp_out_index<NH>(t, j);
            const C w = __ldg(&cs[NH + p]);  // e^{-i pi (4p+1)/(4N)}
            const Real wr = v[j].x * w.x - v[j].y * w.y;
            const Real wi = v[j].x * w.y + v[j].y * w.x;
            out[2 * p] = c * wr;
            // X_{N-1-2p} = -c Im w; DST-IV flips the sign of odd outputs
            out[N - 1 - 2 * p] = (kind == PP_KIND_DST4) ? c * wi : -c * wi;
        }
    }
    __syncthreads();

    // ---- 4. post-processing and coalesced store --------------------------------------
    const Real osc = (Real)a.out_scale;
    for (int idx = tid; idx < total; idx += NT) {
        int l, e;
        if (STRIDED) {
            l = idx & (DL - 1);
            e = idx >> ldl;
        } else {
            l = idx >> LN;
            e = idx & (N - 1);
        }
        if (l >= nl) continue;
        Real re, im = 0;
        if (fftk) {
            const C z = sb[l * P1 + rp_pad(e)];
            re = z.x;
            im = z.y;
        } else if (quarter) {
            re = sr[l * 2 * P4 + e];
        } else {
            const C* line = sb + (l >> 1) * P1;
            const int comp = l & 1;
            if (!INVERSE) {
                int k = e;
                Real sg = 1;
                if (kind == PP_KIND_DST2) {
                    k = N - 1 - e;
                    if (e & 1) sg = -1;
                }
                const C Zk = line[rp_pad(k)];
                const C Zn = line[rp_pad((N - k) & (N - 1))];
                Real vx, vy;
                if (comp == 0) {
                    vx = (Real)0.5 * (Zk.x + Zn.x);
                    vy = (Real)0.5 * (Zk.y - Zn.y);
                } else {
                    vx = (Real)0.5 * (Zk.y + Zn.y);
                    vy = -(Real)0.5 * (Zk.x - Zn.x);
                }
                const C w = __ldg(&cs[k]);  // (cos t_k, sin t_k)
                re = sg * ((Real)2. * (vx * w.x + vy * w.y));
            } else {
                int j = e;
                Real sg = 1;
                if (kind == PP_KIND_DST2) {
                    j = N - 1 - e;
                    if (e & 1) sg = -1;
                }
                const C z = line[rp_pad(mk_pos(j, N))];
                re = sg * (comp == 0 ? z.x : z.y);
            }
        }
        const long off = base + (long)l * a.line_stride + (long)e * a.elem_stride;
        if (a.acc) {
            // u = u_prev + scale * correction + zero-mode constant, in FP64
            const double u = (a.acc_read ? a.acc[off] : 0.0) + a.out_scale * (double)re +
                             (a.zplane ? a.zscale * a.zplane[plane] : 0.0);
            if (a.dst) reinterpret_cast<double2*>(a.dst)[off] = make_double2(u, 0.0);
            else a.acc[off] = u;
            continue;
        }
        if (osc != (Real)1) {
            re = osc * re;
            im = osc * im;
        }
        gstore<TO, Real>(a.dst, off, a.out_cplx, re, im);
    }
}

template <typename Real, int N, int LPC>
size_t lp2_smem_bytes()
{
    using C = typename Vec2<Real>::type;
    const size_t a1 = (size_t)LPC * rp_pitch(N);
    const size_t a4 = (size_t)2 * LPC * rp_pitch(N / 2);
    return (a1 > a4 ? a1 : a4) * sizeof(C);
}

template <typename Real, typename TI, typename TO, int N, int LPC>
cudaError_t lp2_launch_n(const PPLinePassArgs& a, bool inverse, bool strided, cudaStream_t st)
{
    const size_t smem = lp2_smem_bytes<Real, N, LPC>();
    dim3 grid(a.nplanes * a.tiles_per_plane), block(LPC * N / 8);
#define PP_LP2(INV, STR)                                                                                    \
    do {                                                                                                    \
        auto kfn = lp2_kernel<Real, TI, TO, N, LPC, INV, STR>;                                             \
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

}  // namespace

// lines per CTA (complex FFT lines) for a power-of-two length; 0 if the
// length has no specialised kernel
int pp_lp2_lpc(int n)
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

template <typename Real, typename TI, typename TO>
cudaError_t pp_launch_line_pass_pow2(const PPLinePassArgs& a, bool inverse, bool strided, cudaStream_t st)
{
    switch (a.n) {
    case 16: return lp2_launch_n<Real, TI, TO, 16, 16>(a, inverse, strided, st);
    case 32: return lp2_launch_n<Real, TI, TO, 32, 16>(a, inverse, strided, st);
    case 64: return lp2_launch_n<Real, TI, TO, 64, 8>(a, inverse, strided, st);
    case 128: return lp2_launch_n<Real, TI, TO, 128, 8>(a, inverse, strided, st);
    case 256: return lp2_launch_n<Real, TI, TO, 256, 4>(a, inverse, strided, st);
    case 512: return lp2_launch_n<Real, TI, TO, 512, 4>(a, inverse, strided, st);
    case 1024: return lp2_launch_n<Real, TI, TO, 1024, 2>(a, inverse, strided, st);
    case 2048: return lp2_launch_n<Real, TI, TO, 2048, 1>(a, inverse, strided, st);
    default: return cudaErrorInvalidValue;
    }
}

template cudaError_t pp_launch_line_pass_pow2<double, double, double>(const PPLinePassArgs&, bool, bool,
                                                                      cudaStream_t);
// the FP32 passes of the refined mixed-precision solve
template cudaError_t pp_launch_line_pass_pow2<float, float, float>(const PPLinePassArgs&, bool, bool, cudaStream_t);
