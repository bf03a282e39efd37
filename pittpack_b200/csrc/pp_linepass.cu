// Fused line-transform pass: load a tile of lines, apply the boundary
// family's pre-processing, FFT in shared memory, apply the post-processing and
// store.  One kernel covers the four transform passes of a solve:
//
//   forward x   the reference's pre(0) -> performTransformXdir -> post(0)
//               (src/pencilDcmp.cpp:5945-5966), with assignRhs's dz^2 scaling
//               (src/pencilDcmp.cpp:5591-5647) and modifyRhsDirichlet's face
//               correction (src/pencilDcmp.cpp:4623-4835) folded into the load
//   forward y   rearrangeX2Y -> pre(1) -> FFT-Y -> post(1)
//               (src/pencilDcmp.cpp:6013-6050); no transpose is made: a tile
//               of adjacent columns is read as coalesced row segments
//   inverse y   pre-rev(1) -> IFFT-Y -> post-rev(1) -> rearrangeX2YInverse
//               (src/pencilDcmp.cpp:6199-6229)
//   inverse x   pre-rev(0) -> IFFT-X -> post-rev(0) -> rescale
//               (src/pencilDcmp.cpp:6278-6305), rescale folded into the store
//
// Pre/post-processing per family follows src/signalProc.cpp:
//   DCT-II  (N-N, forward): Makhoul reorder v[j] = x[2j], v[N-1-j] = x[2j+1]
//           (:160-195); after the FFT the upper half is replaced by the
//           conjugate of the lower half and X_k = 2 (Re V_k cos t_k + Im V_k sin t_k),
//           t_k = (pi/2/N) k (:32-71).
//   DCT-III (N-N, inverse): V_0 = X_0 / 2, V_k = (1/2) e^{i t_k} (X_k - i X_{N-k}),
//           k <= N/2, conjugate upper half (:112-154); after the inverse FFT
//           x[2i] = Re v[i], x[2i+1] = Re v[N-1-i] (:76-108).
//   DST-II/III (D-D): the same with swap x'[j] = (-1)^j x[N-1-j] before and
//           after (:202-265).
//   FFT     (P-P): the plain unnormalised DFT.
//   DCT-IV / DST-IV (N-D / D-N, not in the reference): even N, an N/2-point
//           complex FFT of z_m = (x_{2m} + i x_{N-1-2m}) e^{-i pi m/N}, then
//           w_p = e^{-i pi (4p+1)/(4N)} Z_p, X_{2p} = c Re w_p, X_{N-1-2p} = -c Im w_p;
//           odd N, a 2N-point FFT of y_m = x_m e^{-i pi m/(2N)} (m < N, zero
//           above), then X_k = c Re(e^{-i pi (2k+1)/(4N)} Y_k), k < N
//           (c = 2 forward, 1 inverse); DST-IV reverses the input and flips
//           the sign of odd outputs.
// The DCT/DST families read only the real part of their input, as the
// reference's pre-processing does.
//
// The kernel runs in FP64 (the plain solve) or FP32 (the correction solves of
// the refined mixed-precision mode, for lengths the power-of-two kernel does
// not cover).  In FP32 the inverse x pass ends in the refinement epilogue:
// u = u_prev + v / (nx ny) + zero-mode constant, accumulated in FP64.
#include "pp_common.cuh"
#include "pp_fft.cuh"
#include "pp_kernels.h"

namespace {

template <typename R>
struct Vec2T;
template <>
struct Vec2T<double> {
    using type = double2;
};
template <>
struct Vec2T<float> {
    using type = float2;
};

// Makhoul even/odd position: where input element e goes (and, inverse, where
// output element e is read from)
PP_D int makhoul_pos(int e, int n) { return (e & 1) ? (n - 1 - (e >> 1)) : (e >> 1); }

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

template <typename R, bool INVERSE, bool STRIDED, bool IN_CPLX, bool OUT_CPLX>
__global__ void __launch_bounds__(PP_LINE_THREADS) line_pass_kernel(PPLinePassArgs a)
{
    using C = typename Vec2T<R>::type;
    extern __shared__ __align__(16) unsigned char pp_lp_smem[];
    C* smem = reinterpret_cast<C*>(pp_lp_smem);
    const int n = a.n;
    const int kind = a.kind;
    const bool quarter = pp_kind_is_quarter(kind);
    const bool q_odd = quarter && (n & 1);  // quarter-wave, odd length: 2n-point FFT
    const int nf = a.fft.n;  // n; n/2 (even) or 2n (odd) for the quarter-wave families
    const int tid = threadIdx.x;
    const int nth = blockDim.x;
    // FFT and family twiddles in the kernel's precision
    const C* tw;
    const C* cs;
    if constexpr (sizeof(R) == 8) {
        tw = reinterpret_cast<const C*>(a.fft.tw);
        cs = reinterpret_cast<const C*>(a.cs);
    } else {
        tw = reinterpret_cast<const C*>(a.tw);
        cs = reinterpret_cast<const C*>(a.cs2);
    }
    const R* src = reinterpret_cast<const R*>(a.src);

    const int tile = blockIdx.x;
    const int plane = tile / a.tiles_per_plane;
    const int l0 = (tile - plane * a.tiles_per_plane) * a.L;
    const int nl = min(a.L, a.nlines - l0);
    const long base = (long)plane * a.plane_stride + (long)l0 * a.line_stride;

    C* bufA = smem;
    C* bufB = smem + (size_t)a.L * nf;
    R* stage = reinterpret_cast<R*>(bufB);  // raw real lines, n per line

    const bool staged = quarter || (INVERSE && kind != PP_KIND_FFT);

    // ---- 1. load -----------------------------------------------------------
    const int total = nl * n;
    for (int idx = tid; idx < total; idx += nth) {
        int l, e;
        if (STRIDED) {
            l = idx % nl;
            e = idx / nl;
        } else {
            l = idx / n;
            e = idx - l * n;
        }
        const long off = base + (long)l * a.line_stride + (long)e * a.elem_stride;
        C v;
        if (IN_CPLX) v = reinterpret_cast<const C*>(src)[off];
        else v = mkc<C>(src[off], (R)0);
        if (a.rhs_scale) {
            v.x = v.x * (R)a.dz * (R)a.dz;
            v.y = v.y * (R)a.dz * (R)a.dz;
            if (a.lift.any) {
                // forward x-pass: line index = y index j, plane = z index k
                v.x = v.x - (R)lift_at(a.lift, e, l0 + l, plane, a.nx, a.ny, a.nz);
            }
        }
        if (kind == PP_KIND_FFT) {
            bufA[l * nf + e] = v;
        } else if (!staged) {
            // forward DCT-II / DST-II: reorder straight into the FFT input
            if (kind == PP_KIND_DCT2) {
                bufA[l * nf + makhoul_pos(e, n)] = mkc<C>(v.x, (R)0);
            } else {  // DST-II: x'[j] = (-1)^j x[n-1-j]
                const int j = n - 1 - e;
                const R s = (j & 1) ? (R)-1 : (R)1;
                bufA[l * nf + makhoul_pos(j, n)] = mkc<C>(s * v.x, (R)0);
            }
        } else {
            // stage the real part (reversed / sign-swapped where the family says)
            if (kind == PP_KIND_DST2) {  // inverse DST: swap first
                const int j = n - 1 - e;
                stage[l * n + j] = (j & 1) ? -v.x : v.x;
            } else if (kind == PP_KIND_DST4) {
                stage[l * n + (n - 1 - e)] = v.x;
            } else {
                stage[l * n + e] = v.x;
            }
        }
    }
    __syncthreads();

    // ---- 2. pre-processing that needs the whole line ------------------------
    if (staged) {
        const int tot2 = nl * nf;
        for (int idx = tid; idx < tot2; idx += nth) {
            const int l = idx / nf;
            const int k = idx - l * nf;
            const R* X = stage + l * n;
            C V;
            if (q_odd) {
                if (k < n) {
                    const C w = __ldg(&cs[k]);  // e^{-i pi k / (2n)}
                    V = mkc<C>(X[k] * w.x, X[k] * w.y);
                } else {
                    V = mkc<C>((R)0, (R)0);
                }
            } else if (quarter) {
                const C w = __ldg(&cs[k]);  // e^{-i pi k / n}
                const R xa = X[2 * k], xb = X[n - 1 - 2 * k];
                V = mkc<C>(xa * w.x - xb * w.y, xa * w.y + xb * w.x);
            } else if (k == 0) {
                V = mkc<C>((R)0.5 * X[0], (R)0);
            } else if (k <= n / 2) {
                const C t = __ldg(&cs[k]);  // (cos t_k, sin t_k)
                V.y = (R)0.5 * (t.y * X[k] - t.x * X[n - k]);
                V.x = (R)0.5 * (t.x * X[k] + t.y * X[n - k]);
            } else {
                const int kk = n - k;
                const C t = __ldg(&cs[kk]);
                V.y = -((R)0.5 * (t.y * X[kk] - t.x * X[n - kk]));
                V.x = (R)0.5 * (t.x * X[kk] + t.y * X[n - kk]);
            }
            bufA[l * nf + k] = V;
        }
        __syncthreads();
    }

    // ---- 3. FFT --------------------------------------------------------------
    const bool backward = INVERSE && !quarter;
    C* res = backward ? fft_lines<+1>(bufA, bufB, nl, a.fft, tw, tid, nth)
                      : fft_lines<-1>(bufA, bufB, nl, a.fft, tw, tid, nth);

    // ---- 4. post-processing and store ---------------------------------------
    for (int idx = tid; idx < total; idx += nth) {
        int l, e;
        if (STRIDED) {
            l = idx % nl;
            e = idx / nl;
        } else {
            l = idx / n;
            e = idx - l * n;
        }
        const C* Rl = res + l * nf;
        C o;
        if (kind == PP_KIND_FFT) {
            o = Rl[e];
        } else if (q_odd) {
            const C w = __ldg(&cs[n + e]);  // e^{-i pi (2e+1)/(4n)}
            const C z = Rl[e];
            R v = z.x * w.x - z.y * w.y;
            v *= INVERSE ? (R)1 : (R)2;
            if (kind == PP_KIND_DST4 && (e & 1)) v = -v;
            o = mkc<C>(v, (R)0);
        } else if (quarter) {
            const int k = e;
            const int p = (k & 1) == 0 ? (k >> 1) : ((n - 1 - k) >> 1);
            const C w = __ldg(&cs[nf + p]);  // e^{-i pi (4p+1)/(4n)}
            const C z = Rl[p];
            const R wr = z.x * w.x - z.y * w.y;
            const R wi = z.x * w.y + z.y * w.x;
            R v = ((k & 1) == 0) ? wr : -wi;
            v *= INVERSE ? (R)1 : (R)2;
            if (kind == PP_KIND_DST4 && (k & 1)) v = -v;
            o = mkc<C>(v, (R)0);
        } else if (!INVERSE) {
            // DCT-II value at k, optionally through the DST swap
            int k = e;
            R sgn = 1;
            if (kind == PP_KIND_DST2) {
                sgn = (e & 1) ? (R)-1 : (R)1;
                k = n - 1 - e;
            }
            C V;
            if (k > n / 2) {
                V = Rl[n - k];
                V.y = -V.y;
            } else {
                V = Rl[k];
            }
            const C t = __ldg(&cs[k]);
            o = mkc<C>(sgn * ((R)2. * (V.x * t.x + V.y * t.y)), (R)0);
        } else {
            // DCT-III output reorder, optionally through the DST swap
            if (kind == PP_KIND_DST2) {
                const int j = n - 1 - e;
                const R s = (e & 1) ? (R)-1 : (R)1;
                o = mkc<C>(s * Rl[makhoul_pos(j, n)].x, (R)0);
            } else {
                o = mkc<C>(Rl[makhoul_pos(e, n)].x, (R)0);
            }
        }
        const long off = base + (long)l * a.line_stride + (long)e * a.elem_stride;
        if (a.acc) {
            // u = u_prev + scale * correction + zero-mode constant, in FP64
            const double u = (a.acc_read ? a.acc[off] : 0.0) + a.out_scale * (double)o.x +
                             (a.zplane ? a.zscale * a.zplane[plane] : 0.0);
            if (a.dst) reinterpret_cast<double2*>(a.dst)[off] = make_double2(u, 0.0);
            else a.acc[off] = u;
            continue;
        }
        if (a.out_scale != 1.0) {
            o.x = (R)a.out_scale * o.x;
            o.y = (R)a.out_scale * o.y;
        }
        R* dst = reinterpret_cast<R*>(a.dst);
        if (OUT_CPLX) reinterpret_cast<C*>(dst)[off] = o;
        else dst[off] = o.x;
    }
}

template <typename R, bool INVERSE, bool STRIDED>
cudaError_t launch_typed(const PPLinePassArgs& a, bool in_cplx, bool out_cplx, size_t smem, cudaStream_t st)
{
    dim3 grid(a.nplanes * a.tiles_per_plane);
    dim3 block(PP_LINE_THREADS);
#define PP_LAUNCH(IC, OC)                                                                                   \
    do {                                                                                                    \
        auto kfn = line_pass_kernel<R, INVERSE, STRIDED, IC, OC>;                                          \
        cudaError_t e = cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem); \
        if (e != cudaSuccess) return e;                                                                     \
        kfn<<<grid, block, smem, st>>>(a);                                                                  \
        return cudaGetLastError();                                                                          \
    } while (0)
    if (in_cplx && out_cplx) PP_LAUNCH(true, true);
    if (in_cplx && !out_cplx) PP_LAUNCH(true, false);
    if (!in_cplx && out_cplx) PP_LAUNCH(false, true);
    PP_LAUNCH(false, false);
#undef PP_LAUNCH
}

template <typename R>
cudaError_t launch_prec(const PPLinePassArgs& a, bool inverse, bool strided, bool in_cplx, bool out_cplx,
                        cudaStream_t st)
{
    const size_t smem = pp_line_pass_smem(a.L, a.fft.n, sizeof(R) == 4);
    if (inverse) {
        return strided ? launch_typed<R, true, true>(a, in_cplx, out_cplx, smem, st)
                       : launch_typed<R, true, false>(a, in_cplx, out_cplx, smem, st);
    }
    return strided ? launch_typed<R, false, true>(a, in_cplx, out_cplx, smem, st)
                   : launch_typed<R, false, false>(a, in_cplx, out_cplx, smem, st);
}

}  // namespace

size_t pp_line_pass_smem(int L, int nfft, bool fp32)
{
    return 2 * (size_t)L * nfft * (fp32 ? sizeof(float2) : sizeof(double2));
}

cudaError_t pp_launch_line_pass(const PPLinePassArgs& a, bool inverse, bool strided, bool in_cplx, bool out_cplx,
                                cudaStream_t st, bool fp32)
{
    return fp32 ? launch_prec<float>(a, inverse, strided, in_cplx, out_cplx, st)
                : launch_prec<double>(a, inverse, strided, in_cplx, out_cplx, st);
}
