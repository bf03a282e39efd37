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
//   DCT-IV / DST-IV (N-D / D-N, not in the reference): N/2-point complex FFT
//           of z_m = (x_{2m} + i x_{N-1-2m}) e^{-i pi m/N}, then
//           w_p = e^{-i pi (4p+1)/(4N)} Z_p, X_{2p} = c Re w_p, X_{N-1-2p} = -c Im w_p
//           (c = 2 forward, 1 inverse); DST-IV reverses the input and flips
//           the sign of odd outputs.
// The DCT/DST families read only the real part of their input, as the
// reference's pre-processing does.
#include "pp_common.cuh"
#include "pp_fft.cuh"
#include "pp_kernels.h"

namespace {

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

template <bool INVERSE, bool STRIDED, bool IN_CPLX, bool OUT_CPLX>
__global__ void __launch_bounds__(PP_LINE_THREADS) line_pass_kernel(PPLinePassArgs a)
{
    extern __shared__ double2 smem[];
    const int n = a.n;
    const int kind = a.kind;
    const bool quarter = pp_kind_is_quarter(kind);
    const int nf = a.fft.n;  // n, or n/2 for the quarter-wave families
    const int tid = threadIdx.x;
    const int nth = blockDim.x;

    const int tile = blockIdx.x;
    const int plane = tile / a.tiles_per_plane;
    const int l0 = (tile - plane * a.tiles_per_plane) * a.L;
    const int nl = min(a.L, a.nlines - l0);
    const long base = (long)plane * a.plane_stride + (long)l0 * a.line_stride;

    double2* bufA = smem;
    double2* bufB = smem + (size_t)a.L * nf;
    double* stage = reinterpret_cast<double*>(bufB);  // raw real lines, n per line

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
        double2 v;
        if (IN_CPLX) v = reinterpret_cast<const double2*>(a.src)[off];
        else v = make_double2(a.src[off], 0.0);
        if (a.rhs_scale) {
            v.x = v.x * a.dz * a.dz;
            v.y = v.y * a.dz * a.dz;
            if (a.lift.any) {
                // forward x-pass: line index = y index j, plane = z index k
                v.x = v.x - lift_at(a.lift, e, l0 + l, plane, a.nx, a.ny, a.nz);
            }
        }
        if (kind == PP_KIND_FFT) {
            bufA[l * nf + e] = v;
        } else if (!staged) {
            // forward DCT-II / DST-II: reorder straight into the FFT input
            if (kind == PP_KIND_DCT2) {
                bufA[l * nf + makhoul_pos(e, n)] = make_double2(v.x, 0.0);
            } else {  // DST-II: x'[j] = (-1)^j x[n-1-j]
                const int j = n - 1 - e;
                const double s = (j & 1) ? -1.0 : 1.0;
                bufA[l * nf + makhoul_pos(j, n)] = make_double2(s * v.x, 0.0);
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
            const double* X = stage + l * n;
            double2 V;
            if (quarter) {
                const double2 w = __ldg(&a.cs[k]);  // e^{-i pi k / n}
                const double xa = X[2 * k], xb = X[n - 1 - 2 * k];
                V = make_double2(xa * w.x - xb * w.y, xa * w.y + xb * w.x);
            } else if (k == 0) {
                V = make_double2(0.5 * 1.0 * X[0], 0.0);
            } else if (k <= n / 2) {
                const double2 t = __ldg(&a.cs[k]);  // (cos t_k, sin t_k)
                V.y = 0.5 * (t.y * X[k] - t.x * X[n - k]);
                V.x = 0.5 * (t.x * X[k] + t.y * X[n - k]);
            } else {
                const int kk = n - k;
                const double2 t = __ldg(&a.cs[kk]);
                V.y = -(0.5 * (t.y * X[kk] - t.x * X[n - kk]));
                V.x = 0.5 * (t.x * X[kk] + t.y * X[n - kk]);
            }
            bufA[l * nf + k] = V;
        }
        __syncthreads();
    }

    // ---- 3. FFT --------------------------------------------------------------
    const bool backward = INVERSE && !quarter;
    double2* res = backward ? fft_lines<+1>(bufA, bufB, nl, a.fft, tid, nth)
                            : fft_lines<-1>(bufA, bufB, nl, a.fft, tid, nth);

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
        const double2* R = res + l * nf;
        double2 o;
        if (kind == PP_KIND_FFT) {
            o = R[e];
        } else if (quarter) {
            const int k = e;
            int p;
            double v;
            if ((k & 1) == 0) {
                p = k >> 1;
            } else {
                p = (n - 1 - k) >> 1;
            }
            const double2 w = __ldg(&a.cs[nf + p]);  // e^{-i pi (4p+1)/(4n)}
            const double2 z = R[p];
            const double wr = z.x * w.x - z.y * w.y;
            const double wi = z.x * w.y + z.y * w.x;
            v = ((k & 1) == 0) ? wr : -wi;
            v *= INVERSE ? 1.0 : 2.0;
            if (kind == PP_KIND_DST4 && (k & 1)) v = -v;
            o = make_double2(v, 0.0);
        } else if (!INVERSE) {
            // DCT-II value at k, optionally through the DST swap
            int k = e;
            double sgn = 1.0;
            if (kind == PP_KIND_DST2) {
                sgn = (e & 1) ? -1.0 : 1.0;
                k = n - 1 - e;
            }
            double2 V;
            if (k > n / 2) {
                V = R[n - k];
                V.y = -V.y;
            } else {
                V = R[k];
            }
            const double2 t = __ldg(&a.cs[k]);
            o = make_double2(sgn * (2. * (V.x * t.x + V.y * t.y)), 0.0);
        } else {
            // DCT-III output reorder, optionally through the DST swap
            if (kind == PP_KIND_DST2) {
                const int j = n - 1 - e;
                const double s = (e & 1) ? -1.0 : 1.0;
                o = make_double2(s * R[makhoul_pos(j, n)].x, 0.0);
            } else {
                o = make_double2(R[makhoul_pos(e, n)].x, 0.0);
            }
        }
        if (a.out_scale != 1.0) {
            o.x = a.out_scale * o.x;
            o.y = a.out_scale * o.y;
        }
        const long off = base + (long)l * a.line_stride + (long)e * a.elem_stride;
        if (OUT_CPLX) reinterpret_cast<double2*>(a.dst)[off] = o;
        else a.dst[off] = o.x;
    }
}

template <bool INVERSE, bool STRIDED>
cudaError_t launch_typed(const PPLinePassArgs& a, bool in_cplx, bool out_cplx, size_t smem, cudaStream_t st)
{
    dim3 grid(a.nplanes * a.tiles_per_plane);
    dim3 block(PP_LINE_THREADS);
#define PP_LAUNCH(IC, OC)                                                                                   \
    do {                                                                                                    \
        auto kfn = line_pass_kernel<INVERSE, STRIDED, IC, OC>;                                             \
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

}  // namespace

size_t pp_line_pass_smem(int L, int nfft) { return 2 * (size_t)L * nfft * sizeof(double2); }

cudaError_t pp_launch_line_pass(const PPLinePassArgs& a, bool inverse, bool strided, bool in_cplx, bool out_cplx,
                                cudaStream_t st)
{
    const size_t smem = pp_line_pass_smem(a.L, a.fft.n);
    if (inverse) {
        return strided ? launch_typed<true, true>(a, in_cplx, out_cplx, smem, st)
                       : launch_typed<true, false>(a, in_cplx, out_cplx, smem, st);
    }
    return strided ? launch_typed<false, true>(a, in_cplx, out_cplx, smem, st)
                   : launch_typed<false, false>(a, in_cplx, out_cplx, smem, st);
}
