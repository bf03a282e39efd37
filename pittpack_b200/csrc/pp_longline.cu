// Transform passes for lines longer than one tile of the generic kernel holds
// (its two shared-memory buffers of one line: an FFT length past 7264 in
// FP64).  The reference hands any length to cuFFT / FFTW
// (src/poissonGPU.cpp:13, src/poissonCPU.cpp:56); here such a pass runs
// through a global scratch array W:
//
//   pre      the family's load and pre-processing of the generic kernel
//            (pp_linepass.cu, steps 1-2), one FFT input point per thread,
//            into W in natural order;
//   FFT      nf = n1 n2 by the four-step method, both steps on the generic
//            kernel (complex family, in place): n1-point FFTs over the
//            stride-n2 columns m1 of m = m1 n2 + m2, the twiddles
//            W_nf^(k1 m2), n2-point FFTs over the rows, which leaves X[k1 + n1 k2]
//            at k1 n2 + k2;
//   post     the family's post-processing and store of the generic kernel
//            (step 4), reading X through that index map.
//
// An FFT length with a prime factor past one tile takes the chirp
// z-transform (Bluestein): with c_k = e^{i pi k^2 / nf},
//   sum_m V_m e^{-2 pi i m k / nf} = conj(c_k) sum_m (V_m conj(c_m)) c_{k-m},
// a cyclic convolution of length M (a power of two >= 2 nf - 1, split
// M = n1 n2): the pre kernel writes V conj(c) padded with zeros to M points,
// a four-step FFT leaves its spectrum in the transposed order, which is
// multiplied by the chirp kernel's spectrum (a table in that order), and the
// inverse four-step run in the reverse order of its steps returns the
// convolution in natural order; the post kernel reads conj(c_k) / M times it.
// The backward transform conjugates every chirp.
//
// W keeps a line's points contiguous for the contiguous (x) passes and the
// lines of a plane contiguous ([plane][m][line]) for the strided (y) passes,
// so that the pre and post kernels read and write the pass's arrays with
// adjacent threads on adjacent addresses.  Both precisions (the refined
// solve's FP32 passes).
#include <cmath>

#include "pp_common.cuh"
#include "pp_fft.cuh"
#include "pp_kernels.h"

namespace {

template <typename R>
struct LlVec;
template <>
struct LlVec<double> {
    using type = double2;
};
template <>
struct LlVec<float> {
    using type = float2;
};

PP_D int ll_makhoul_pos(int e, int n) { return (e & 1) ? (n - 1 - (e >> 1)) : (e >> 1); }
// the element whose Makhoul position is p
PP_D int ll_makhoul_src(int p, int n) { return p < (n + 1) / 2 ? 2 * p : 2 * (n - 1 - p) + 1; }

PP_D double ll_lift_at(const PPLift& L, int i, int j, int k, int nx, int ny, int nz)
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

// the pass's input element e of line l in plane p, after the forward x
// pass's dz^2 scaling and Dirichlet correction
template <typename R>
PP_D typename LlVec<R>::type ll_load(const PPLinePassArgs& a, const R* src, bool in_cplx, long base, int l, int p, int e)
{
    using C = typename LlVec<R>::type;
    const long off = base + (long)e * a.elem_stride;
    C v;
    if (in_cplx) v = reinterpret_cast<const C*>(src)[off];
    else v = mkc<C>(src[off], (R)0);
    if (a.rhs_scale) {
        v.x = v.x * (R)a.dz * (R)a.dz;
        v.y = v.y * (R)a.dz * (R)a.dz;
        if (a.lift.any) v.x = v.x - (R)ll_lift_at(a.lift, e, l, p, a.nx, a.ny, a.nz);
    }
    return v;
}

// position of point m of line (p, l) in W (lines of lw points)
PP_D long ll_w(bool strided, int nl, int lw, int p, int l, int m)
{
    return strided ? ((long)p * lw + m) * nl + l : ((long)p * nl + l) * lw + m;
}

// the chirp factor of point k: conj(c_k) forward, c_k backward
template <typename C>
PP_D C ll_chirp(const C* chirp, int k, int back)
{
    C c = __ldg(&chirp[k]);
    if (!back) c.y = -c.y;
    return c;
}

// ---- pre: one FFT input point per thread ------------------------------------------------
// lw = nf (four-step), or M (chirp z-transform: the input times the chirp
// factor, zero from nf to M)
template <typename R>
__global__ void ll_pre_kernel(PPLinePassArgs a, typename LlVec<R>::type* W, int nf, int lw,
                              const typename LlVec<R>::type* __restrict__ chirp, int back, int inverse, int strided,
                              int in_cplx)
{
    using C = typename LlVec<R>::type;
    const R* src = reinterpret_cast<const R*>(a.src);
    const C* cs = sizeof(R) == 8 ? reinterpret_cast<const C*>(a.cs) : reinterpret_cast<const C*>(a.cs2);
    const int n = a.n, kind = a.kind, nl = a.nlines;
    const bool quarter = pp_kind_is_quarter(kind);
    const bool q_odd = quarter && (n & 1);
    const bool staged = quarter || (inverse && kind != PP_KIND_FFT);
    const long total = (long)a.nplanes * nl * lw;
    for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < total; idx += (long)gridDim.x * blockDim.x) {
        int p, l, k;
        if (strided) {
            p = (int)(idx / ((long)lw * nl));
            const long r = idx - (long)p * lw * nl;
            k = (int)(r / nl);
            l = (int)(r - (long)k * nl);
        } else {
            const long g = idx / lw;
            k = (int)(idx - g * lw);
            p = (int)(g / nl);
            l = (int)(g - (long)p * nl);
        }
        if (k >= nf) {
            W[ll_w(strided, nl, lw, p, l, k)] = mkc<C>((R)0, (R)0);
            continue;
        }
        const long base = (long)p * a.plane_stride + (long)l * a.line_stride;
        // the real line the staged families transform (reversed / sign-swapped)
        auto X = [&](int j) -> R {
            if (kind == PP_KIND_DST2) {
                const R v = ll_load<R>(a, src, in_cplx, base, l, p, n - 1 - j).x;
                return (j & 1) ? -v : v;
            }
            if (kind == PP_KIND_DST4) return ll_load<R>(a, src, in_cplx, base, l, p, n - 1 - j).x;
            return ll_load<R>(a, src, in_cplx, base, l, p, j).x;
        };
        C V;
        if (kind == PP_KIND_FFT) {
            V = ll_load<R>(a, src, in_cplx, base, l, p, k);
        } else if (!staged) {
            // forward DCT-II / DST-II: the point at Makhoul position k
            const int j = ll_makhoul_src(k, n);
            if (kind == PP_KIND_DCT2) {
                V = mkc<C>(ll_load<R>(a, src, in_cplx, base, l, p, j).x, (R)0);
            } else {  // DST-II: x'[j] = (-1)^j x[n-1-j]
                const R v = ll_load<R>(a, src, in_cplx, base, l, p, n - 1 - j).x;
                V = mkc<C>((j & 1) ? -v : v, (R)0);
            }
        } else if (q_odd) {
            if (k < n) {
                const C w = __ldg(&cs[k]);  // e^{-i pi k / (2n)}
                const R x = X(k);
                V = mkc<C>(x * w.x, x * w.y);
            } else {
                V = mkc<C>((R)0, (R)0);
            }
        } else if (quarter) {
            const C w = __ldg(&cs[k]);  // e^{-i pi k / n}
            const R xa = X(2 * k), xb = X(n - 1 - 2 * k);
            V = mkc<C>(xa * w.x - xb * w.y, xa * w.y + xb * w.x);
        } else if (k == 0) {
            V = mkc<C>((R)0.5 * X(0), (R)0);
        } else if (k <= n / 2) {
            const C t = __ldg(&cs[k]);  // (cos t_k, sin t_k)
            const R xk = X(k), xn = X(n - k);
            V.y = (R)0.5 * (t.y * xk - t.x * xn);
            V.x = (R)0.5 * (t.x * xk + t.y * xn);
        } else {
            const int kk = n - k;
            const C t = __ldg(&cs[kk]);
            const R xk = X(kk), xn = X(n - kk);
            V.y = -((R)0.5 * (t.y * xk - t.x * xn));
            V.x = (R)0.5 * (t.x * xk + t.y * xn);
        }
        if (chirp) V = c_mul(V, ll_chirp(chirp, k, back));
        W[ll_w(strided, nl, lw, p, l, k)] = V;
    }
}

// ---- chirp z-transform: the spectrum times the chirp kernel's (same order) ---------
template <typename R>
__global__ void ll_kernel_mul(typename LlVec<R>::type* W, const typename LlVec<R>::type* __restrict__ bhat, long total,
                              int nl, int lw, int strided)
{
    for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < total; idx += (long)gridDim.x * blockDim.x) {
        const int m = strided ? (int)((idx / nl) % lw) : (int)(idx % lw);
        W[idx] = c_mul(W[idx], __ldg(&bhat[m]));
    }
}

// ---- four-step twiddles: point (k1, m2) times W_nf^(k1 m2) (conjugate backward) -------
template <typename R>
__global__ void ll_twiddle_kernel(typename LlVec<R>::type* W, const typename LlVec<R>::type* __restrict__ twl,
                                  long total, int nl, int nf, int n2, int strided, int backward)
{
    using C = typename LlVec<R>::type;
    for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < total; idx += (long)gridDim.x * blockDim.x) {
        // the point's index m within its line
        const int m = strided ? (int)((idx / nl) % nf) : (int)(idx % nf);
        const int k1 = m / n2, m2 = m - k1 * n2;
        if (k1 == 0 || m2 == 0) continue;
        C w = __ldg(&twl[(int)(((long)k1 * m2) % nf)]);
        if (backward) w.y = -w.y;
        W[idx] = c_mul(W[idx], w);
    }
}

// ---- post: one output element per thread -------------------------------------------------
// nf: the transform's FFT length; M > 0: the chirp z-transform's convolution
// length (X natural, times the chirp factor / M), else X at the four-step order
template <typename R>
__global__ void ll_post_kernel(PPLinePassArgs a, const typename LlVec<R>::type* W, int nf, int n1, int n2, int M,
                               const typename LlVec<R>::type* __restrict__ chirp, int back, int inverse, int strided,
                               int out_cplx)
{
    using C = typename LlVec<R>::type;
    const C* cs = sizeof(R) == 8 ? reinterpret_cast<const C*>(a.cs) : reinterpret_cast<const C*>(a.cs2);
    const int n = a.n, kind = a.kind, nl = a.nlines;
    const int lw = M ? M : nf;
    const R inv_m = M ? (R)1 / (R)M : (R)1;
    const bool quarter = pp_kind_is_quarter(kind);
    const bool q_odd = quarter && (n & 1);
    const long total = (long)a.nplanes * nl * n;
    for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < total; idx += (long)gridDim.x * blockDim.x) {
        int p, l, e;
        if (strided) {
            p = (int)(idx / ((long)n * nl));
            const long r = idx - (long)p * n * nl;
            e = (int)(r / nl);
            l = (int)(r - (long)e * nl);
        } else {
            const long g = idx / n;
            e = (int)(idx - g * n);
            p = (int)(g / nl);
            l = (int)(g - (long)p * nl);
        }
        // X[k] of this line: the four-step leaves it at (k mod n1) n2 + k / n1;
        // the chirp z-transform's convolution at k, times the chirp factor / M
        auto Xk = [&](int k) -> C {
            if (M) return c_scale(c_mul(W[ll_w(strided, nl, lw, p, l, k)], ll_chirp(chirp, k, back)), inv_m);
            const int k2 = k / n1;
            return W[ll_w(strided, nl, lw, p, l, (k - k2 * n1) * n2 + k2)];
        };
        C o;
        if (kind == PP_KIND_FFT) {
            o = Xk(e);
        } else if (q_odd) {
            const C w = __ldg(&cs[n + e]);  // e^{-i pi (2e+1)/(4n)}
            const C z = Xk(e);
            R v = z.x * w.x - z.y * w.y;
            v *= inverse ? (R)1 : (R)2;
            if (kind == PP_KIND_DST4 && (e & 1)) v = -v;
            o = mkc<C>(v, (R)0);
        } else if (quarter) {
            const int q = (e & 1) == 0 ? (e >> 1) : ((n - 1 - e) >> 1);
            const C w = __ldg(&cs[nf + q]);  // e^{-i pi (4q+1)/(4n)}
            const C z = Xk(q);
            const R wr = z.x * w.x - z.y * w.y;
            const R wi = z.x * w.y + z.y * w.x;
            R v = ((e & 1) == 0) ? wr : -wi;
            v *= inverse ? (R)1 : (R)2;
            if (kind == PP_KIND_DST4 && (e & 1)) v = -v;
            o = mkc<C>(v, (R)0);
        } else if (!inverse) {
            // DCT-II value at k, optionally through the DST swap
            int k = e;
            R sgn = 1;
            if (kind == PP_KIND_DST2) {
                sgn = (e & 1) ? (R)-1 : (R)1;
                k = n - 1 - e;
            }
            C V;
            if (k > n / 2) {
                V = Xk(n - k);
                V.y = -V.y;
            } else {
                V = Xk(k);
            }
            const C t = __ldg(&cs[k]);
            o = mkc<C>(sgn * ((R)2. * (V.x * t.x + V.y * t.y)), (R)0);
        } else if (kind == PP_KIND_DST2) {
            // DCT-III output reorder through the DST swap
            const int j = n - 1 - e;
            const R s = (e & 1) ? (R)-1 : (R)1;
            o = mkc<C>(s * Xk(ll_makhoul_pos(j, n)).x, (R)0);
        } else {
            o = mkc<C>(Xk(ll_makhoul_pos(e, n)).x, (R)0);
        }
        const long off = (long)p * a.plane_stride + (long)l * a.line_stride + (long)e * a.elem_stride;
        if (a.acc) {
            // u = u_prev + scale * correction + zero-mode constant, in FP64
            const double u = (a.acc_read ? a.acc[off] : 0.0) + a.out_scale * (double)o.x +
                             (a.zplane ? a.zscale * a.zplane[p] : 0.0);
            if (a.dst) reinterpret_cast<double2*>(a.dst)[off] = make_double2(u, 0.0);
            else a.acc[off] = u;
            continue;
        }
        if (a.out_scale != 1.0) {
            o.x = (R)a.out_scale * o.x;
            o.y = (R)a.out_scale * o.y;
        }
        R* dst = reinterpret_cast<R*>(a.dst);
        if (out_cplx) reinterpret_cast<C*>(dst)[off] = o;
        else dst[off] = o.x;
    }
}

unsigned ll_blocks(long total)
{
    const long b = (total + 255) / 256;
    return (unsigned)(b < 148L * 16 ? (b > 0 ? b : 1) : 148L * 16);
}

// lines per tile of a four-step FFT step: the two buffers within 64 KB
int ll_lines(int n, bool fp32)
{
    int L = 16;
    while (L > 1 && pp_line_pass_smem(L, n, fp32) > 64 * 1024) L >>= 1;
    return L;
}

// one four-step step on the generic kernel, in place over W (lines of lw =
// n1 n2 points): A, the n1-point FFTs over the stride-n2 columns; B, the
// n2-point FFTs over the contiguous rows
cudaError_t ll_step(void* W, const PPLongPlan& lp, bool step_a, int nl, int nplanes, bool strided, bool backward,
                    bool fp32, const PPLinePassArgs& a, cudaStream_t st)
{
    const int n1 = lp.n1, n2 = lp.n2, lw = n1 * n2;
    PPLinePassArgs s{};
    s.src = static_cast<const double*>(W);
    s.dst = static_cast<double*>(W);
    s.kind = PP_KIND_FFT;
    s.out_scale = 1.0;
    s.nx = a.nx;
    s.ny = a.ny;
    s.nz = a.nz;
    if (step_a) {
        s.n = n1;
        s.fft = lp.f1;
        s.tw = lp.tw1f;
        s.elem_stride = strided ? (long)n2 * nl : n2;
        s.line_stride = 1;
        s.nlines = strided ? n2 * nl : n2;
        s.nplanes = strided ? nplanes : nplanes * nl;
        s.plane_stride = strided ? (long)lw * nl : lw;
    } else {
        s.n = n2;
        s.fft = lp.f2;
        s.tw = lp.tw2f;
        s.elem_stride = strided ? nl : 1;
        s.line_stride = strided ? 1 : n2;
        s.nlines = strided ? nl : n1;
        s.nplanes = strided ? nplanes * n1 : nplanes * nl;
        s.plane_stride = strided ? (long)n2 * nl : lw;
    }
    s.L = ll_lines(s.n, fp32);
    s.tiles_per_plane = (s.nlines + s.L - 1) / s.L;
    // step A reads lines at a stride (adjacent lines adjacent in memory);
    // step B is contiguous in the line layout, strided in the plane layout
    return pp_launch_line_pass(s, backward, step_a ? true : strided, true, true, st, fp32);
}

template <typename R>
cudaError_t ll_launch(const PPLinePassArgs& a, const PPLongPlan& lp, bool inverse, bool strided, bool in_cplx,
                      bool out_cplx, cudaStream_t st)
{
    using C = typename LlVec<R>::type;
    const bool fp32 = sizeof(R) == 4;
    const int n1 = lp.n1, n2 = lp.n2, lw = n1 * n2, nl = a.nlines;
    const int nf = lp.M ? lp.nf : lw;
    const bool backward = inverse && !pp_kind_is_quarter(a.kind);
    const int back = backward ? 1 : 0;
    C* W = static_cast<C*>(lp.scratch);
    const C* chirp = lp.M ? static_cast<const C*>(fp32 ? lp.chirpf : (const void*)lp.chirp) : nullptr;
    const C* twl = static_cast<const C*>(fp32 ? lp.twlf : (const void*)lp.twl);
    const long total = (long)a.nplanes * nl * lw;
    ll_pre_kernel<R><<<ll_blocks(total), 256, 0, st>>>(a, W, nf, lw, chirp, back, inverse, strided, in_cplx);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    // forward four-step (the transform's own sign, or -1 for the convolution)
    const bool fsign = lp.M ? false : backward;
    if ((e = ll_step(W, lp, true, nl, a.nplanes, strided, fsign, fp32, a, st)) != cudaSuccess) return e;
    ll_twiddle_kernel<R><<<ll_blocks(total), 256, 0, st>>>(W, twl, total, nl, lw, n2, strided, fsign);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if ((e = ll_step(W, lp, false, nl, a.nplanes, strided, fsign, fp32, a, st)) != cudaSuccess) return e;
    if (lp.M) {
        // times the chirp kernel's spectrum, then the inverse four-step in
        // the reverse order of its steps (transposed in, natural out)
        const C* bhat = static_cast<const C*>(fp32 ? lp.bhatf[back] : (const void*)lp.bhat[back]);
        ll_kernel_mul<R><<<ll_blocks(total), 256, 0, st>>>(W, bhat, total, nl, lw, strided);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        if ((e = ll_step(W, lp, false, nl, a.nplanes, strided, true, fp32, a, st)) != cudaSuccess) return e;
        ll_twiddle_kernel<R><<<ll_blocks(total), 256, 0, st>>>(W, twl, total, nl, lw, n2, strided, 1);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        if ((e = ll_step(W, lp, true, nl, a.nplanes, strided, true, fp32, a, st)) != cudaSuccess) return e;
    }
    const long outs = (long)a.nplanes * nl * a.n;
    ll_post_kernel<R><<<ll_blocks(outs), 256, 0, st>>>(a, W, nf, n1, n2, lp.M, chirp, back, inverse, strided, out_cplx);
    return cudaGetLastError();
}

}  // namespace

bool pp_bluestein_split(int nf, int* M, int* n1, int* n2)
{
    long m = 1;
    while (m < 2L * nf - 1) m <<= 1;
    if (m > (1L << 26)) return false;
    *M = (int)m;
    return pp_long_split((int)m, n1, n2);
}

bool pp_long_split(int nf, int* n1, int* n2)
{
    // the divisor pair nearest the square root whose parts both fit one tile
    // of the generic kernel in FP64
    int best = 0;
    for (int d = 2; (long)d * d <= nf; ++d)
        if (nf % d == 0 && pp_line_pass_smem(1, nf / d) <= 227 * 1024) best = d;
    if (!best) return false;
    *n1 = best;
    *n2 = nf / best;
    return true;
}

size_t pp_long_scratch_bytes(long lines, int nf) { return (size_t)lines * nf * sizeof(double2); }

cudaError_t pp_launch_long_line_pass(const PPLinePassArgs& a, const PPLongPlan& lp, bool inverse, bool strided,
                                     bool in_cplx, bool out_cplx, cudaStream_t st, bool fp32)
{
    if (!lp.scratch || lp.n1 < 2 || lp.n2 < 2) return cudaErrorInvalidValue;
    return fp32 ? ll_launch<float>(a, lp, inverse, strided, in_cplx, out_cplx, st)
                : ll_launch<double>(a, lp, inverse, strided, in_cplx, out_cplx, st);
}
