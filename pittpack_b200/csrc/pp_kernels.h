// Kernel argument blocks and launchers shared by the solver's host code.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>

#include "pp_fft.cuh"

#define PP_LINE_THREADS 256
#define PP_Z_THREADS 256

// Dirichlet face corrections subtracted from the dz^2-scaled RHS
// (modifyRhsDirichlet, src/pencilDcmp.cpp:4623-4835); null where a face is
// not Dirichlet.  z faces are [j][i], x faces [k][j], y faces [k][i].
struct PPLift {
    const double* z0;
    const double* z1;
    const double* x0;
    const double* x1;
    const double* y0;
    const double* y1;
    int any;
};

struct PPLinePassArgs {
    const double* src;
    double* dst;
    int n;             // points along the transformed direction
    int kind;          // PPKind
    int nlines;        // lines per plane
    int nplanes;
    long elem_stride;  // strides in elements (complex elements count once)
    long line_stride;
    long plane_stride;
    // power-of-two kernel only: the tile of lines l0.. starts at
    // plane * plane_stride + l0 * tile_stride (0: l0 * line_stride), and the
    // output may use its own strides (o_*; o_elem_stride = 0: the input's).
    // This lets the y passes write / read the z-tiled spectrum layout.
    long tile_stride;
    long o_elem_stride, o_line_stride, o_plane_stride, o_tile_stride;
    int L;             // lines per CTA tile
    int tiles_per_plane;
    PPFftPlan fft;     // length n, or n/2 for the quarter-wave families
    const double2* cs; // pre/post twiddles of the family (see pp_linepass.cu)
    int rhs_scale;     // forward x-pass: multiply by dz twice and subtract the lift
    double dz;
    PPLift lift;
    int nx, ny, nz;
    double out_scale;  // inverse x-pass: 1 / (nx ny)
    // twiddles in the kernel's precision: used by the power-of-two kernel
    // (pp_linepass_pow2.cu) and by the FP32 generic kernel
    const void* tw;    // FFT twiddles (double2 or float2), length n or n/2
    const void* cs2;   // family twiddles in the kernel's precision
    int in_cplx, out_cplx;
    int vec16;          // power-of-two kernel: src and its run starts are 16-byte aligned
    int half;           // power-of-two periodic x pass of a real RHS on half spectra
                        // (N/2 + 1 complex per line): forward real -> half, inverse half -> real
    // refinement epilogue of the inverse x pass (acc != null): the real part v
    // of each output becomes u = acc + out_scale v + zplane[plane] in FP64;
    // written to acc, or (dst != null) as the final complex-interleaved P
    double* acc;
    const double* zplane;
    double zscale;      // zplane[plane] is multiplied by this
    int acc_read;       // 0: the previous u is zero (first sweep), acc is not read
    // bounded waits (the bulk-copy staging of the contiguous passes): a CTA
    // whose wait runs out adds 1 here (if set) and returns without output
    int* err;
};

// shared memory of the generic kernel: two buffers of L lines of nfft complex
// points in FP64, or in FP32 (fp32)
size_t pp_line_pass_smem(int L, int nfft, bool fp32 = false);

// Lines whose FFT length nf is past one generic-kernel tile (pp_longline.cu):
// the FFT in four steps, nf = n1 n2, through a global scratch array of
// nplanes x nlines x nf complex points; or, where nf has a prime factor past
// one tile, by the chirp z-transform: a cyclic convolution of length
// M = n1 n2 (a power of two >= 2 nf - 1) by two four-step FFTs
struct PPLongPlan {
    int n1, n2;
    PPFftPlan f1, f2;      // plans of n1 and n2 with their FP64 twiddles
    const void* tw1f;      // FP32 twiddles of n1 and n2
    const void* tw2f;
    const double2* twl;    // W_(n1 n2)^j, j < n1 n2, FP64 and FP32
    const void* twlf;
    void* scratch;
    // chirp z-transform (M = n1 n2 > 0): c_k = e^{i pi k^2 / nf}, k < nf, and
    // the FFT of the chirp kernel for the forward and backward transforms, in
    // the four-step output order; FP64 and FP32
    int M;
    int nf;                // the transform's FFT length (n1 n2 without the chirp z-transform)
    const double2* chirp;
    const void* chirpf;
    const double2* bhat[2];
    const void* bhatf[2];
};
// the split nf = n1 n2 (n1 <= n2, nearest the square root, both within one
// generic-kernel tile); false where there is none (a prime beyond that size)
bool pp_long_split(int nf, int* n1, int* n2);
// the chirp z-transform's convolution length for nf (a power of two >= 2 nf - 1)
// and its split; false past the four-step's reach
bool pp_bluestein_split(int nf, int* M, int* n1, int* n2);
size_t pp_long_scratch_bytes(long lines, int nf);
cudaError_t pp_launch_long_line_pass(const PPLinePassArgs& a, const PPLongPlan& lp, bool inverse, bool strided,
                                     bool in_cplx, bool out_cplx, cudaStream_t st, bool fp32);
// power-of-two lengths 16..2048: complex FFT lines per CTA (0 = not covered);
// a tile holds this many data lines for the periodic family and twice as many
// for the real families
int pp_lp2_lpc(int n);
template <typename Real, typename TI, typename TO>
cudaError_t pp_launch_line_pass_pow2(const PPLinePassArgs& a, bool inverse, bool strided, cudaStream_t st);
// the same kernel for the lengths 3 2^k (48 .. 1536), 5 2^k (80 .. 1280),
// 9 2^k (144 .. 1152) and 15 2^k (240 .. 960):
// complex FFT lines per CTA (0 = not covered), and the FP64 / FP32 launches
int pp_lpm_lpc(int n);
cudaError_t pp_launch_line_pass_mixed(const PPLinePassArgs& a, bool inverse, bool strided, cudaStream_t st);
cudaError_t pp_launch_line_pass_mixed_f32(const PPLinePassArgs& a, bool inverse, bool strided, cudaStream_t st);
// 9 2^k and 15 2^k (144 .. 1152), called by the two above
cudaError_t pp_launch_line_pass_mixed915(const PPLinePassArgs& a, bool inverse, bool strided, cudaStream_t st);
cudaError_t pp_launch_line_pass_mixed915_f32(const PPLinePassArgs& a, bool inverse, bool strided, cudaStream_t st);
// every other length (pp_fft_plan); fp32: the FP32 kernel, twiddles from a.tw and
// a.cs2 (FP64: a.fft.tw and a.cs), with the refinement epilogue when a.acc is set
cudaError_t pp_launch_line_pass(const PPLinePassArgs& a, bool inverse, bool strided, bool in_cplx, bool out_cplx,
                                cudaStream_t st, bool fp32 = false);

// z-boundary kinds of the tridiagonal systems
enum PPZBc : int { PP_Z_DIRICHLET = 0, PP_Z_NEUMANN = 1, PP_Z_PERIODIC = 2 };

struct PPZArgs {
    double* data;       // spectrum [k][ky][kx], real or complex
    int nx, ny, nz;
    int TS;             // systems (adjacent kx) per CTA
    int tiles_x;
    const double* ax;   // -2 + 2 cos((kx + num) f / (nx + den)), per kx
    const double* ay;   // same per ky
    double Cx, Cy;      // (dz/dx)^2, (dz/dy)^2
    int zlo, zhi;       // PPZBc of the two z ends
    int pin_always;     // 1: zero-mode row replacement whatever the z ends (reference)
    int P;              // lanes per system (0: the default for nz)
    int data_fp32;      // spectrum stored as float / float2 (solved in FP64)
    int skip_zero;      // write zeros for the kx = ky = 0 column
    int tiled;          // spectrum in the z-tiled layout: tile (ky, kx / TS) is the
                        // contiguous block [k][kx % TS] at (ky (nx / TS) + kx / TS) nz TS
    int* err;           // counts CTAs whose bounded waits ran out (may be null)
};

// lanes that share one z system (a power of two <= 32)
int pp_zsolve_lanes(int nz, bool cplx, bool large = false);
// grids of at least this many z systems (kx x ky columns) keep uneven row
// counts in registers too (the register capacity path of the z solve)
#define PP_Z_LARGE_SYSTEMS 65536L
bool pp_zsolve_large(long systems);
// systems per CTA and threads per CTA of the z solve
void pp_zsolve_config(int nz, bool cplx, int nx, int* TS, int* threads);
// the same for a chosen lane count (0 or invalid: the default); the launch
// must then carry P = that lane count
void pp_zsolve_config_p(int nz, bool cplx, int nx, int lanes, int* TS, int* threads, int systems = 0, int ny = 0);
int pp_zsolve_valid_lanes(int nz, int P);
size_t pp_zsolve_smem_p(int TS, int nz, bool cplx, int P);
// the longest z systems the z solve takes: a CTA of one system on 32 lanes
// whose column, pivot table and scratch fit the opt-in shared memory of a
// CTA (cplx: complex spectra; g32: the refined solve's FP32 spectra, staged
// beside the tile); about 25,000 rows for real spectra, 13,000 for complex
int pp_zsolve_max_nz(bool cplx, bool g32);

// FP64 residual r = f dz^2 - lift - A u of the refined solve (pp_mixed.cu)
struct PPResidArgs {
    const double* f;   // real RHS, unscaled
    const double* u;   // current solution (real), or null for u = 0
    float* r;          // FP32 residual out
    double* part;      // FP64 sums of r per (plane, xy tile): [nz][pp_resid_tiles], or null
    int nx, ny, nz;
    double dz, Cx, Cy;
    int bc[6];         // face codes: 0 Dirichlet, 1 Neumann, 2 periodic
    PPLift lift;
    double* upart;     // FP64 sums of u, same layout, or null
};
// xy tiles per plane of the residual kernel (the partial sums' row length)
int pp_resid_tiles(int nx, int ny);
cudaError_t pp_launch_resid(const PPResidArgs& a, cudaStream_t st);
// The kx = ky = 0 column of a refined sweep from per-CTA partial sums
// ([plane][tpp] each), added in a fixed order (one block per plane):
// zcol[k] = scale * sum_t part[k tpp + t]; if upart is set, uplane[k] = the
// plane's sum of upart and *usum = the sum of uplane (nz doubles of scratch).
cudaError_t pp_launch_zero_mode_sums(const double* part, const double* upart, int tpp, int nz, double scale,
                                     double* zcol, double* usum, double* uplane, cudaStream_t st);
// zero-mean solution (pp_mean.cu): the mean of the real parts of the n
// complex-interleaved values of P is subtracted from them; scratch holds
// pp_zero_mean_scratch_doubles() doubles
size_t pp_zero_mean_scratch_doubles();
cudaError_t pp_launch_zero_mean(double* P, long n, double* scratch, cudaStream_t st);
// u[i] = P[2 i] for the n complex-interleaved values of P (P 16-byte aligned)
cudaError_t pp_launch_real_part(const double* P, double* u, long n, cudaStream_t st);
// Singular problems: keep the null-space constant of the refined solution at
// the value implied by the pinned FP64 zero-mode solve of b (see pp_mixed.cu).
cudaError_t pp_launch_zero_mode_anchor(double* zcol, int nz, const double* usum, double* mstar, double zscale,
                                       double npts, int first, cudaStream_t st);
cudaError_t pp_launch_zsolve(const PPZArgs& a, bool cplx, cudaStream_t st);

// alternate z solve by multigrid V-cycles (pp_zsolve_mg.cu): the same systems
// as pp_launch_zsolve, FP64 spectra
struct PPZMgArgs {
    double* data;       // spectrum [k][ky][kx], real or complex
    int nx, ny, nz;
    const double* ax;
    const double* ay;
    double Cx, Cy;
    int zlo, zhi;
    int pin_always;
    int max_cycles;     // bound on V-cycles per system
    int* stats;         // [0] max cycles used, [1] systems stopped at the bound; or null
    int G;              // systems per CTA (set by the launcher)
    int tot;            // cells of all levels (set by the launcher)
};
int pp_zsolve_mg_levels_total(int nz);
size_t pp_zsolve_mg_smem(int G, int nz, bool cplx);
// cudaErrorInvalidValue when one system's levels do not fit shared memory
cudaError_t pp_launch_zsolve_mg(PPZMgArgs a, bool cplx, cudaStream_t st);

// the reference's alternate z solvers as its CPU build computes them
// (pp_zsolve_ref.cu): method PP_ZSOLVE_REF_PCR or PP_ZSOLVE_REF_CRP on the
// [k][ky][kx] spectrum (parts = 2: complex-interleaved), in place
struct PPZRefArgs {
    double* data;
    int nx, ny, nz;   // spectrum columns, rows, planes
    int parts;
    const double* ax;
    const double* ay;
    double Cx, Cy;
    int zlo, zhi;     // PP_Z_DIRICHLET / PP_Z_NEUMANN / PP_Z_PERIODIC
    int method;
};
bool pp_zsolve_ref_defined(int method, int nz, int zlo, int zhi);
cudaError_t pp_launch_zsolve_ref(const PPZRefArgs& a, cudaStream_t st);
