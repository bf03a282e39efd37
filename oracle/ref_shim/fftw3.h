/*
 * Stand-in for the part of FFTW 3.3.x that the PittPack CPU path calls.
 * TEST INFRASTRUCTURE ONLY (oracle/_ref).  FFTW is a third-party library that
 * is not vendored in the PittPack tree; its published definitions are restated
 * in fftw_shim.cpp:
 *   fftw_plan_dft_1d(n, in, out, sign, flags):
 *       out[k] = sum_j in[j] exp(sign * 2 pi i j k / n), unnormalised,
 *       FFTW_FORWARD = -1, FFTW_BACKWARD = +1;
 *   fftw_plan_r2r_1d with REDFT10/REDFT01/RODFT10/RODFT01 (the FFTW manual's
 *       "real even/odd DFTs" section).
 * Two arithmetic modes (environment variable PP_SHIM_FFT): "exact" (default)
 * evaluates the DFT in long double, "fast" uses a double-precision mixed-radix
 * FFT for timing runs.
 */
#ifndef PP_SHIM_FFTW3_H
#define PP_SHIM_FFTW3_H
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef double fftw_complex[2];
typedef struct pp_shim_fftw_plan_s* fftw_plan;
typedef int fftw_r2r_kind;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)

#define FFTW_R2HC 0
#define FFTW_HC2R 1
#define FFTW_DHT 2
#define FFTW_REDFT00 3
#define FFTW_REDFT01 4
#define FFTW_REDFT10 5
#define FFTW_REDFT11 6
#define FFTW_RODFT00 7
#define FFTW_RODFT01 8
#define FFTW_RODFT10 9
#define FFTW_RODFT11 10

void* fftw_malloc(size_t n);
void fftw_free(void* p);
fftw_plan fftw_plan_dft_1d(int n, fftw_complex* in, fftw_complex* out, int sign, unsigned flags);
fftw_plan fftw_plan_r2r_1d(int n, double* in, double* out, fftw_r2r_kind kind, unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);
void fftw_cleanup(void);

#ifdef __cplusplus
}
#endif
#endif
