/*
 * pittpack_b200.h -- C ABI of the B200 PittPack Poisson solver.
 *
 * Drop-in for the solve path of PittPack's PencilDcmp / PoissonGPU
 * (src/include/pencilDcmp.hpp:442-522).  One handle = one grid on one GPU;
 * the reference's MPI pencil decomposition is not used (single rank, p0 = 1).
 * Every call returns a status code whose values mirror the reference's
 * PittPackResult (src/include/params.h:86-114); no call exits the process.
 * Plain pointers and sizes only.  Paths in the citations are relative to the
 * PittPack source tree.
 *
 * Data layout (chunkedArray, src/chunkedArray.cpp:100-199): point (i,j,k),
 * i = x index fastest, linear index p = i + nx*j + nx*ny*k; the RHS is real
 * (rhs[p]) or complex-interleaved (rhs[2p], rhs[2p+1]); the solution P is
 * complex-interleaved P[2p], P[2p+1], real part = u.
 */
#ifndef PITTPACK_B200_H
#define PITTPACK_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes: 0..23 are the reference's PittPackResult values */
enum {
    PP_SUCCESS = 0,
    PP_GPU_INIT_FAILURE = 1,
    PP_SOLVER_ARRAY_INCONSISTENT = 2,
    PP_MESH_DIVISIBLE = 6,
    PP_ALLOCATION_FAIL = 15,
    PP_THOMAS_FAIL = 18,
    PP_INPUT_ARGS = 19,
    PP_CUFFT_FAIL_X = 20,     /* forward x transform pass failed */
    PP_CUFFT_FAIL_INV_X = 21, /* inverse x transform pass failed */
    PP_CUFFT_FAIL_Y = 22,     /* forward y transform pass failed */
    PP_CUFFT_FAIL_INV_Y = 23, /* inverse y transform pass failed */
    /* codes added by this library */
    PP_INVALID_HANDLE = 24,
    PP_NOT_READY = 25, /* boundary or RHS not assigned yet */
    PP_CUDA_ERROR = 26,
    PP_UNSUPPORTED = 27, /* a size or option the GPU kernels do not cover */
    PP_NOALLOC_TOO_LARGE = 28 /* the grid does not fit pp_solve_noalloc's fixed scratch */
};

/* precision of the solve */
enum { PP_PRECISION_FP64 = 0, PP_PRECISION_MIXED = 1 };
/* z solver of the plain FP64 solve: the direct partition-method / PCR solve
 * (default; the reference's Thomas path, src/pencilDcmp.cpp:5066-5105), or
 * multigrid V-cycles on the same systems (the reference's alternate
 * MultiGrid solver, src/multiGrid.cpp:1105-1515), or one of two parity modes
 * that reproduce the reference's alternates as its CPU build computes them
 * (SOLUTIONMETHOD 1 and 2, src/pencilDcmp.cpp:6102-6148): its normalised PCR
 * (src/pencilDcmp.cpp:5239-5270, src/triDiag.cpp:1442-1542; Dirichlet or
 * Neumann z ends, nz <= 256 and not a power of two; its result is constant
 * along z) and its CR-P (src/pencilDcmp.cpp:5275-5315,
 * src/triDiag.cpp:1285-1437; Dirichlet z ends, nz = 2^L - 1).  Other sizes
 * return PP_UNSUPPORTED from the solve.  Neither alternate solves the
 * reference's own system: they exist to reproduce its outputs. */
enum { PP_ZSOLVE_DIRECT = 0, PP_ZSOLVE_MULTIGRID = 1, PP_ZSOLVE_REF_PCR = 2, PP_ZSOLVE_REF_CRP = 3 };

typedef struct pp_solver_s* pp_handle;

/* launch-shape choices of a handle; 0 in a field = the built-in default.  The
 * reference has no counterpart (cuFFT plans its own launches,
 * src/poissonGPU.cpp:5-97, and its Thomas loop is one OpenACC gang per line,
 * src/pencilDcmp.cpp:5066-5105). */
typedef struct {
    int zsolve_lanes; /* lanes sharing one z system: 1..32, a power of two */
    int line_tile;    /* lines per CTA of the generic transform kernel (lengths other than
                         m 2^k, m = 1, 3, 5, 9, 15), 1..32 */
    int zsolve_tile;  /* z systems (adjacent kx) per CTA of the z solve: 1..32, a power of two */
} pp_tuning;

/* runtime options; the reference keeps these as compile-time switches in
 * src/include/params.h (SOLUTIONMETHOD, NITER, ...) */
typedef struct {
    int precision;        /* PP_PRECISION_FP64 (default) or PP_PRECISION_MIXED: FP32
                             transforms + FP64 iterative refinement of the true
                             7-point system (exact zero mode); real RHS */
    int max_sweeps;       /* refinement sweeps after the first FP32 solve (0..16) */
    double tolerance;     /* target the caller checks; sweeps are a fixed count (no host sync) */
    int compat_zero_mode; /* 1 (default): reference zero-mode row replacement, src/triDiag.cpp:1753-1776 */
    int dirichlet_lift;   /* 1 (default): reference modifyRhsDirichlet, src/pencilDcmp.cpp:4623-4835 */
    int z_solver;         /* PP_ZSOLVE_DIRECT (default), PP_ZSOLVE_MULTIGRID, PP_ZSOLVE_REF_PCR or
                             PP_ZSOLVE_REF_CRP (the last three: plain FP64 solve only) */
    int zero_mean;        /* 0 (default) or 1: subtract the mean of the solution's real part, the
                             reference's ZERO_MEAN (subtractMeanValue, src/pencilDcmp.cpp:5649-5683) */
} pp_options;

/* the reference's PittPackGetErrorEnum (src/pencilDcmp.cpp:4869-4913) */
const char* pp_result_string(int code);

/* make_Poisson / PencilDcmp(argc, argv, nx, ny, nz) (src/pencilDcmp.cpp:232-452,
 * 6432-6440): a solver for an nx*ny*nz grid on the current CUDA device */
int pp_create(int nx, int ny, int nz, pp_handle* h);
/* ~PencilDcmp (src/pencilDcmp.cpp:528-658) */
int pp_destroy(pp_handle h);

/* setBox + setCoords(2) (src/pencilDcmp.cpp:470-480, 748-831):
 * X = {Xa, Xb, Ya, Yb, Za, Zb}; default unit box */
int pp_set_box(pp_handle h, const double X[6]);
/* assignBoundary (src/pencilDcmp.cpp:3578-3634): bc = xmin xmax ymin ymax zmin
 * zmax, letters 'P' 'N' 'D'.  x and y take P-P, N-N, D-D, N-D or D-N; z takes
 * D/N at either end or P-P. */
int pp_assign_boundary(pp_handle h, const char bc[6]);
/* Non-homogeneous boundary data, no counterpart in the reference (whose
 * modifyRhsDirichlet, src/pencilDcmp.cpp:4623-4835, adds only its own
 * manufactured solution): values g on face 'face' (0..5 = xmin, xmax, ymin,
 * ymax, zmin, zmax, the order of the bc string) -- the boundary value on a
 * Dirichlet face, the outward normal derivative on a Neumann face -- at the
 * face's cell centres: x faces g[j + ny k], y faces g[i + nx k], z faces
 * g[i + nx j].  They enter the right-hand side through the ghost-cell
 * relations (Dirichlet u_ghost = 2 g - u_0, Neumann u_ghost = u_0 + h g)
 * with the face's stencil weight ((dz/dx)^2, (dz/dy)^2, 1).  A face with data
 * replaces the manufactured lift of the dirichlet_lift option on that face;
 * g = NULL clears it.  The data are copied.  After pp_assign_boundary
 * (PP_NOT_READY before); a periodic face takes none (PP_INPUT_ARGS). */
int pp_set_face_values(pp_handle h, int face, const double* g);

int pp_default_options(pp_options* opt);
int pp_set_options(pp_handle h, const pp_options* opt);
int pp_get_options(pp_handle h, pp_options* opt);

/* assignRhs (src/pencilDcmp.cpp:5591-5647): real host RHS, nx*ny*nz doubles */
int pp_assign_rhs(pp_handle h, const double* rhs);
/* complex host RHS, 2*nx*ny*nz doubles interleaved */
int pp_assign_rhs_complex(pp_handle h, const double* rhs);
/* RHS already on the device (real or interleaved complex); copied on the
 * handle's stream */
int pp_assign_rhs_device(pp_handle h, const double* d_rhs, int is_complex);
/* real host RHS copied on the handle's stream without waiting: the buffer
 * (page-locked for a truly asynchronous copy) must stay unchanged until the
 * stream has passed the next pp_solve.  No counterpart in the reference. */
int pp_assign_rhs_async(pp_handle h, const double* rhs);
/* zero copy, no counterpart in the reference: later solves read the RHS from
 * d_rhs (real, or interleaved complex if is_complex) and write P to d_P
 * (2*nx*ny*nz doubles), both caller-owned device memory that must outlive
 * the binding; either may be null to keep the handle's own buffer.  A later
 * pp_assign_rhs* call unbinds d_rhs. */
int pp_bind_device_buffers(pp_handle h, const double* d_rhs, int is_complex, double* d_P);

/* pittPack() once (src/pencilDcmp.cpp:5801-6430), asynchronous on the
 * handle's stream */
int pp_solve(pp_handle h);
/* profiling hook, no counterpart in the reference (which times the whole
 * solve with MPI_Wtime, src/pencilDcmp.cpp:5900-6333): one solve with CUDA
 * events around its stages; kernel_ms[0..5] = forward x, forward y, z solve,
 * inverse y, inverse x, residual + zero mode (refined solve only), in
 * milliseconds summed over the sweeps.  Synchronises the handle's stream. */
#define PP_SOLVE_STAGES 6
int pp_profile_solve(pp_handle h, double* kernel_ms, int n);
/* live per-stage timing, no counterpart in the reference: between
 * pp_timing_begin and pp_timing_end the first max_solves calls of pp_solve
 * record CUDA events around their stages on the handle's stream (no extra
 * synchronisation); pp_timing_end waits for the last one and returns the
 * summed milliseconds per stage (PP_SOLVE_STAGES slots, as pp_profile_solve)
 * and the number of solves recorded. */
int pp_timing_begin(pp_handle h, int max_solves);
int pp_timing_end(pp_handle h, double* kernel_ms_total, int n, int* solves);
/* the solution P (2*nx*ny*nz doubles, chunkedArray layout) to host memory;
 * synchronises the handle's stream */
int pp_get_solution(pp_handle h, double* P);
/* the solution to device memory (2*nx*ny*nz doubles), on the handle's stream */
int pp_get_solution_device(pp_handle h, double* d_P);
/* device pointer of the handle's solution buffer (valid until pp_destroy),
 * or of the bound d_P */
int pp_solution_device_ptr(pp_handle h, const double** d_P);
/* the solution to host memory on the handle's stream without waiting (P
 * page-locked for a truly asynchronous copy); no counterpart in the reference */
int pp_get_solution_async(pp_handle h, double* P);
/* the real part of the solution alone, u[i] = P[2 i] (nx*ny*nz doubles, x
 * fastest): half the bytes of P over PCIe, for callers with a real RHS, whose
 * solution's imaginary part is zero (a complex periodic RHS needs the full P).
 * Packed on the device on the handle's stream, then copied; the _async form
 * returns without waiting (u page-locked for a truly asynchronous copy).  No
 * counterpart in the reference, which leaves the complex P in host memory. */
int pp_get_solution_real(pp_handle h, double* u);
int pp_get_solution_real_async(pp_handle h, double* u);
/* PencilDcmp::IO (src/pencilDcmp.cpp:1827-1832): the solution for ParaView /
 * VisIt as soln/Pxdmf3d<app>.xmf, the reference's XDMF file name, with its
 * Collection "AMR" of one Uniform grid "mesh0" and the real part of P as the
 * cell-centred attribute "Q" (Phdf5::writeMultiBlockCellCenter,
 * src/phdf5.cpp:1299-1808).  No HDF5 library is required: Q is a raw
 * little-endian float64 file, soln/Pxdmf3d<app>_Q.bin ([k][j][i], i fastest),
 * referenced as an XDMF Binary data item, and the uniform grid is a
 * 3DCoRectMesh with origin and spacing instead of X/Y/Z node arrays.  One
 * block at one rank: dir and aligndir (0..2), which order the reference's
 * pencil chunks, do not change it.  soln/ is created when absent.  Returns
 * PP_NOT_READY before a solve, PP_INPUT_ARGS when a file cannot be written. */
int pp_io(pp_handle h, unsigned app, int dir, int aligndir);

/* Staged solve of one z-slab of a grid decomposed over several GPUs (the
 * reference's pencil decomposition, src/pencilDcmp.cpp:851-1825, as z slabs:
 * a rank holds planes k0 .. k0 + nz_local - 1).  The handle is created for
 * the slab (pp_create(nx, ny, nz_local)) with the slab's own z extent as its
 * box, the same boundary letters as the whole grid, and pp_set_slab, which
 * says whether the slab owns the grid's z-min / z-max faces (only those take
 * the Dirichlet lift).  Then, for each solve:
 *   pp_stage_forward     x and y transforms of the assigned RHS into the
 *                        slab's spectrum, [k][ky][col] with pp_stage_spectrum's
 *                        col count and doubles per point (2: complex);
 *   (caller)             gather, for its share of spectrum rows ky = j0 ..
 *                        j0 + rows - 1, every slab's planes into one array
 *                        [k][ky - j0][col] (an all-to-all), k over the grid;
 *   pp_stage_zsolve      the z solve of those columns, in place;
 *   (caller)             scatter them back (the reverse all-to-all);
 *   pp_stage_inverse     inverse y and x transforms into the slab's P.
 * All launches go to the handle's stream.  Plain FP64 solve with the direct
 * z solve; pp_solve on a slab handle returns PP_UNSUPPORTED.
 * pittpack_b200/distributed.py does the exchanges with torch.distributed. */
int pp_set_slab(pp_handle h, int owns_zmin, int owns_zmax);
int pp_stage_forward(pp_handle h);
int pp_stage_spectrum(pp_handle h, double** d_spec, int* ncol, int* parts);
int pp_stage_zsolve(pp_handle h, double* d_cols, int nz_total, int rows, int j0);
int pp_stage_inverse(pp_handle h);

/* getError (src/pencilDcmp.cpp:2040-2208): RMS error of the solution against
 * the reference's manufactured solution; does not modify the solution */
int pp_get_error_manufactured(pp_handle h, double* err);
/* fillTrigonometric (src/pencilDcmp.cpp:5685-5759, called by src/main.cpp:115
 * before assignRhs): the reference's analytic RHS f = -4 pi^2 cos(2 pi z) at
 * the cell centres z = Za + (k + 1/2) dz of the handle's box, written to rhs
 * (nx*ny*nz doubles, x fastest).  Host only.  The _box form takes the sizes
 * and box directly and needs neither a handle nor a GPU. */
int pp_fill_trigonometric(pp_handle h, double* rhs);
int pp_fill_trigonometric_box(int nx, int ny, int nz, const double box[6], double* rhs);
/* multigrid z solver: the most V-cycles any system of the last solve took,
 * and how many systems stopped at the cycle bound above 1e-10 relative
 * residual (waits for the handle's stream); no counterpart in the reference,
 * whose MultiGrid prints its residuals (src/multiGrid.cpp:1415-1515) */
int pp_zsolve_stats(pp_handle h, int* max_cycles, int* unconverged);

/* thread blocks of this handle's transform passes whose bounded wait for
 * their bulk-copied tile ran out (each left without output, so the solve is
 * wrong if this is not 0); waits for the handle's stream.  No counterpart in
 * the reference. */
int pp_kernel_timeouts(pp_handle h, int* count);
/* CUDA stream for the handle's work (cudaStream_t passed as void*); 0 = legacy */
int pp_set_stream(pp_handle h, void* stream);
int pp_synchronize(pp_handle h);

/* pinned host buffers for fast copies */
int pp_host_alloc(size_t bytes, void** p);
int pp_host_free(void* p);

/* device memory the handle holds, in bytes */
int pp_workspace_bytes(pp_handle h, size_t* bytes);

/* launch shapes (see pp_tuning); invalid values return PP_INPUT_ARGS */
int pp_set_tuning(pp_handle h, const pp_tuning* t);
int pp_get_tuning(pp_handle h, pp_tuning* t);
/* autotuner, no counterpart in the reference: times 'reps' solves of the
 * assigned RHS for each candidate lane count of the z solve, then each
 * number of z systems per CTA and, when x or y runs the generic transform
 * kernel (lengths other than m 2^k, m = 1, 3, 5, 9, 15), each of its line
 * tiles (one coordinate after the other); keeps the fastest shape in the
 * handle and reports it with its milliseconds per solve.  Synchronises the
 * stream; the handle's solution is overwritten. */
int pp_autotune(pp_handle h, int reps, pp_tuning* chosen, double* best_ms);

/* ---- batched solves (no counterpart in the reference, which solves one grid
 * per PencilDcmp object, src/main.cpp:73-134): many grids of uneven sizes and
 * boundary conditions, each bound zero-copy to caller device buffers, solved
 * by one CUDA-graph launch ----------------------------------------------- */
typedef struct {
    int nx, ny, nz;
    char bc[6];
    double box[6];
    const double* d_rhs; /* device, real, nx*ny*nz doubles */
    double* d_P;         /* device, 2*nx*ny*nz doubles (chunkedArray layout) */
} pp_batch_item;
typedef struct pp_batch_s* pp_batch;
/* builds one handle per grid (options 'opt', or the defaults if null),
 * autotunes each size class once when 'autotune' is set, solves every grid
 * once and captures all solves into one graph whose 'branches' streams run
 * concurrently; on the current device */
int pp_batch_create(const pp_batch_item* items, int n, const pp_options* opt, int branches, int autotune,
                    pp_batch* out);
/* one launch of the captured graph on 'stream' (cudaStream_t as void*) */
int pp_batch_run(pp_batch b, void* stream);
/* number of grids and of graph nodes */
int pp_batch_info(pp_batch b, int* grids, int* graph_nodes);
int pp_batch_destroy(pp_batch b);

/* ---- request server (no counterpart in the reference): single solves
 * arriving over time, continuously batched on the current GPU -------------- */
typedef struct {
    int nx, ny, nz;
    char bc[6];
    double box[6];
    int precision;     /* PP_PRECISION_FP64, or PP_PRECISION_MIXED (refined) */
    int sweeps;        /* refinement sweeps of the mixed mode */
    const double* rhs; /* host, real, nx*ny*nz doubles; page-locked for overlap */
    double* P;         /* host, written when the request completes: 2*nx*ny*nz doubles
                        * (complex P, chunkedArray layout), or nx*ny*nz doubles, the
                        * solution's real part, when output_real is 1 */
    int output_real;   /* 0: complex P; 1: the real part alone (half the copy; the
                        * RHS is real, so the imaginary part is zero) */
} pp_request;
typedef struct pp_server_s* pp_server;
/* 'streams' requests can be on the GPU at once; handles (plans, twiddles and
 * workspaces) are kept per shape within hbm_fraction of the free device
 * memory at creation, idle ones evicted least recently used */
int pp_server_create(int streams, double hbm_fraction, pp_server* out);
/* queue a request (the buffers must stay valid until pp_server_wait returns) */
int pp_server_submit(pp_server s, const pp_request* r, unsigned long long* ticket);
/* wait for a request: its status, latency (submit to solution in host
 * memory, ms) and the precision it ran in */
int pp_server_wait(pp_server s, unsigned long long ticket, double* latency_ms, int* precision);
/* requests completed, most requests on the GPU at once, bytes of pooled handles */
int pp_server_stats(pp_server s, long long* completed, int* max_inflight, size_t* pool_bytes);
/* pooled handles created and evicted so far (each creation allocates device
 * memory, each eviction frees it) */
int pp_server_pool_stats(pp_server s, long long* created, long long* evicted);
/* finishes queued requests, then frees everything */
int pp_server_destroy(pp_server s);

/* pp_solve_noalloc -- no counterpart in the reference.  One plain FP64 solve
 * (the reference's semantics and default options, like pp_solve) that
 * allocates no device memory, for callers that cannot call cudaMalloc: a
 * service whose device memory all belongs to its own pool allocator, a plugin
 * that must not grow the device heap of the process that loads it, any
 * allocation-restricted context that still owns its input and output
 * buffers.  The caller passes device pointers: d_rhs (real RHS, nx*ny*nz
 * doubles, x fastest) and d_P (the solution, 2*nx*ny*nz doubles,
 * chunkedArray layout); 'stream' is a cudaStream_t (0 = legacy).  The tables
 * are computed on the device, nothing is copied from the host, and the call
 * returns once its kernels are enqueued on 'stream'.  The spectra and tables
 * live in one fixed 32 MiB device array inside the library (held by every GPU
 * that loads it until exit): about 16 bytes per point for the real families
 * and 32 bytes per point when x or y is periodic, so up to ~2 M and ~1 M
 * points; larger grids return PP_NOALLOC_TOO_LARGE before anything is
 * launched.  All calls share that array and it keeps the last call's
 * contents (each call writes everything it reads): calls that overlap on the
 * GPU race, so serialise them on one stream.  The first call on a device
 * looks up the array's device address; make it before any stream capture.
 * Like any call that launches work it must not be made from a stream
 * callback (cudaLaunchHostFunc), where CUDA forbids CUDA calls. */
int pp_solve_noalloc(int nx, int ny, int nz, const char bc[6], const double box[6], const double* d_rhs,
                     double* d_P, void* stream);

#ifdef __cplusplus
}
#endif
#endif
