/*
 * Compile-time switches for the single-rank reference build (oracle/_ref).
 * TEST INFRASTRUCTURE ONLY.
 *
 * The PittPack tree keeps its configuration as macros and enumerators in
 * src/include/params.h.  This header is force-included (-include) ahead of
 * every reference source and claims that header's include guard, so the
 * reference compiles against these values instead.  Every name and value is
 * the shipped one except three switches, changed so that pittPack() solves a
 * caller-supplied RHS once and writes no run report:
 *   INITANALYTIC 1 -> 0   (src/pencilDcmp.cpp:5874-5880 would overwrite the RHS)
 *   NITER       10 -> 1
 *   RUNINFO      1 -> 0
 * SOLUTIONMETHOD (z-solver: 0 Thomas, 1 PCR, 2 CR-P) can be chosen with
 * -DPP_REF_SOLUTIONMETHOD=<n>, and ZERO_MEAN (subtract the mean of the
 * solution's real part after the solve) with -DPP_REF_ZERO_MEAN=1; the
 * defaults are the shipped 0.
 */
#ifndef _PARAMS_H_
#define _PARAMS_H_

#ifndef PP_REF_SOLUTIONMETHOD
#define PP_REF_SOLUTIONMETHOD 0
#endif
#ifndef PP_REF_ZERO_MEAN
#define PP_REF_ZERO_MEAN 0
#endif

#define PITTPACKACC _OPENACC
#define EXACT 0
#define DEBUG2 0
#define DEBUG_COMM 0
#define DEBUG1 0
#define DEBUG0 0
#define DEBUG 0
#define COMM_PATTERN 2
#define SHORT_ 0
#define ZSIZE 64
#define MULTIGRIDON 0
#define NXCHUNK1 256
#define NYCHUNK1 256
#define TMPSIZE 256
#define COMM_ON 1
#define DISABLE_CHECKS 1
#define MIN(x, y) (((x) < (y)) ? (x) : (y))

enum PittPackParams {
    I_O = 0,
    SHIFT = 1,
    This = 0,
    GPUAW = 1,
    GPUAW2 = 1,
    MPI_ERROR_DISABLE = 0,
    PITT_ABORT = 0,
    INCLUDE_ERROE_CAL_IN_TIMING = 0,
    SOLUTIONMETHOD = PP_REF_SOLUTIONMETHOD,
    INITANALYTIC = 0,
    PIVOT = 1,
    INNERITER = 10,
    OUTERITER = 20,
    TRI_NUM_GANG = 10000,
    VECLENGTH = 256,
    MAXLEVEL = 20,
    COEFF0 = 1,
    COEFF1 = 2,
    COEFF2 = 3,
    AMPL0 = 0,
    AMPL1 = 0,
    AMPL2 = 0,
    CUFFT_STREAMS = 0,
    MONITOR_MEM = 0,
    PROFILE_COMM = 0,
    NITER = 1,
    RUNINFO = 0,
    ZERO_MEAN = PP_REF_ZERO_MEAN,
};

struct PittPackInputStruct {
    int nxChunk;
    int nychunk;
    int nzChunk;
    char bc[6];
    int IO;
    int sol_method;
};
extern PittPackInputStruct PittPackIn;

typedef enum PittPackErrorCodes {
    SUCCESS = 0,
    GPU_INIT_FAILURE = 1,
    SOLVER_ARRAY_INCONSISTENT = 2,
    MPI_INIT_FAIL = 3,
    MPI_DUP_FAIL = 4,
    COMSIZE_FAIL = 5,
    MESH_DIVISIBLE = 6,
    MPI_GET_RANK_FAIL = 7,
    MPI_COMSIZE_FAIL = 8,
    MPI_DIST_GTAPH_FAIL_X = 9,
    MPI_DIST_GTAPH_FAIL_Y = 10,
    GRAPH_CREATE_FAIL = 11,
    MPI_INEIGHBOR_FAIL_ZX = 12,
    MPI_INEIGHBOR_FAIL_XY = 13,
    BLOCK_NUMBER_FAIL = 14,
    ALLOCATION_FAIL = 15,
    MPI_FINALIZE_FAIL = 16,
    MPI_ERROR_HANDLE_FAIL = 16,
    CONNECTIVITY_CONSTRUCTION_FAIL = 17,
    THOMAS_FAIL = 18,
    INPUT_ARGS = 19,
    CUFFT_FAIL_X = 20,
    CUFFT_FAIL_INV_X = 21,
    CUFFT_FAIL_Y = 22,
    CUFFT_FAIL_INV_Y = 23,
} PittPackResult;

const double pi = 3.1415926535897932384;

#define POSS 1
#define SOLVE 1
#define IFFTX 1
#define IFFTY 1
#define FFTX 1
#define FFTY 1
#define USE_SHARED 0
#define REVTRSP 1
#define R_COPY 1
#define THOM_FULL_BATCH 0
#define JIC 0

PittPackResult OPENACC_Init(int& my_rank, int& com_size);
PittPackResult HostToDeviceAssign(int& my_rank, int& com_size);
const char* PittPackGetErrorEnum(PittPackResult error);

#endif
