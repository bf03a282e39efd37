// Zero-mean solution: the reference's ZERO_MEAN switch (subtractMeanValue,
// src/pencilDcmp.cpp:5649-5683, called after the solve at
// src/pencilDcmp.cpp:6404-6407) subtracts the mean of the real part of P over
// the grid from it.  Three small kernels: fixed-size partial sums, one block
// adding them up in a fixed order (the same bits on every run), and the
// subtraction.
#include "pp_common.cuh"
#include "pp_kernels.h"

namespace {

constexpr int MEAN_BLOCKS = 1184;  // 8 per SM
constexpr int MEAN_THREADS = 256;

__global__ void __launch_bounds__(MEAN_THREADS) mean_partial_kernel(const double* __restrict__ P, long n,
                                                                   double* __restrict__ part)
{
    double s = 0.0;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        s += P[2 * i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    __shared__ double w[MEAN_THREADS / 32];
    if ((threadIdx.x & 31) == 0) w[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int q = 0; q < MEAN_THREADS / 32; ++q) t += w[q];
        part[blockIdx.x] = t;
    }
}

__global__ void __launch_bounds__(MEAN_THREADS) mean_total_kernel(const double* __restrict__ part, int np, long n,
                                                                 double* __restrict__ mean)
{
    __shared__ double red[MEAN_THREADS];
    double s = 0.0;
    for (int i = threadIdx.x; i < np; i += blockDim.x) s += part[i];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = MEAN_THREADS / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) *mean = red[0] / (double)n;
}

__global__ void __launch_bounds__(MEAN_THREADS) mean_subtract_kernel(double* __restrict__ P, long n,
                                                                    const double* __restrict__ mean)
{
    const double m = *mean;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        P[2 * i] -= m;
}

}  // namespace

size_t pp_zero_mean_scratch_doubles() { return (size_t)MEAN_BLOCKS + 1; }

cudaError_t pp_launch_zero_mean(double* P, long n, double* scratch, cudaStream_t st)
{
    mean_partial_kernel<<<MEAN_BLOCKS, MEAN_THREADS, 0, st>>>(P, n, scratch);
    mean_total_kernel<<<1, MEAN_THREADS, 0, st>>>(scratch, MEAN_BLOCKS, n, scratch + MEAN_BLOCKS);
    mean_subtract_kernel<<<MEAN_BLOCKS, MEAN_THREADS, 0, st>>>(P, n, scratch + MEAN_BLOCKS);
    return cudaGetLastError();
}

// The real part of a complex-interleaved solution, packed: u[i] = P[2 i]
// (16-byte loads, 8-byte stores), for callers that want u alone.
namespace {
__global__ void __launch_bounds__(256) real_part_kernel(const double2* __restrict__ P, double* __restrict__ u, long n)
{
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        u[i] = P[i].x;
}
}  // namespace

cudaError_t pp_launch_real_part(const double* P, double* u, long n, cudaStream_t st)
{
    real_part_kernel<<<MEAN_BLOCKS, 256, 0, st>>>(reinterpret_cast<const double2*>(P), u, n);
    return cudaGetLastError();
}

