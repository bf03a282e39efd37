// FP64 instances of the register-resident transform pass (pp_lp2.cuh) for the
// lengths 9 2^k (144 .. 1152) and 15 2^k (240 .. 960): the odd factor as one
// shared-memory pass of a Cooley-Tukey DFT-9 (3 x 3) or DFT-15 (5 x 3).
#include "pp_lp2.cuh"

cudaError_t pp_launch_line_pass_mixed915(const PPLinePassArgs& a, bool inverse, bool strided, cudaStream_t st)
{
    return pp_lp2::launch_mixed915<double>(a, inverse, strided, st);
}
