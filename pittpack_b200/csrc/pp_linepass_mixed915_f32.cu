// FP32 instances of the register-resident transform pass (pp_lp2.cuh) for the
// lengths 9 2^k and 15 2^k: the correction solves of the refined mode.
#include "pp_lp2.cuh"

cudaError_t pp_launch_line_pass_mixed915_f32(const PPLinePassArgs& a, bool inverse, bool strided, cudaStream_t st)
{
    return pp_lp2::launch_mixed915<float>(a, inverse, strided, st);
}
