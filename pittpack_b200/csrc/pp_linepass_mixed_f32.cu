// FP32 instances of the register-resident transform pass (pp_lp2.cuh) for the
// lengths 3 2^k and 5 2^k: the correction solves of the refined mode.
#include "pp_lp2.cuh"

cudaError_t pp_launch_line_pass_mixed_f32(const PPLinePassArgs& a, bool inverse, bool strided, cudaStream_t st)
{
    if (pp_lp2::lpm_odd9or15(a.n)) return pp_launch_line_pass_mixed915_f32(a, inverse, strided, st);
    return pp_lp2::launch_mixed<float>(a, inverse, strided, st);
}
