// FP32 instances of the power-of-two transform pass (pp_lp2.cuh): the
// correction solves of the refined mixed-precision mode.
#include "pp_lp2.cuh"

template <>
cudaError_t pp_launch_line_pass_pow2<float, float, float>(const PPLinePassArgs& a, bool inverse, bool strided,
                                                          cudaStream_t st)
{
    return pp_lp2::launch<float>(a, inverse, strided, st);
}
