// FP64 instances of the power-of-two transform pass (pp_lp2.cuh): the plain solve.
#include "pp_lp2.cuh"

int pp_lp2_lpc(int n) { return pp_lp2::lpc_of(n); }

template <>
cudaError_t pp_launch_line_pass_pow2<double, double, double>(const PPLinePassArgs& a, bool inverse, bool strided,
                                                             cudaStream_t st)
{
    return pp_lp2::launch<double>(a, inverse, strided, st);
}
