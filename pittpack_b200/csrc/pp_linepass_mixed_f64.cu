// FP64 instances of the register-resident transform pass (pp_lp2.cuh) for the
// lengths 3 2^k and 5 2^k (48 .. 1536): the plain solve (FP32 instances in
// pp_linepass_mixed_f32.cu).  The power-of-two
// factor runs as register passes, the odd factor as one shared-memory pass.
#include "pp_lp2.cuh"

int pp_lpm_lpc(int n) { return pp_lp2::lpm_of(n); }

cudaError_t pp_launch_line_pass_mixed(const PPLinePassArgs& a, bool inverse, bool strided, cudaStream_t st)
{
    if (pp_lp2::lpm_odd9or15(a.n)) return pp_launch_line_pass_mixed915(a, inverse, strided, st);
    return pp_lp2::launch_mixed<double>(a, inverse, strided, st);
}
