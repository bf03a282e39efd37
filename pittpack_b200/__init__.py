"""B200-native PittPack FFT-FFT-tridiagonal Poisson solver.

The compute path is libpittpack_b200.so (hand-written CUDA for sm_100a behind
a C ABI, include/pittpack_b200.h); this package is the host-side mirror of the
reference's PencilDcmp/PoissonGPU interface.
"""
from ._lib import Options, PittPackError, result_string  # noqa: F401
from .poisson import PoissonGPU, make_Poisson  # noqa: F401

__all__ = ["PoissonGPU", "make_Poisson", "Options", "PittPackError", "result_string"]
