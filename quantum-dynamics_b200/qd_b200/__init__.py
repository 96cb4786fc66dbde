"""B200 split-operator wavepacket propagator (Python host mirror of the C ABI).

    from qd_b200 import systems, TimeEvolutionMexCUDA
    data = systems.case_c0()          # the Matlab-struct equivalent
    TimeEvolutionMexCUDA(data)        # propagates in place on the GPU
    print(data.CRP.CRP)               # P(E)

The propagation itself runs only in libqd.so (hand-written sm_100a CUDA);
there is no CPU path.
"""
from . import systems
from ._abi import QdError, QD_PREC_FP32, QD_PREC_FP64
from .timeevolution import (TimeEvolutionMexCUDA, TimeEvolutionMex, Propagator,
                            legendre_matrix_gpu, read_grids, kernel_launch_count)

__all__ = ["systems", "QdError", "QD_PREC_FP32", "QD_PREC_FP64", "TimeEvolutionMexCUDA",
           "TimeEvolutionMex", "Propagator", "legendre_matrix_gpu", "read_grids",
           "kernel_launch_count"]
