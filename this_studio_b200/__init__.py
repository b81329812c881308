"""B200-native DEMSPH particle-interaction path.

The compute path is the native library libdemsph_b200.so (hand-written
sm_100a CUDA kernels behind the C ABI in include/demsph.h).  This package
mirrors the reference's DEMSolver / WCSPHSolver classes over that ABI.
"""
from ._lib import DemsphError, kernel_launches, lib
from .solvers import DEMSolver, DEMSPHCoupling, WCSPHSolver, num_steps

__all__ = ["DEMSolver", "DEMSPHCoupling", "WCSPHSolver", "DemsphError", "kernel_launches", "lib", "num_steps"]
