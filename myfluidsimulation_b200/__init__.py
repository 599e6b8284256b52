"""B200-native D3Q19 lattice-Boltzmann path of FluidSimExtended.

Hand-written sm_100a CUDA kernels (liblbm_b200.so) behind the C-ABI of
include/lbm_capi.h: Legacy BGK and Hybrid(B0) in an in-place AA pattern, the
moment-only HOME update, halfway bounce-back on a voxelized STL mask, FP64
statistics (mass, energy, momentum-exchange drag), and a GPU voxelizer.
"""
from ._lib import LBMError, lib  # noqa: F401
from .solvers import (BC_DUCT, BC_PERIODIC, BOUNCE_HALFWAY, BOUNCE_REFERENCE, METHOD_HOME, METHOD_HYBRID, METHOD_LEGACY, STORE_BF16, STORE_F64,  # noqa: F401
                      STORE_F16, STORE_F32, Domain, LBM3D_Home, LBM3D_Hybrid, LBM3D_Legacy, Solver)

__version__ = "0.1.0"
