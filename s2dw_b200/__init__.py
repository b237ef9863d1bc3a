"""s2dw_b200: the S2DW directional scale-discretised wavelet transform on the
sphere (analysis flm -> wav, synthesis wav -> flm) on NVIDIA B200 (sm_100a).

The compute path is libs2dw_cuda.so (hand-written CUDA, C ABI in
include/s2dw_cuda.h).  `core` mirrors the reference's Fortran module
s2dw_core_mod on host arrays; `device.Plan` runs on CUDA tensors.
"""
from ._lib import LIB_PATH, S2DWError, lib  # noqa: F401
from .core import *  # noqa: F401,F403

__version__ = "0.1.0"
