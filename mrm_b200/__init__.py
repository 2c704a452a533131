"""mrm_b200: B200-native per-timestep grain dynamics of the mrm recording model.

The hot path (stochastic LLG Heun integrator + effective-field assembly +
demag FFT convolution with the FP64 tensor) lives in the CUDA library
mrm_b200/libmrm_gpu.so behind the C ABI of include/mrm_gpu.h.  This package
only marshals arrays into that ABI; it has no CPU fallback.
"""
from . import _lib
from ._lib import FP32, FP64, OPEN, PERIODIC, MrmError, STATS_DTYPE
from .llg import GpuSim, geom_of

__all__ = ["GpuSim", "geom_of", "FP32", "FP64", "OPEN", "PERIODIC", "MrmError", "STATS_DTYPE",
           "load_library"]


def load_library():
    """Loads libmrm_gpu.so (raises ImportError if it has not been built)."""
    return _lib.load()
