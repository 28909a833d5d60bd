"""pimdal_b200: PIMDAL's data-parallel operator layer on one B200 (sm_100a).

Hand-written CUDA kernels behind the C ABI of include/pimdal_gpu.h
(libpimdal_b200.so), with a thin Python host layer (ops.py) over ctypes.
"""
from . import _lib
from ._lib import PimdalError, lib, LIB_PATH

__all__ = ["PimdalError", "lib", "LIB_PATH", "_lib"]
