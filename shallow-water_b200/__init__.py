"""B200 (sm_100a) implementation of the nhswps time-step path of
rse-standrewscs/shallow-water behind the reference's API names.

Modules mirror the reference crate (src/lib.rs:4-15): ``stafft``, ``sta2dfft``,
``spectral``, ``nhswps``, ``parameters``, ``vstrip``, ``balinit``, ``swto3d``.
All numerics of the time step run in libswcuda.so (CUDA, sm_100a) through the
C ABI of include/sw_cuda.h; there is no CPU fallback.
"""
from . import _native
from ._native import SW_FP64, SW_MIXED, SW_FP32, SwError
from . import stafft, sta2dfft, spectral, nhswps, parameters, vstrip, balinit, swto3d
from .spectral import Spectral
from .nhswps import State, Output, advance, psolve, source, cpsource, coeffs, vertical, savegrid

__all__ = ["SW_FP64", "SW_MIXED", "SW_FP32", "SwError", "Spectral", "State", "Output", "advance", "psolve",
           "source", "cpsource", "coeffs", "vertical", "savegrid", "stafft", "sta2dfft", "spectral",
           "nhswps", "parameters", "vstrip", "balinit", "swto3d"]
