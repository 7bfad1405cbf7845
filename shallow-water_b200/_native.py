"""ctypes binding of libswcuda.so (the C ABI of include/sw_cuda.h).

Loading never falls back to anything else: if the library is missing or a
call fails, an exception is raised.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# SW_CUDA_LIB_VARIANT=bc loads the bounds-check debug build (libswcuda_bc.so,
# `python shallow-water_b200/build.py --bounds-check`) instead of the library
LIB_PATH = os.path.join(HERE, "libswcuda_bc.so" if os.environ.get("SW_CUDA_LIB_VARIANT") == "bc" else "libswcuda.so")
HEADER = os.path.join(HERE, "..", "include", "sw_cuda.h")

SW_OK, SW_ERR_FACTORISE, SW_ERR_CUDA = 0, 1, 2
SW_ERR_PSOLVE_DIVERGED, SW_ERR_PSOLVE_MAXITER, SW_ERR_ARG, SW_ERR_STATE = 3, 4, 6, 7
SW_FP64, SW_MIXED, SW_FP32 = 0, 1, 2
FIELDS = ["u", "v", "w", "z", "zx", "zy", "r", "ri", "aa", "zeta",
          "pn", "dpn", "ps", "qs", "ds", "gs"]
FIELD_INDEX = {k: i for i, k in enumerate(FIELDS)}

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_vp = ctypes.c_void_p
_sz = ctypes.c_size_t
_i = ctypes.c_int

# name -> (restype, argtypes)
_SIGS = {
    "sw_last_error": (ctypes.c_char_p, []),
    "sw_version": (_i, []),
    "sw_factorisen": (_i, [_i, _ip]),
    "sw_initfft": (_i, [_i, _ip, _dp]),
    "sw_forfft": (_i, [_i, _i, _dp, _dp, _ip]),
    "sw_revfft": (_i, [_i, _i, _dp, _dp, _ip]),
    "sw_forfft_dev": (_i, [_i, _i, _vp, _i, _vp]),
    "sw_revfft_dev": (_i, [_i, _i, _vp, _i, _vp]),
    "sw_ctx_create": (_i, [_i, _i, _i, _i, _i, ctypes.POINTER(_vp)]),
    "sw_ctx_destroy": (None, [_vp]),
    "sw_ctx_info": (_i, [_vp, _ip, _ip, _ip, _ip]),
    "sw_spectral_get": (_i, [_vp, ctypes.c_char_p, _dp, _sz]),
    "sw_state_set": (_i, [_vp, _i, _i, _dp, _sz]),
    "sw_state_get": (_i, [_vp, _i, _i, _dp, _sz]),
    "sw_state_set_all": (_i, [_vp, _i, _dp, _sz]),
    "sw_state_get_all": (_i, [_vp, _i, _dp, _sz]),
    "sw_set_time": (_i, [_vp, ctypes.c_double]),
    "sw_get_time": (_i, [_vp, _dp]),
    "sw_ptospc": (_i, [_vp, _dp, _dp]),
    "sw_spctop": (_i, [_vp, _dp, _dp]),
    "sw_xderiv": (_i, [_vp, _dp, _dp]),
    "sw_yderiv": (_i, [_vp, _dp, _dp]),
    "sw_jacob": (_i, [_vp, _dp, _dp, _dp]),
    "sw_divs": (_i, [_vp, _dp, _dp, _dp]),
    "sw_deal2d": (_i, [_vp, _dp]),
    "sw_deal3d": (_i, [_vp, _dp]),
    "sw_ptospc3d": (_i, [_vp, _dp, _dp, _i, _i]),
    "sw_spctop3d": (_i, [_vp, _dp, _dp, _i, _i]),
    "sw_spec1d": (_i, [_vp, _dp, _dp]),
    "sw_balinit": (_i, [_vp, _dp, _dp, _dp, _dp, _ip]),
    "sw_main_invert": (_i, [_vp]),
    "sw_vertical": (_i, [_vp]),
    "sw_coeffs": (_i, [_vp, _dp, _dp, _dp, _dp]),
    "sw_cpsource": (_i, [_vp, _dp]),
    "sw_psolve": (_i, [_vp, _i, _ip, _dp]),
    "sw_source": (_i, [_vp, _dp, _dp, _dp]),
    "sw_advance": (_i, [_vp, _i, _i]),
    "sw_set_graphs": (_i, [_vp, _i]),
    "sw_set_fft_chunk": (_i, [_vp, _i, _ip]),
    "sw_set_psolve_toler": (_i, [_vp, ctypes.c_double]),
    "sw_set_psolve_relax": (_i, [_vp, ctypes.c_double]),
    "sw_sweep_counts": (_i, [_vp, ctypes.POINTER(ctypes.c_longlong)]),
    "sw_advance_async": (_i, [_vp, _i, _i]),
    "sw_savegrid": (_i, [_vp, _i, _dp, _dp, _i, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float)]),
    "sw_state_set_all_async": (_i, [_vp, _i, _dp, _sz]),
    "sw_state_get_all_async": (_i, [_vp, _i, _dp, _sz]),
    "sw_tridiag_batched": (_i, [_i, _i, _vp, _vp, _vp, _vp, _vp, _vp]),
    "sw_tridiag_batched_host": (_i, [_i, _i, _dp, _dp, _dp, _dp, _dp]),
    "sw_autotune_fft": (_i, [_vp, _i, _i, _ip, _ip, _ip, ctypes.POINTER(ctypes.c_float), _ip, _ip, _ip, _ip]),
    "sw_set_fft_tile": (_i, [_vp, _i, _ip]),
    "sw_set_fft_single_pass": (_i, [_vp, _i, _ip]),
    "sw_set_fft_overlap": (_i, [_vp, _i, _ip]),
    "sw_diagnose": (_i, [_vp, _i, _dp]),
    "sw_diag_history": (_i, [_vp, _dp, _i, _ip]),
    "sw_energy": (_i, [_vp, _i, _dp]),
    "sw_last_sweeps": (_i, [_vp, _ip]),
    "sw_sync": (_i, [_vp]),
    "sw_field_device_ptr": (_i, [_vp, _i, ctypes.POINTER(_vp), _ip]),
    "sw_stream": (_i, [_vp, ctypes.POINTER(_vp)]),
    "sw_fft2d_dev": (_i, [_vp, _i, _i, _vp, _vp]),
    "sw_fft2d_noalloc": (_i, [_i, _i, _i, _vp, _vp, _vp]),
    "sw_kernel_launches": (_i, [_vp, ctypes.POINTER(ctypes.c_longlong)]),
    "sw_ensemble_create": (_i, [_ip, _ip, _i, _i, _i, ctypes.POINTER(_vp)]),
    "sw_ensemble_destroy": (None, [_vp]),
    "sw_ensemble_info": (_i, [_vp, _ip, _ip]),
    "sw_ensemble_stream": (_i, [_vp, ctypes.POINTER(_vp)]),
    "sw_ensemble_member": (_i, [_vp, _i, ctypes.POINTER(_vp), _ip]),
    "sw_ensemble_advance": (_i, [_vp, _i, _i]),
    "sw_ensemble_advance_async": (_i, [_vp, _i, _i]),
    "sw_ensemble_sync": (_i, [_vp]),
}

_lib = None


class SwError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__("shallow-water CUDA error %d: %s" % (status, msg))
        self.status = status


def declared_symbols():
    """Entry points declared in include/sw_cuda.h."""
    import re
    text = open(HEADER).read()
    return sorted(set(re.findall(r"\b(sw_[a-z0-9_]+)\s*\(", text)))


def lib():
    """Load libswcuda.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise OSError("%s not built: run python shallow-water_b200/build.py" % os.path.basename(LIB_PATH))
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(status):
    if status != SW_OK:
        msg = lib().sw_last_error()
        raise SwError(status, msg.decode() if msg else "")
    return status


def dptr(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"], "need a contiguous float64 array"
    return a.ctypes.data_as(_dp)
