"""Balanced 2-D initial fields (reference src/balinit.rs:21-435).

The fixed-point iteration of the reference runs on the device (sw_balinit):
transforms, derivatives, products, filters and the scalar sums stay in device
memory, and the host reads two numbers per iteration for the stop test.
"""
import ctypes
import os

import numpy as np

from ._native import check, dptr, lib
from .spectral import Spectral


def balance(ng, nz, qq_init, spectral=None):
    """(qq, dd, gg) balanced fields from the PV strip qq_init (flat, Fortran order):
    the reference's fixed-point iteration run on the device by sw_balinit, on a
    float64 context of the grid (or `spectral`, which must be float64)."""
    sp = spectral if spectral is not None else Spectral(ng, nz)
    n2 = ng * ng
    q0 = np.ascontiguousarray(np.asarray(qq_init, dtype=np.float64).reshape(-1))
    if q0.size != n2:
        raise ValueError("qq_init needs %d values" % n2)
    qq, dd, gg = np.zeros(n2), np.zeros(n2), np.zeros(n2)
    it = ctypes.c_int()
    check(lib().sw_balinit(sp.ctx, dptr(q0), dptr(qq), dptr(dd), dptr(gg), ctypes.byref(it)))
    return qq, dd, gg


def balinit(parameters):
    """Read qq_init.r8, write sw_init.r8 = 3 x (header + ng*ng) (balinit.rs:423-435)."""
    num = parameters.numerical
    ng, nz = num.grid_resolution, num.vertical_layers
    d = str(parameters.environment.output_directory)
    qq0 = np.fromfile(os.path.join(d, "qq_init.r8"), dtype="<f8")[1:]
    qq, dd, gg = balance(ng, nz, qq0)
    np.concatenate([[0.0], qq, [0.0], dd, [0.0], gg]).astype("<f8").tofile(os.path.join(d, "sw_init.r8"))
