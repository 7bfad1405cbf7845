"""Mixed-radix real FFTs (reference src/stafft/mod.rs) on the GPU.

``forfft(m, n, x, trig, factors)`` transforms, in place, the m vectors of
length n held as x[i + m*j] (x of shape (m, n) in Fortran order, or flat),
like the reference.  ``trig`` and ``factors`` come from ``initfft`` and are
checked against n; the GPU keeps its own twiddle tables.
"""
import ctypes

import numpy as np

from ._native import check, dptr, lib


def factorisen(n):
    """Greedy 6/4/2/3/5 factorisation (src/stafft/mod.rs:97-150)."""
    f = (ctypes.c_int * 5)()
    check(lib().sw_factorisen(int(n), f))
    return list(f)


def initfft(n):
    """(factors, trig) for length n (src/stafft/mod.rs:67-95)."""
    f = (ctypes.c_int * 5)()
    trig = np.zeros(2 * n)
    check(lib().sw_initfft(int(n), f, dptr(trig)))
    return list(f), trig


def _run(fn, m, n, x, trig, factors):
    a = np.ascontiguousarray(np.ravel(np.asarray(x, dtype=np.float64), order="F"))
    if a.size != m * n:
        raise ValueError("x must hold m*n values")
    fac = None if factors is None else (ctypes.c_int * 5)(*factors)
    tp = None if trig is None else dptr(np.ascontiguousarray(trig, dtype=np.float64))
    check(fn(int(m), int(n), dptr(a), tp, fac))
    if isinstance(x, np.ndarray) and x.dtype == np.float64 and x.flags.writeable:
        x[...] = a.reshape(x.shape, order="F") if x.ndim > 1 else a
        return x
    return a


def forfft(m, n, x, trig=None, factors=None):
    """Forward transform to Hermitian form (src/stafft/mod.rs:158-293)."""
    return _run(lib().sw_forfft, m, n, x, trig, factors)


def revfft(m, n, x, trig=None, factors=None):
    """Reverse transform from Hermitian form (src/stafft/mod.rs:301-452)."""
    return _run(lib().sw_revfft, m, n, x, trig, factors)
