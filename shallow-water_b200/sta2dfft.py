"""2-D transforms and spectral derivatives (reference src/sta2dfft.rs)."""
import numpy as np

from .spectral import Spectral
from . import stafft


class D2FFT:
    """``D2FFT::new(nx, ny, lx, ly, kx, ky)`` (src/sta2dfft.rs:37-85) for the
    square doubly periodic grids of nhswps (nx == ny, lx == ly == 2 pi)."""

    def __init__(self, nx, ny, lx=2.0 * np.pi, ly=2.0 * np.pi, nz=2, spectral=None):
        if nx != ny or lx != ly:
            raise ValueError("only square domains are supported (nhswps uses ng x ng, 2 pi x 2 pi)")
        if lx == 0.0:
            raise ValueError("Wavenumber array definition not possible, domain length in x equal to zero not allowed!")
        self.nx, self.ny = nx, ny
        self.xfactors, self.xtrig = stafft.initfft(nx)
        self.yfactors, self.ytrig = stafft.initfft(ny)
        sc = np.pi / lx
        self.kx = sc * np.arange(1, nx + 1, dtype=np.float64)
        self.ky = sc * np.arange(1, ny + 1, dtype=np.float64)
        if abs(lx - 2.0 * np.pi) > 1e-15:
            raise ValueError("the GPU derivatives assume lx = ly = 2 pi")
        self._sp = spectral if spectral is not None else Spectral(nx, nz)

    def ptospc(self, rvar, svar):
        return self._sp.ptospc(rvar, svar)

    def spctop(self, svar, rvar):
        return self._sp.spctop(svar, rvar)

    def _check_k(self, rk, own, axis):
        # The GPU derivative multiplies by the integer wavenumber of each mode, which
        # is the reference's rk array (pi / l) * k on the 2 pi domain; another array
        # would silently give another derivative, so it is refused.
        rk = np.asarray(rk, dtype=np.float64).ravel()
        if rk.shape != own.shape or np.abs(rk - own).max() > 1e-12 * np.abs(own).max():
            raise ValueError("D2FFT.%sderiv: only the domain's own wavenumbers (D2FFT.k%s) are supported" % (axis, axis))

    def xderiv(self, rkx, var, der):
        """x derivative of a spectral field (src/sta2dfft.rs:128-152)."""
        self._check_k(rkx, self.kx, "x")
        return self._sp.xderiv(var, der)

    def yderiv(self, rky, var, der):
        """y derivative of a spectral field (src/sta2dfft.rs:157-184)."""
        self._check_k(rky, self.ky, "y")
        return self._sp.yderiv(var, der)
