"""Balanced 2-D initial fields (reference src/balinit.rs:21-435).

The fixed-point iteration of the reference, with every transform, derivative,
Jacobian and divergence done on the GPU through ``Spectral`` and the pointwise
work on host arrays (it runs once, before the time loop).
"""
import os

import numpy as np

from .spectral import Spectral

COF = 4.0 * np.pi


def balance(ng, nz, qq_init, spectral=None):
    """(qq, dd, gg) balanced fields from the PV strip qq_init (flat, Fortran order)."""
    sp = spectral if spectral is not None else Spectral(ng, nz)
    n2 = ng * ng
    toler, small, dsumi = 1.0e-9, 1.0e-12, 1.0 / (ng * ng)
    F = lambda a: np.ravel(a, order="F")
    filt, rlap, opak, helm, c2g2 = (F(getattr(sp, k)) for k in ("filt", "rlap", "opak", "helm", "c2g2"))
    qq = np.array(qq_init, dtype=np.float64)
    zz = qq.copy()
    dd = np.zeros(n2)
    gg = np.zeros(n2)
    qq += -dsumi * qq.sum()
    qbar = dsumi * qq.sum()
    wkb = sp.ptospc(COF * qq)
    hh = sp.spctop(filt * wkb / (opak - COF * qbar))
    htot = 1.0 + hh
    qq += -dsumi * (htot * qq).sum()
    zz = htot * (COF + qq) - COF
    wkb = sp.ptospc(zz)
    wka = rlap * wkb
    zz = sp.spctop(wkb * filt)
    wkd = sp.xderiv(wka)
    uu = sp.spctop(-sp.yderiv(wka))
    vv = sp.spctop(wkd)
    uu += -(hh * uu).sum() * dsumi
    toterrpre = 1.0 / small ** 2
    toterr = 0.5
    ddpre, ggpre = dd.copy(), gg.copy()
    while toterr > toler:
        wkb = sp.jacob(uu, vv)
        wka = sp.divs(dd * uu, dd * vv)
        gs = filt * (wka - 2.0 * wkb)
        gg = sp.spctop(gs)
        ggrmserr = ((gg - ggpre) ** 2).sum() / ((ggpre ** 2).sum() + small)
        wka = sp.divs(hh * uu, hh * vv)
        wkb = sp.divs(zz * uu, zz * vv)
        ds = helm * (COF * wkb - c2g2 * wka)
        dd = sp.spctop(ds)
        ddrmserr = ((dd - ddpre) ** 2).sum() / ((ddpre ** 2).sum() + small)
        htot = 1.0 + hh
        qq += -dsumi * (qq * htot).sum()
        qbar = dsumi * qq.sum()
        wkb = sp.ptospc(COF * (qq + hh * (qq - qbar)) - gg)
        hh = sp.spctop(filt * wkb / (opak - COF * qbar))
        htot = 1.0 + hh
        qq += -dsumi * (qq * htot).sum()
        zz = htot * (COF + qq) - COF
        wkb = sp.ptospc(zz)
        wka = rlap * wkb
        zz = sp.spctop(wkb * filt)
        wkd = sp.xderiv(wka)
        wkb = sp.yderiv(wka)
        wke = rlap * ds
        wka = sp.xderiv(wke)
        wkc = sp.yderiv(wke)
        uu = sp.spctop(wka - wkb)
        vv = sp.spctop(wkd + wkc)
        uu += -(hh * uu).sum() * dsumi
        vv += -(hh * vv).sum() * dsumi
        toterr = 0.5 * (ddrmserr + ggrmserr)
        if toterrpre <= toterr:
            break
        ddpre, ggpre = dd.copy(), gg.copy()
        toterrpre = toterr
    return zz - COF * hh, dd, gg


def balinit(parameters):
    """Read qq_init.r8, write sw_init.r8 = 3 x (header + ng*ng) (balinit.rs:423-435)."""
    num = parameters.numerical
    ng, nz = num.grid_resolution, num.vertical_layers
    d = str(parameters.environment.output_directory)
    qq0 = np.fromfile(os.path.join(d, "qq_init.r8"), dtype="<f8")[1:]
    qq, dd, gg = balance(ng, nz, qq0)
    np.concatenate([[0.0], qq, [0.0], dd, [0.0], gg]).astype("<f8").tofile(os.path.join(d, "sw_init.r8"))
