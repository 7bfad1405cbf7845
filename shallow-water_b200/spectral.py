"""Spectral operators and transforms on the GPU (reference src/spectral/mod.rs).

``Spectral(ng, nz)`` mirrors ``Spectral::new`` (src/spectral/mod.rs:65-299):
it owns one device context holding the operators and the state fields of an
(ng, nz) grid.  Arrays follow the reference's ndarray layout: shape
``(ng, ng)`` or ``(ng, ng, nz+1)`` indexed ``[x, y, z]`` in Fortran order, i.e.
a physical plane is ``rvar[iy, ix]`` and a spectral plane ``svar[kx, ky]``;
flat float64 arrays in that memory order are accepted too.
"""
import ctypes

import numpy as np

from ._native import FIELD_INDEX, SW_FP64, check, dptr, lib

OPERATORS = ("hlap", "glap", "rlap", "helm", "c2g2", "simp", "rope", "fope", "filt", "diss",
             "opak", "rdis", "ap")
VERTICAL = ("etd1", "htd1", "theta", "weight", "hrkx", "hrky", "rk", "spmf", "alk")


def flat(a):
    """Fortran-order flat float64 copy of an array (any shape)."""
    return np.ascontiguousarray(np.ravel(np.asarray(a, dtype=np.float64), order="F"))


def put(dst, flat_values):
    """Write flat Fortran-order values into dst (ndarray of any shape) in place."""
    if dst is None:
        return
    if dst.ndim == 1:
        dst[...] = flat_values
    else:
        dst[...] = flat_values.reshape(dst.shape, order="F")


class Spectral:
    """GPU counterpart of the reference's ``Spectral`` (one device context)."""

    def __init__(self, ng, nz, precision=SW_FP64, nmembers=1, device=0):
        self.ng, self.nz, self.nmembers, self.precision = int(ng), int(nz), int(nmembers), int(precision)
        h = ctypes.c_void_p()
        check(lib().sw_ctx_create(self.ng, self.nz, self.nmembers, self.precision, int(device), ctypes.byref(h)))
        self._ctx = h
        self._cache = {}

    @classmethod
    def borrowed(cls, ctx, owner):
        """A view of a context that `owner` (an Ensemble) created and destroys."""
        self = cls.__new__(cls)
        ng, nz, nm, pr = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        check(lib().sw_ctx_info(ctx, ctypes.byref(ng), ctypes.byref(nz), ctypes.byref(nm), ctypes.byref(pr)))
        self.ng, self.nz, self.nmembers, self.precision = ng.value, nz.value, nm.value, pr.value
        self._ctx = ctx
        self._cache = {}
        self._owner = owner
        return self

    def close(self):
        if getattr(self, "_owner", None) is not None:
            self._ctx = ctypes.c_void_p()
            return
        if getattr(self, "_ctx", None) and self._ctx.value:
            lib().sw_ctx_destroy(self._ctx)
            self._ctx = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def ctx(self):
        return self._ctx

    def set_fft_chunk(self, planes):
        """Planes per pair of 2-D transform launches (clamped; <= 0 only queries);
        returns the value in use."""
        v = ctypes.c_int()
        check(lib().sw_set_fft_chunk(self._ctx, int(planes), ctypes.byref(v)))
        return v.value

    def set_fft_tile(self, columns):
        """Columns per tile of the n = 256 passes (16 or 32; <= 0 only queries);
        returns the value in use."""
        v = ctypes.c_int()
        check(lib().sw_set_fft_tile(self._ctx, int(columns), ctypes.byref(v)))
        return v.value

    def autotune(self, reps=5, maxc=64):
        """Time the candidate tile widths, transform chunks and the two-stream chunk
        pipeline on this context's grid and keep the fastest.  Returns {"tile":
        columns, "chosen": planes, "overlap": 0/1, "candidates": [(columns, planes,
        overlap, ms), ...]}."""
        tiles = (ctypes.c_int * maxc)()
        chunks = (ctypes.c_int * maxc)()
        ovls = (ctypes.c_int * maxc)()
        ms = (ctypes.c_float * maxc)()
        n, tile, chosen, ovl = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        check(lib().sw_autotune_fft(self._ctx, int(reps), maxc, tiles, chunks, ovls, ms, ctypes.byref(n),
                                    ctypes.byref(tile), ctypes.byref(chosen), ctypes.byref(ovl)))
        return {"tile": tile.value, "chosen": chosen.value, "overlap": ovl.value,
                "candidates": [(tiles[i], chunks[i], ovls[i], float(ms[i])) for i in range(n.value)]}

    @property
    def n2(self):
        return self.ng * self.ng

    @property
    def n3(self):
        return self.ng * self.ng * (self.nz + 1)

    def _get(self, name, n):
        out = np.zeros(n)
        check(lib().sw_spectral_get(self._ctx, name.encode(), dptr(out), n))
        return out

    def __getattr__(self, name):
        if name.startswith("_"):
            raise AttributeError(name)
        ng, nz = self.ng, self.nz
        if name in self._cache:
            return self._cache[name]
        if name in OPERATORS:
            val = self._get(name, ng * ng).reshape((ng, ng), order="F")
        elif name in ("etdv", "htdv"):
            val = self._get(name, ng * ng * nz).reshape((ng, ng, nz), order="F")
        elif name in ("etd1", "htd1"):
            val = self._get(name, nz)
        elif name in ("theta", "weight"):
            val = self._get(name, nz + 1)
        elif name in ("hrkx", "hrky", "rk", "alk"):
            val = self._get(name, ng)
        elif name == "spmf":
            val = self._get(name, ng + 1)
        elif name == "kmag":
            val = self._get(name, ng * ng).astype(np.int64).reshape((ng, ng), order="F")
        elif name in ("kmax", "kmaxred"):
            val = int(self._get(name, 1)[0])
        else:
            raise AttributeError(name)
        self._cache[name] = val
        return val

    # ---- 2-D transforms (src/sta2dfft.rs) ----------------------------------
    def ptospc(self, rvar, svar=None):
        out = np.zeros(self.n2)
        check(lib().sw_ptospc(self._ctx, dptr(flat(rvar)), dptr(out)))
        put(svar, out)
        return out if svar is None else svar

    def spctop(self, svar, rvar=None):
        out = np.zeros(self.n2)
        check(lib().sw_spctop(self._ctx, dptr(flat(svar)), dptr(out)))
        put(rvar, out)
        return out if rvar is None else rvar

    def xderiv(self, var, der=None):
        out = np.zeros(self.n2)
        check(lib().sw_xderiv(self._ctx, dptr(flat(var)), dptr(out)))
        put(der, out)
        return out if der is None else der

    def yderiv(self, var, der=None):
        out = np.zeros(self.n2)
        check(lib().sw_yderiv(self._ctx, dptr(flat(var)), dptr(out)))
        put(der, out)
        return out if der is None else der

    # ---- Spectral methods (src/spectral/mod.rs:305-591) -----------------------
    def main_invert(self, qs, ds, gs, r=None, u=None, v=None, zeta=None):
        """(qs, ds, gs) spectral -> (r, u, v, zeta) physical.  Uses member 0 of
        this context's state storage."""
        L = lib()
        for name, arr in (("qs", qs), ("ds", ds), ("gs", gs)):
            check(L.sw_state_set(self._ctx, FIELD_INDEX[name], 0, dptr(flat(arr)), self.n3))
        check(L.sw_main_invert(self._ctx))
        outs = []
        for name, dst in (("r", r), ("u", u), ("v", v), ("zeta", zeta)):
            o = np.zeros(self.n3)
            check(L.sw_state_get(self._ctx, FIELD_INDEX[name], 0, dptr(o), self.n3))
            put(dst, o)
            outs.append(o if dst is None else dst)
        return tuple(outs)

    def jacob(self, aa, bb, cs=None):
        out = np.zeros(self.n2)
        check(lib().sw_jacob(self._ctx, dptr(flat(aa)), dptr(flat(bb)), dptr(out)))
        put(cs, out)
        return out if cs is None else cs

    def divs(self, aa, bb, cs=None):
        out = np.zeros(self.n2)
        check(lib().sw_divs(self._ctx, dptr(flat(aa)), dptr(flat(bb)), dptr(out)))
        put(cs, out)
        return out if cs is None else cs

    def ptospc3d(self, fp, fs, izbeg, izend):
        out = flat(fs).copy()
        check(lib().sw_ptospc3d(self._ctx, dptr(flat(fp)), dptr(out), int(izbeg), int(izend)))
        if isinstance(fs, np.ndarray) and fs.flags.writeable:
            put(fs, out)
            return fs
        return out

    def spctop3d(self, fs, fp, izbeg, izend):
        out = flat(fp).copy()
        check(lib().sw_spctop3d(self._ctx, dptr(flat(fs)), dptr(out), int(izbeg), int(izend)))
        if isinstance(fp, np.ndarray) and fp.flags.writeable:
            put(fp, out)
            return fp
        return out

    def deal3d(self, fp):
        out = flat(fp).copy()
        check(lib().sw_deal3d(self._ctx, dptr(out)))
        if isinstance(fp, np.ndarray) and fp.flags.writeable:
            put(fp, out)
            return fp
        return out

    def deal2d(self, fp):
        out = flat(fp).copy()
        check(lib().sw_deal2d(self._ctx, dptr(out)))
        if isinstance(fp, np.ndarray) and fp.flags.writeable:
            put(fp, out)
            return fp
        return out

    def spec1d(self, ss, spec=None):
        out = np.zeros(self.ng + 1) if spec is None else np.ascontiguousarray(spec, dtype=np.float64)
        check(lib().sw_spec1d(self._ctx, dptr(flat(ss)), dptr(out)))
        if spec is not None and out is not spec:
            spec[...] = out
            return spec
        return out
