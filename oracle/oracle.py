"""ctypes binding of the CPU oracle (test infrastructure only).

The oracle is a plain-C FP64 restatement of the reference's nhswps hot path
(``oracle/sw_oracle.c``).  Only the tests, ``__graft_entry__.smoke()`` and the
CPU-baseline legs of ``bench.py`` use this module, as the checker or as the
timed CPU baseline; the product package never imports it.

All fields are flat float64 arrays in the reference's Fortran order
(``src/utils.rs:6-32``): physical ``p[iy + ng*ix + ng*ng*iz]``, spectral
``s[kx + ng*ky + ng*ng*iz]``.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")

FIELDS = ["u", "v", "w", "z", "zx", "zy", "r", "ri", "aa", "zeta",
          "pn", "dpn", "ps", "qs", "ds", "gs"]

OK, ERR_FACTORISE, ERR_PSOLVE_DIVERGED, ERR_PSOLVE_MAXITER, ERR_ARG = 0, 1, 3, 4, 6

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_lib = None


def build():
    """Compile the oracle with its Makefile (gcc, OpenMP)."""
    subprocess.check_call(["make", "-s", "-C", HERE])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        L.orc_spectral_new.restype = ctypes.c_void_p
        L.orc_spectral_new.argtypes = [ctypes.c_int, ctypes.c_int]
        L.orc_spectral_free.argtypes = [ctypes.c_void_p]
        L.orc_spectral_get.restype = ctypes.c_long
        L.orc_spectral_get.argtypes = [ctypes.c_void_p, ctypes.c_char_p, _dp]
        for fn in ("orc_ptospc", "orc_spctop", "orc_xderiv", "orc_yderiv", "orc_deal2d",
                   "orc_deal3d", "orc_spec1d"):
            getattr(L, fn).restype = None
        L.orc_num_threads.restype = ctypes.c_int
        L.orc_diagnose.restype = None
        L.orc_energy.restype = None
        _lib = L
    return _lib


def _p(a):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_dp)


def num_threads():
    return lib().orc_num_threads()


def set_num_threads(n):
    lib().orc_set_num_threads(int(n))


def set_fft_order(order):
    """Radix schedule of the oracle's transforms for Spectral objects made after
    this call: 0 (default) radix 4/2/3/5, 1 radix 5/3/2 (rounds differently)."""
    lib().orc_set_fft_order(int(order))


def get_fft_order():
    return lib().orc_get_fft_order()


# ---- stafft --------------------------------------------------------------
def factorisen(n):
    f = (ctypes.c_int * 5)()
    st = lib().orc_factorisen(int(n), f)
    return st, list(f)


def initfft(n):
    f = (ctypes.c_int * 5)()
    trig = np.zeros(2 * n)
    st = lib().orc_initfft(int(n), f, _p(trig))
    if st:
        raise ValueError("factorisation of %d failed" % n)
    return list(f), trig


def forfft(m, n, x):
    x = np.ascontiguousarray(x, dtype=np.float64).copy()
    assert x.size == m * n
    st = lib().orc_forfft(int(m), int(n), _p(x))
    if st:
        raise ValueError("factorisation of %d failed" % n)
    return x


def revfft(m, n, x):
    x = np.ascontiguousarray(x, dtype=np.float64).copy()
    assert x.size == m * n
    st = lib().orc_revfft(int(m), int(n), _p(x))
    if st:
        raise ValueError("factorisation of %d failed" % n)
    return x


# ---- spectral ---------------------------------------------------------------
class Spectral:
    """Oracle counterpart of ``Spectral::new(ng, nz)`` (src/spectral/mod.rs:65)."""

    def __init__(self, ng, nz):
        self.ng, self.nz = ng, nz
        self._h = lib().orc_spectral_new(int(ng), int(nz))
        if not self._h:
            raise ValueError("bad spectral size ng=%d nz=%d" % (ng, nz))

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.orc_spectral_free(self._h)
            self._h = None

    @property
    def n2(self):
        return self.ng * self.ng

    @property
    def n3(self):
        return self.ng * self.ng * (self.nz + 1)

    def get(self, name):
        n = lib().orc_spectral_get(self._h, name.encode(), None)
        if n < 0:
            raise KeyError(name)
        out = np.zeros(n)
        lib().orc_spectral_get(self._h, name.encode(), _p(out))
        return out

    def ptospc(self, rvar):
        out = np.zeros(self.n2)
        lib().orc_ptospc(ctypes.c_void_p(self._h), _p(np.ascontiguousarray(rvar, np.float64)), _p(out))
        return out

    def spctop(self, svar):
        out = np.zeros(self.n2)
        lib().orc_spctop(ctypes.c_void_p(self._h), _p(np.ascontiguousarray(svar, np.float64)), _p(out))
        return out

    def xderiv(self, var):
        out = np.zeros(self.n2)
        lib().orc_xderiv(ctypes.c_void_p(self._h), _p(np.ascontiguousarray(var, np.float64)), _p(out))
        return out

    def yderiv(self, var):
        out = np.zeros(self.n2)
        lib().orc_yderiv(ctypes.c_void_p(self._h), _p(np.ascontiguousarray(var, np.float64)), _p(out))
        return out

    def main_invert(self, qs, ds, gs):
        r, u, v, zeta = (np.zeros(self.n3) for _ in range(4))
        lib().orc_main_invert(ctypes.c_void_p(self._h), _p(_c(qs)), _p(_c(ds)), _p(_c(gs)),
                              _p(r), _p(u), _p(v), _p(zeta))
        return r, u, v, zeta

    def jacob(self, aa, bb):
        cs = np.zeros(self.n2)
        lib().orc_jacob(ctypes.c_void_p(self._h), _p(_c(aa)), _p(_c(bb)), _p(cs))
        return cs

    def divs(self, aa, bb):
        cs = np.zeros(self.n2)
        lib().orc_divs(ctypes.c_void_p(self._h), _p(_c(aa)), _p(_c(bb)), _p(cs))
        return cs

    def ptospc3d(self, fp, fs, izbeg, izend):
        fs = _c(fs).copy()
        lib().orc_ptospc3d(ctypes.c_void_p(self._h), _p(_c(fp)), _p(fs), int(izbeg), int(izend))
        return fs

    def spctop3d(self, fs, fp, izbeg, izend):
        fp = _c(fp).copy()
        lib().orc_spctop3d(ctypes.c_void_p(self._h), _p(_c(fs)), _p(fp), int(izbeg), int(izend))
        return fp

    def deal3d(self, fp):
        fp = _c(fp).copy()
        lib().orc_deal3d(ctypes.c_void_p(self._h), _p(fp))
        return fp

    def deal2d(self, fp):
        fp = _c(fp).copy()
        lib().orc_deal2d(ctypes.c_void_p(self._h), _p(fp))
        return fp

    def spec1d(self, ss):
        spec = np.zeros(self.ng + 1)
        lib().orc_spec1d(ctypes.c_void_p(self._h), _p(_c(ss)), _p(spec))
        return spec


def _c(a):
    return np.ascontiguousarray(a, dtype=np.float64)


# ---- nhswps ---------------------------------------------------------------
class State:
    """The 16 fields of ``nhswps::State`` (src/nhswps/mod.rs:87-148), flat."""

    def __init__(self, ng, nz, fields=None):
        self.ng, self.nz = ng, nz
        n3 = ng * ng * (nz + 1)
        self.f = {k: np.zeros(n3) for k in FIELDS}
        if fields:
            for k, v in fields.items():
                self.f[k] = _c(v).copy().reshape(-1)
                assert self.f[k].size == n3, k
        self.t = 0.0

    def ptrs(self):
        arr = (_dp * len(FIELDS))()
        for i, k in enumerate(FIELDS):
            arr[i] = _p(self.f[k])
        return arr

    def copy(self):
        s = State(self.ng, self.nz, self.f)
        s.t = self.t
        return s


def vertical(sp, st):
    lib().orc_vertical(ctypes.c_void_p(sp._h), st.ptrs())


def coeffs(sp, st):
    out = [np.zeros(sp.n3) for _ in range(4)]
    lib().orc_coeffs(ctypes.c_void_p(sp._h), st.ptrs(), *[_p(o) for o in out])
    return out


def cpsource(sp, st):
    sp0 = np.zeros(sp.n3)
    lib().orc_cpsource(ctypes.c_void_p(sp._h), st.ptrs(), _p(sp0))
    return sp0


def psolve(sp, st, nitmax=100):
    it = ctypes.c_int(0)
    e = ctypes.c_double(0.0)
    status = lib().orc_psolve_ex(ctypes.c_void_p(sp._h), st.ptrs(), int(nitmax), ctypes.byref(it), ctypes.byref(e))
    return status, it.value, e.value


def source(sp, st):
    out = [np.zeros(sp.n3) for _ in range(3)]
    lib().orc_source(ctypes.c_void_p(sp._h), st.ptrs(), *[_p(o) for o in out])
    return out


def diagnose(sp, st):
    out = np.zeros(4)
    lib().orc_diagnose(ctypes.c_void_p(sp._h), st.ptrs(), _p(out))
    return out


def energy(sp, st):
    out = np.zeros(3)
    lib().orc_energy(ctypes.c_void_p(sp._h), st.ptrs(), _p(out))
    return out


def advance(sp, st, ggen=True):
    """One predictor-corrector step (src/nhswps/advance.rs:13-279).
    Returns (status, diagnose values at the start of the step, psolve sweeps)."""
    t = ctypes.c_double(st.t)
    diag = np.zeros(4)
    iters = (ctypes.c_int * 3)()
    status = lib().orc_advance(ctypes.c_void_p(sp._h), st.ptrs(), int(bool(ggen)), ctypes.byref(t), _p(diag), iters)
    st.t = t.value
    return status, diag, list(iters)


# ---- initial conditions -------------------------------------------------------
def vstrip(ng, strip_width=0.4, a2=0.02, a3=-0.01):
    qq = np.zeros(ng * ng)
    lib().orc_vstrip(int(ng), ctypes.c_double(strip_width), ctypes.c_double(a2), ctypes.c_double(a3), _p(qq))
    return qq


def balinit(ng, nz, qq_init):
    qq, dd, gg = np.zeros(ng * ng), np.zeros(ng * ng), np.zeros(ng * ng)
    n = lib().orc_balinit(int(ng), int(nz), _p(_c(qq_init)), _p(qq), _p(dd), _p(gg))
    if n < 0:
        raise ValueError("balinit failed")
    return qq, dd, gg


def initial_state(ng, nz, qq, dd, gg):
    """The nhswps start-up transform (src/nhswps/mod.rs:238-285): ptospc3d of
    the 3-D initial fields, zero (0,0) mode, dealias, then main_invert."""
    sp = Spectral(ng, nz)
    st = State(ng, nz)
    filt = sp.get("filt")
    for name, src in (("qs", qq), ("ds", dd), ("gs", gg)):
        fs = sp.ptospc3d(_c(src), np.zeros(sp.n3), 0, nz)
        fs = fs.reshape(nz + 1, ng * ng)
        fs[:, 0] = 0.0
        fs *= filt[None, :]
        st.f[name] = fs.reshape(-1).copy()
    r, u, v, zeta = sp.main_invert(st.f["qs"], st.f["ds"], st.f["gs"])
    st.f.update(r=r, u=u, v=v, zeta=zeta)
    return sp, st


def swto3d(nz, qq, dd, gg):
    """Replicate 2-D fields over nz+1 levels (src/swto3d.rs:10-39)."""
    return tuple(np.tile(np.asarray(a, np.float64).reshape(-1), nz + 1) for a in (qq, dd, gg))


def _round_half_away(x):
    """Rust's f64::round (half away from zero); Python's round() is half-even."""
    return int(np.floor(abs(x) + 0.5)) * (1 if x >= 0 else -1)


def run_nhswps(ng, nz, dt, tgsave, tsim, qq3d, dd3d, gg3d):
    """The nhswps time loop with its save schedule (src/nhswps/mod.rs:150-345).
    Returns (monitor lines, ecomp lines, psolve sweep counts)."""
    sp, st = initial_state(ng, nz, qq3d, dd3d, gg3d)
    ngsave = _round_half_away(tgsave / dt)
    monitor, ecomp, sweeps = [], [], []

    def save():
        ek, ep, et = energy(sp, st)
        ecomp.append("%.6f %.9f %.9f %.9f %.9f %.9f" % (st.t, 0.0, ek, ek, ep, et))

    while st.t <= tsim:
        itime = _round_half_away(st.t / dt)
        jtime = itime // ngsave
        if ngsave * jtime == itime:
            r, u, v, zeta = sp.main_invert(st.f["qs"], st.f["ds"], st.f["gs"])
            st.f.update(r=r, u=u, v=v, zeta=zeta)
            status, it, _ = psolve(sp, st)
            if status:
                raise RuntimeError("psolve failed with status %d" % status)
            save()
            ggen = False
        else:
            ggen = True
        t = st.t
        status, diag, iters = advance(sp, st, ggen)
        if status:
            raise RuntimeError("advance failed with status %d" % status)
        sweeps.append(iters)
        monitor.append("%.5f %.6f %.6f %.6f %.6f" % (t, diag[0], diag[1], diag[2], diag[3]))
    itime = int(st.t / dt)
    jtime = itime // ngsave
    if ngsave * jtime == itime:
        r, u, v, zeta = sp.main_invert(st.f["qs"], st.f["ds"], st.f["gs"])
        st.f.update(r=r, u=u, v=v, zeta=zeta)
        psolve(sp, st)
        save()
    return monitor, ecomp, sweeps
