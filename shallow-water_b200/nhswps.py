"""The nhswps time-step path on the GPU (reference src/nhswps/).

``State`` mirrors ``nhswps::State`` (src/nhswps/mod.rs:87-148).  Its 16 fields
live on the device inside the ``Spectral`` context; reading ``state.u`` copies
the field to a numpy array of shape (ng, ng, nz+1) (Fortran order) and
assigning uploads.  The numerical entry points keep the reference's names and
argument meaning; where the reference quits the process on a numerical failure
(psolve.rs:349-366) these raise ``SwError`` with the same status.
"""
import ctypes
import os

import numpy as np

from ._native import FIELDS, FIELD_INDEX, SW_FP64 as SW_FP64_DEFAULT, SwError, check, dptr, lib
from .spectral import Spectral, flat, put

HBAR = 0.4
COF = 4.0 * np.pi
CSQ = (2.0 * np.pi) ** 2


class State:
    """Device-resident ``nhswps::State`` of one member (member 0 of the context)."""

    def __init__(self, spectral, t=0.0, ngsave=0, itime=0, jtime=0, ggen=False, member=0, **fields):
        object.__setattr__(self, "spectral", spectral)
        object.__setattr__(self, "member", member)
        object.__setattr__(self, "ngsave", ngsave)
        object.__setattr__(self, "itime", itime)
        object.__setattr__(self, "jtime", jtime)
        object.__setattr__(self, "ggen", ggen)
        check(lib().sw_set_time(spectral.ctx, float(t)))
        for k, v in fields.items():
            setattr(self, k, v)

    @property
    def t(self):
        t = ctypes.c_double()
        check(lib().sw_get_time(self.spectral.ctx, ctypes.byref(t)))
        return t.value

    @t.setter
    def t(self, value):
        check(lib().sw_set_time(self.spectral.ctx, float(value)))

    def get(self, name):
        sp = self.spectral
        out = np.zeros(sp.n3)
        check(lib().sw_state_get(sp.ctx, FIELD_INDEX[name], self.member, dptr(out), sp.n3))
        return out.reshape((sp.ng, sp.ng, sp.nz + 1), order="F")

    def set(self, name, value):
        sp = self.spectral
        a = flat(value)
        if a.size != sp.n3:
            raise ValueError("%s needs %d values" % (name, sp.n3))
        check(lib().sw_state_set(sp.ctx, FIELD_INDEX[name], self.member, dptr(a), sp.n3))

    def __getattr__(self, name):
        if name in FIELD_INDEX:
            return self.get(name)
        raise AttributeError(name)

    def __setattr__(self, name, value):
        if name in FIELD_INDEX:
            self.set(name, value)
        elif name == "t":
            State.t.fset(self, value)
        else:
            object.__setattr__(self, name, value)

    def fields(self):
        return {k: self.get(k) for k in FIELDS}


def _n3(state):
    return state.spectral.n3


def vertical(state):
    """z, zx, zy, aa, w from r, u, v, ds (src/nhswps/vertical.rs:8-143)."""
    check(lib().sw_vertical(state.spectral.ctx))


def coeffs(state, sigx=None, sigy=None, cpt1=None, cpt2=None):
    """Pressure-iteration coefficients (src/nhswps/coeffs.rs:8-101)."""
    n = _n3(state)
    outs = [np.zeros(n) for _ in range(4)]
    check(lib().sw_coeffs(state.spectral.ctx, *[dptr(o) for o in outs]))
    for dst, o in zip((sigx, sigy, cpt1, cpt2), outs):
        put(dst, o)
    return outs


def cpsource(state, sp0=None):
    """Constant part of the pressure source (src/nhswps/cpsource.rs:13-261)."""
    out = np.zeros(_n3(state))
    check(lib().sw_cpsource(state.spectral.ctx, dptr(out)))
    put(sp0, out)
    return out


def psolve(state, nitmax=100):
    """Non-hydrostatic pressure (src/nhswps/psolve.rs:16-411).
    Returns (sweeps, final relative change)."""
    it = ctypes.c_int()
    e = ctypes.c_double()
    check(lib().sw_psolve(state.spectral.ctx, int(nitmax), ctypes.byref(it), ctypes.byref(e)))
    return it.value, e.value


def tridiag_batched(a, b, c, d):
    """Solve nsys tridiagonal systems of n <= 33 unknowns in float64 on the GPU
    (the vertical Thomas solve of psolve.rs:285-327 for general coefficients).
    Arrays have shape (n, nsys), system index contiguous:
    a[i] x[i-1] + b[i] x[i] + c[i] x[i+1] = d[i].  Returns x, shape (n, nsys)."""
    arrs = [np.ascontiguousarray(np.asarray(v, dtype=np.float64)) for v in (a, b, c, d)]
    n, nsys = arrs[0].shape
    for v in arrs:
        if v.shape != (n, nsys):
            raise ValueError("a, b, c, d need the same (n, nsys) shape")
    x = np.zeros((n, nsys))
    check(lib().sw_tridiag_batched_host(n, nsys, *[dptr(v) for v in arrs], dptr(x)))
    return x


def source(state, sqs=None, sds=None, sgs=None):
    """Nonlinear source terms in spectral space (src/nhswps/source.rs:19-138)."""
    n = _n3(state)
    outs = [np.zeros(n) for _ in range(3)]
    check(lib().sw_source(state.spectral.ctx, *[dptr(o) for o in outs]))
    for dst, o in zip((sqs, sds, sgs), outs):
        put(dst, o)
    return outs


def diagnose(state):
    """(0.5*zrms^2, zrms, zmax, umax) of the current state (src/nhswps/mod.rs:666-711)."""
    out = np.zeros(4)
    check(lib().sw_diagnose(state.spectral.ctx, state.member, dptr(out)))
    return out


def energy(state):
    """(ekin, epot, etot) as computed by savegrid (src/nhswps/mod.rs:365-410)."""
    out = np.zeros(3)
    check(lib().sw_energy(state.spectral.ctx, state.member, dptr(out)))
    return out


def diag_history(spectral, cap=4096):
    """Diagnostics recorded at the start of each advance step since the last call."""
    out = np.zeros((cap, 4))
    cnt = ctypes.c_int()
    check(lib().sw_diag_history(spectral.ctx, dptr(out), cap, ctypes.byref(cnt)))
    return out[: cnt.value]


def advance(state, output=None, nsteps=1):
    """Predictor-corrector step(s) t -> t + dt (src/nhswps/advance.rs:13-279).
    Writes the monitor.asc line of each step to ``output`` when given."""
    t0 = state.t
    check(lib().sw_advance(state.spectral.ctx, int(nsteps), int(bool(state.ggen))))
    if output is not None:
        rows = diag_history(state.spectral)
        dt = 1.0 / state.spectral.ng
        for k, d in enumerate(rows[-nsteps:]):
            output.monitor.write("%.5f %.6f %.6f %.6f %.6f\n" % (t0 + k * dt, d[0], d[1], d[2], d[3]))
    return state


def advance_async(spectral, nsteps=1, ggen=True):
    """Queue nsteps graph-captured steps of every member of the context without
    waiting (see sync); contexts on different streams run concurrently."""
    check(lib().sw_advance_async(spectral.ctx, int(nsteps), int(bool(ggen))))


def sync(spectral):
    """Wait for the context's queued work; raises if a pressure solve failed."""
    check(lib().sw_sync(spectral.ctx))


def last_sweeps(spectral):
    out = (ctypes.c_int * 3)()
    check(lib().sw_last_sweeps(spectral.ctx, out))
    return list(out)


# ---- run driver and output (src/nhswps/mod.rs:32-85, 150-663) -----------------------
class Output:
    """The 14 output files of nhswps (src/nhswps/mod.rs:32-85).  The float32
    snapshot records of savegrid are appended by one background writer thread in
    submission order (`flush()`/`close()` wait for it), so the time loop does not
    wait for file I/O."""

    NAMES = {
        "ecomp": "ecomp.asc", "monitor": "monitor.asc", "spectra": "spectra.asc",
        "d3ql": "3d/ql.r4", "d3d": "3d/d.r4", "d3g": "3d/g.r4", "d3r": "3d/r.r4", "d3w": "3d/w.r4",
        "d3pn": "3d/pn.r4", "d2q": "2d/q.r4", "d2d": "2d/d.r4", "d2g": "2d/g.r4", "d2h": "2d/h.r4",
        "d2zeta": "2d/zeta.r4",
    }

    def __init__(self, files):
        self.__dict__.update(files)
        self._pool = None
        self._pending = []

    @classmethod
    def from_path(cls, path):
        os.makedirs(os.path.join(path, "2d"), exist_ok=True)
        os.makedirs(os.path.join(path, "3d"), exist_ok=True)
        files = {}
        for k, rel in cls.NAMES.items():
            files[k] = open(os.path.join(path, rel), "w" if rel.endswith(".asc") else "wb")
        return cls(files)

    def submit(self, fn, *args):
        """Run fn(*args) on the writer thread (in order)."""
        if self._pool is None:
            from concurrent.futures import ThreadPoolExecutor
            self._pool = ThreadPoolExecutor(max_workers=1)
        self._pending.append(self._pool.submit(fn, *args))

    def flush(self):
        for f in self._pending:
            f.result()
        self._pending = []

    def close(self):
        self.flush()
        if self._pool is not None:
            self._pool.shutdown()
            self._pool = None
        for k in self.NAMES:
            getattr(self, k).close()


def _append_r4(f, t, data):
    f.write(np.float32(t).astype("<f4").tobytes())
    f.write(np.asarray(data, dtype="<f4").reshape(-1, order="F").tobytes(order="F"))


def savegrid_data(state):
    """savegrid's numbers computed on the device in one call (sw_savegrid):
    (energies[3], spectra (3, kmax+1), fields3 {name: float32 flat}, fields2
    {name: float32 flat})."""
    sp = state.spectral
    n2, n3 = sp.n2, sp.n3
    nb = sp.kmax + 1
    energies = np.zeros(3)
    spectra = np.zeros(3 * nb)
    f3 = np.zeros(6 * n3, dtype=np.float32)
    f2 = np.zeros(5 * n2, dtype=np.float32)
    fp = ctypes.POINTER(ctypes.c_float)
    check(lib().sw_savegrid(sp.ctx, state.member, dptr(energies), dptr(spectra), 3 * nb,
                            f3.ctypes.data_as(fp), f2.ctypes.data_as(fp)))
    names3 = ("qs", "ds", "gs", "r", "w", "pn")
    names2 = ("d", "zeta", "q", "g", "h")
    return (energies, spectra.reshape(3, nb), {k: f3[i * n3:(i + 1) * n3] for i, k in enumerate(names3)},
            {k: f2[i * n2:(i + 1) * n2] for i, k in enumerate(names2)})


def _write_records(output, t, f3, f2):
    for key, name in (("d3ql", "qs"), ("d3d", "ds"), ("d3g", "gs"), ("d3r", "r"), ("d3w", "w"), ("d3pn", "pn")):
        _append_r4(getattr(output, key), t, f3[name])
    for key, name in (("d2d", "d"), ("d2zeta", "zeta"), ("d2q", "q"), ("d2g", "g"), ("d2h", "h")):
        _append_r4(getattr(output, key), t, f2[name])


def savegrid(state, output):
    """Energies, spectra and f32 snapshots at a save time (src/nhswps/mod.rs:347-663).
    The numbers come from the device in one call; the text lines are written here
    and the binary records by the output's writer thread."""
    sp = state.spectral
    t = state.t
    (ekin, epot, etot), spec, f3, f2 = savegrid_data(state)
    output.ecomp.write("%.6f %.9f %.9f %.9f %.9f %.9f\n" % (t, 0.0, ekin, ekin, epot, etot))
    zspec, dspec, gspec = spec
    output.spectra.write("%.6f %d\n" % (t, sp.kmaxred))
    alk = sp.alk
    with np.errstate(divide="ignore"):
        for k in range(1, sp.kmaxred + 1):
            output.spectra.write("%.8f %.8f %.8f %.8f\n" % (alk[k - 1], np.log10(zspec[k]),
                                                          np.log10(dspec[k] + 1.0e-32), np.log10(gspec[k] + 1.0e-32)))
    if hasattr(output, "submit"):
        output.submit(_write_records, output, t, f3, f2)
    else:
        _write_records(output, t, f3, f2)


def _round_half_away(x):
    """Rust's f64::round (half away from zero)."""
    return int(np.floor(abs(x) + 0.5)) * (1 if x >= 0 else -1)


def initial_state(spectral, qq, dd, gg, member=0, invert=True):
    """The start-up of nhswps (src/nhswps/mod.rs:238-285): physical initial
    fields (ng*ng*(nz+1) each) -> filtered spectral qs, ds, gs with zero mean,
    then main_invert.  For an ensemble context, load each member with
    invert=False and call main_invert once (it acts on all members)."""
    sp = spectral
    ng, nz = sp.ng, sp.nz
    st = State(sp, member=member)
    filt = flat(sp.filt)
    for name, src in (("qs", qq), ("ds", dd), ("gs", gg)):
        fs = sp.ptospc3d(flat(src), np.zeros(sp.n3), 0, nz).reshape(nz + 1, ng * ng)
        fs[:, 0] = 0.0
        fs *= filt[None, :]
        st.set(name, fs.reshape(-1))
    if invert:
        check(lib().sw_main_invert(sp.ctx))
    return st


def main_invert_all(spectral):
    """main_invert for every member of the context (src/spectral/mod.rs:305-417)."""
    check(lib().sw_main_invert(spectral.ctx))


class Ensemble:
    """Members with uneven grids advanced together (sw_ensemble_*): member k has
    grid ngs[k] x ngs[k] x (nzs[k] + 1).  Members of one (ng, nz) share a batched
    context; one step of every member is one CUDA graph launch whose branches are
    the groups' steps.  ``state(k)`` is member k's State (fields read and written
    through its context)."""

    def __init__(self, ngs, nzs, precision=SW_FP64_DEFAULT, device=0):
        ngs = (ctypes.c_int * len(ngs))(*[int(v) for v in ngs])
        nzs = (ctypes.c_int * len(nzs))(*[int(v) for v in nzs])
        h = ctypes.c_void_p()
        check(lib().sw_ensemble_create(ngs, nzs, len(ngs), int(precision), int(device), ctypes.byref(h)))
        self._h = h
        self.nmembers = len(ngs)
        self._spectral = {}

    def member(self, k):
        """(Spectral of the member's context, the member's index in it)."""
        c, i = ctypes.c_void_p(), ctypes.c_int()
        check(lib().sw_ensemble_member(self._h, int(k), ctypes.byref(c), ctypes.byref(i)))
        if c.value not in self._spectral:
            self._spectral[c.value] = Spectral.borrowed(c, self)
        return self._spectral[c.value], i.value

    def state(self, k):
        sp, i = self.member(k)
        st = State.__new__(State)
        object.__setattr__(st, "spectral", sp)
        object.__setattr__(st, "member", i)
        return st

    def initial_state(self, k, qq, dd, gg):
        """Member k's start-up fields (as initial_state); call invert_all() after
        loading every member."""
        sp, i = self.member(k)
        initial_state(sp, qq, dd, gg, member=i, invert=False)

    def invert_all(self):
        for sp in {id(v): v for v in self._spectral.values()}.values():
            check(lib().sw_main_invert(sp.ctx))

    def stream(self):
        """The stream the ensemble's step graphs run on (an int cudaStream_t)."""
        s = ctypes.c_void_p()
        check(lib().sw_ensemble_stream(self._h, ctypes.byref(s)))
        return s.value

    def advance(self, nsteps=1, ggen=True):
        check(lib().sw_ensemble_advance(self._h, int(nsteps), int(bool(ggen))))

    def advance_async(self, nsteps=1, ggen=True):
        check(lib().sw_ensemble_advance_async(self._h, int(nsteps), int(bool(ggen))))

    def sync(self):
        check(lib().sw_ensemble_sync(self._h))

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            for sp in self._spectral.values():
                sp._ctx = ctypes.c_void_p()
            lib().sw_ensemble_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _read_r8(path):
    raw = np.fromfile(path, dtype="<f8")
    return raw[1:]


def nhswps(parameters, precision=0, device=0):
    """Run nhswps from qq/dd/gg_init.r8 in the output directory (src/nhswps/mod.rs:150-345)."""
    num = parameters.numerical
    ng, nz = num.grid_resolution, num.vertical_layers
    dt, tgsave, tsim = num.time_step, num.save_interval, num.duration
    out_dir = str(parameters.environment.output_directory)
    qq = _read_r8(os.path.join(out_dir, "qq_init.r8"))
    dd = _read_r8(os.path.join(out_dir, "dd_init.r8"))
    gg = _read_r8(os.path.join(out_dir, "gg_init.r8"))
    sp = Spectral(ng, nz, precision=precision, device=device)
    state = initial_state(sp, qq, dd, gg)
    output = Output.from_path(out_dir)
    try:
        state.ngsave = _round_half_away(tgsave / dt)
        while state.t <= tsim:
            state.itime = _round_half_away(state.t / dt)
            state.jtime = state.itime // state.ngsave
            if state.ngsave * state.jtime == state.itime:
                check(lib().sw_main_invert(sp.ctx))
                psolve(state)
                savegrid(state, output)
                state.ggen = False
            else:
                state.ggen = True
            advance(state, output)
        state.itime = int(state.t / dt)
        state.jtime = state.itime // state.ngsave
        if state.ngsave * state.jtime == state.itime:
            check(lib().sw_main_invert(sp.ctx))
            psolve(state)
            savegrid(state, output)
    finally:
        output.close()
    return state
