"""Pins the oracle's nhswps functions against the reference's golden vectors.

Each fixture case ``<ng>_<nz>`` holds the input fields ``<name>.bin`` and the
expected outputs ``<name>2.bin``; tolerance is the reference's 1e-10 absolute
(src/nhswps/{vertical,coeffs,cpsource,source,psolve,advance}.rs tests) or
1e-13 where the reference uses assert_approx_eq_slice (cpsource, source).
cpsource is held to 1e-12: its result (|sp0| ~ 0.1) is the difference of
terms of size ~50 (g*Lap(h), f*zeta), and the oracle's FFT rounds differently
from the reference's radix kernels, so 1e-13 absolute is below its noise.
"""
import numpy as np
import pytest

from conftest import golden
from oracle.oracle import FIELDS


def load_state(orc, group, case, ng, nz):
    g = golden("nhswps")
    fields = {}
    for name in FIELDS:
        for key in ("%s/%s_%s.bin" % (group, case, name), "%s/%s/%s.bin" % (group, case, name)):
            if key in g:
                fields[name] = g[key]
    return orc.State(ng, nz, fields)


def expect(group, case, name):
    g = golden("nhswps")
    for key in ("%s/%s_%s2.bin" % (group, case, name), "%s/%s/%s2.bin" % (group, case, name)):
        if key in g:
            return g[key]
    raise KeyError(name)


def _close(a, b, tol):
    err = np.abs(np.asarray(a).reshape(-1) - np.asarray(b).reshape(-1)).max()
    assert err <= tol, "max abs err %.3e > %.1e" % (err, tol)


@pytest.mark.parametrize("ng,nz", [(18, 2), (32, 4)])
def test_vertical(oracle, ng, nz):
    sp = oracle.Spectral(ng, nz)
    st = load_state(oracle, "vertical", "%d_%d" % (ng, nz), ng, nz)
    oracle.vertical(sp, st)
    for name in ("z", "zx", "zy", "w", "aa"):
        _close(st.f[name], expect("vertical", "%d_%d" % (ng, nz), name), 1e-10)


@pytest.mark.parametrize("ng,nz", [(18, 2), (32, 4)])
def test_coeffs(oracle, ng, nz):
    sp = oracle.Spectral(ng, nz)
    case = "%d_%d" % (ng, nz)
    st = load_state(oracle, "coeffs", case, ng, nz)
    sigx, sigy, cpt1, cpt2 = oracle.coeffs(sp, st)
    g = golden("nhswps")
    _close(sigx, g["coeffs/%s_sigx2.bin" % case], 1e-10)
    _close(sigy, g["coeffs/%s_sigy2.bin" % case], 1e-10)
    _close(cpt1, g["coeffs/%s_cpt12.bin" % case], 1e-10)
    _close(cpt2, g["coeffs/%s_cpt22.bin" % case], 1e-10)


@pytest.mark.parametrize("ng,nz", [(18, 2), (32, 4)])
def test_cpsource(oracle, ng, nz):
    sp = oracle.Spectral(ng, nz)
    case = "%d_%d" % (ng, nz)
    st = load_state(oracle, "cpsource", case, ng, nz)
    sp0 = oracle.cpsource(sp, st)
    _close(sp0, golden("nhswps")["cpsource/%s_sp02.bin" % case], 1e-12)


@pytest.mark.parametrize("ng,nz", [(18, 2), (32, 4)])
def test_source(oracle, ng, nz):
    sp = oracle.Spectral(ng, nz)
    case = "%d_%d" % (ng, nz)
    st = load_state(oracle, "source", case, ng, nz)
    sqs, sds, sgs = oracle.source(sp, st)
    g = golden("nhswps")
    for name, got in (("sqs", sqs), ("sds", sds), ("sgs", sgs)):
        ref = g["source/%s_%s2.bin" % (case, name)]
        _close(got, ref, 1e-13 * max(1.0, np.abs(ref).max()))


@pytest.mark.parametrize("ng,nz", [(24, 4), (32, 4)])
def test_psolve(oracle, ng, nz):
    sp = oracle.Spectral(ng, nz)
    case = "%d_%d" % (ng, nz)
    st = load_state(oracle, "psolve", case, ng, nz)
    status, iters, errp = oracle.psolve(sp, st)
    assert status == 0 and 1 <= iters < 100 and errp <= 1e-9
    for name in ("z", "zx", "zy", "w", "aa", "ri", "pn", "ps", "dpn"):
        _close(st.f[name], expect("psolve", case, name), 1e-10)


@pytest.mark.parametrize("ng,nz,t0,t1", [(18, 6, 5.555_555_555_555_555E-2, 0.111_111_111_111_111_1),
                                         (24, 4, 0.624_999_999_999_999_9, None)])
def test_advance(oracle, ng, nz, t0, t1):
    sp = oracle.Spectral(ng, nz)
    case = "%d_%d" % (ng, nz)
    st = load_state(oracle, "advance", case, ng, nz)
    st.t = t0
    status, diag, iters = oracle.advance(sp, st, ggen=True)
    assert status == 0
    for name in FIELDS:
        _close(st.f[name], expect("advance", case, name), 1e-10)
    if t1 is not None:
        assert abs(st.t - t1) <= 1e-10


def test_psolve_maxiter_status(oracle):
    """A sweep cap that cannot be met returns the error status the reference
    turns into quit::with_code(1) (src/nhswps/psolve.rs:360-366)."""
    sp = oracle.Spectral(24, 4)
    st = load_state(oracle, "psolve", "24_4", 24, 4)
    status, iters, _ = oracle.psolve(sp, st, nitmax=1)
    assert status == oracle.ERR_PSOLVE_MAXITER and iters == 1
