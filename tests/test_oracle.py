"""Pins the CPU oracle against the reference's own golden vectors.

Tolerances are the reference's: 1e-13 for stafft/trig/spec1d slices
(src/utils.rs:35-39), 1e-10 for the spectral and nhswps functions
(src/spectral/test.rs, src/nhswps/*.rs tests).  The reference compares its
FFT fixtures bit-exactly; the oracle's butterflies are its own, so those
comparisons use 1e-13 relative to the fixture's largest entry.
"""
import numpy as np
import pytest

from conftest import golden

FFT_CASES = [(n, s) for n in (12, 15, 16, 18, 24) for s in (1, 2)]


def _close(a, b, tol):
    a = np.asarray(a).reshape(-1)
    b = np.asarray(b).reshape(-1)
    assert a.shape == b.shape
    err = np.abs(a - b).max()
    assert err <= tol, "max abs err %.3e > %.1e" % (err, tol)


def _rel(a, b, tol=1e-13):
    scale = max(np.abs(b).max(), 1e-300)
    _close(np.asarray(a) / scale, np.asarray(b) / scale, tol)


def test_factorisen(oracle):
    assert oracle.factorisen(16) == (0, [0, 2, 0, 0, 0])
    assert oracle.factorisen(8640) == (0, [3, 1, 1, 0, 1])
    assert oracle.factorisen(256)[1] == [0, 4, 0, 0, 0]
    assert oracle.factorisen(160)[1] == [0, 2, 1, 0, 1]
    assert oracle.factorisen(14)[0] != 0  # prime factor 7: factorisation fails


@pytest.mark.parametrize("n", [18, 30, 32])
def test_initfft(oracle, n):
    _, trig = oracle.initfft(n)
    _close(trig, golden("stafft")["initfft/%d_trig.bin" % n], 1e-13)


@pytest.mark.parametrize("n,s", FFT_CASES)
def test_forfft(oracle, n, s):
    g = golden("stafft")
    x = g["forfft/forfft_ng%d_%d_x.bin" % (n, s)]
    _rel(oracle.forfft(n, n, x), g["forfft/forfft_ng%d_%d_x2.bin" % (n, s)])


@pytest.mark.parametrize("n,s", FFT_CASES)
def test_revfft(oracle, n, s):
    g = golden("stafft")
    x = g["revfft/revfft_ng%d_%d_x.bin" % (n, s)]
    _rel(oracle.revfft(n, n, x), g["revfft/revfft_ng%d_%d_x2.bin" % (n, s)])


@pytest.mark.parametrize("n", [32, 96, 160, 256, 384, 512])
def test_fft_numpy(oracle, n):
    """Config sizes not in the fixtures (n=160 aborts in the reference's forrdx2)."""
    rng = np.random.default_rng(2)
    m = 7
    x = rng.standard_normal((n, m))  # x[j, i] -> flat i + m*j
    h = oracle.forfft(m, n, x.reshape(-1)).reshape(n, m)
    F = np.fft.fft(x, axis=0) / np.sqrt(n)
    ref = np.zeros_like(x)
    ref[: n // 2 + 1] = F[: n // 2 + 1].real
    for k in range(1, (n - 1) // 2 + 1):
        ref[n - k] = F[k].imag
    _close(h, ref, 1e-13 * np.sqrt(n))
    _close(oracle.revfft(m, n, h.reshape(-1)), x.reshape(-1), 1e-13 * np.sqrt(n))


def test_ptospc_spctop(oracle):
    g = golden("sta2dfft")
    sp = oracle.Spectral(32, 4)
    _rel(sp.ptospc(g["ptospc/ptospc_ng32_rvar.bin"]), g["ptospc/ptospc_ng32_svar2.bin"])
    _rel(sp.spctop(g["spctop/spctop_ng32_svar.bin"]), g["spctop/spctop_ng32_rvar2.bin"])


@pytest.mark.parametrize("which,case,ng", [("x", 1, 32), ("x", 2, 24), ("y", 1, 32), ("y", 2, 24)])
def test_deriv(oracle, which, case, ng):
    g = golden("sta2dfft")
    sp = oracle.Spectral(ng, 4)
    var = g["deriv/%sderiv_%d_var.bin" % (which, case)]
    out = sp.xderiv(var) if which == "x" else sp.yderiv(var)
    _close(out, g["deriv/%sderiv_%d_der2.bin" % (which, case)], 0.0)


@pytest.mark.parametrize("n", [30, 120])
def test_init2dfft_trig(oracle, n):
    _, trig = oracle.initfft(n)
    _close(trig, golden("sta2dfft")["init2dfft/ng%d_trig.bin" % n], 1e-13)


SPECTRAL_OPS = ["hlap", "glap", "rlap", "helm", "c2g2", "simp", "rope", "fope", "filt", "diss",
                "opak", "rdis", "etdv", "htdv", "ap", "etd1", "htd1", "theta", "weight", "hrkx",
                "hrky", "rk", "spmf", "alk"]


@pytest.mark.parametrize("name", SPECTRAL_OPS)
def test_init_spectral(oracle, name):
    sp = oracle.Spectral(32, 4)
    ref = golden("spectral")["init_spectral/32_4_%s.bin" % name]
    got = sp.get(name)
    if name == "alk":
        _close(got[: ref.size], ref, 1e-13)
    else:
        _rel(got, ref, 1e-15)


def test_init_spectral_kmag(oracle):
    sp = oracle.Spectral(32, 4)
    ref = golden("spectral")["init_spectral/32_4_kmag.bin"].astype(">f8").view(">u8").astype(np.int64)
    assert np.array_equal(sp.get("kmag").astype(np.int64), ref)
    assert sp.get("kmax")[0] == 23 and sp.get("kmaxred")[0] == 16


@pytest.mark.parametrize("ng,nz", [(18, 2), (30, 4), (48, 6)])
def test_main_invert(oracle, ng, nz):
    g = golden("spectral")
    k = "main_invert/%d_%d_" % (ng, nz)
    sp = oracle.Spectral(ng, nz)
    r, u, v, zeta = sp.main_invert(g[k + "qs.bin"], g[k + "ds.bin"], g[k + "gs.bin"])
    for name, got in (("r", r), ("u", u), ("v", v), ("zeta", zeta)):
        _close(got, g[k + name + ".bin"], 1e-10)


@pytest.mark.parametrize("fn", ["jacob", "divs"])
@pytest.mark.parametrize("ng,nz", [(30, 4), (48, 6)])
def test_jacob_divs(oracle, fn, ng, nz):
    g = golden("spectral")
    k = "%s/%d_%d_" % (fn, ng, nz)
    sp = oracle.Spectral(ng, nz)
    got = getattr(sp, fn)(g[k + "aa.bin"], g[k + "bb.bin"])
    _close(got, g[k + "cs.bin"], 1e-10)


@pytest.mark.parametrize("ng,nz", [(18, 2), (30, 4)])
def test_ptospc3d_spctop3d(oracle, ng, nz):
    g = golden("spectral")
    sp = oracle.Spectral(ng, nz)
    k = "ptospc3d/%d_%d_" % (ng, nz)
    fs = sp.ptospc3d(g[k + "fp.bin"], g[k + "fs.bin"], 0, nz - 1)
    _close(fs, g[k + "fs2.bin"], 1e-10)
    k = "spctop3d/%d_%d_" % (ng, nz)
    fp = sp.spctop3d(g[k + "fs.bin"], g[k + "fp.bin"], 0, nz - 1)
    _close(fp, g[k + "fp2.bin"], 1e-10)


@pytest.mark.parametrize("ng,nz", [(18, 2), (30, 4)])
def test_deal3d(oracle, ng, nz):
    g = golden("spectral")
    k = "deal3d/%d_%d_" % (ng, nz)
    _close(oracle.Spectral(ng, nz).deal3d(g[k + "fp.bin"]), g[k + "fp2.bin"], 1e-10)


@pytest.mark.parametrize("ng,nz", [(18, 2), (32, 4)])
def test_deal2d(oracle, ng, nz):
    g = golden("spectral")
    k = "deal2d/%d_%d_" % (ng, nz)
    _close(oracle.Spectral(ng, nz).deal2d(g[k + "fp.bin"]), g[k + "fp2.bin"], 1e-10)


@pytest.mark.parametrize("ng,nz", [(18, 2), (48, 4)])
def test_spec1d(oracle, ng, nz):
    g = golden("spectral")
    k = "spec1d/%d_%d_" % (ng, nz)
    spec = oracle.Spectral(ng, nz).spec1d(g[k + "ss.bin"])
    ref = g[k + "spec2.bin"]
    kmax = int(oracle.Spectral(ng, nz).get("kmax")[0])
    _close(spec[: kmax + 1], ref[: kmax + 1], 1e-13)


@pytest.mark.parametrize("n,s", FFT_CASES)
def test_second_radix_schedule_matches_golden(oracle, n, s):
    """The oracle's second radix schedule (5, 3, 2; the float64 floor of the GPU
    tests comes from comparing the two schedules) computes the same transforms."""
    g = golden("stafft")
    oracle.set_fft_order(1)
    try:
        _rel(oracle.forfft(n, n, g["forfft/forfft_ng%d_%d_x.bin" % (n, s)]), g["forfft/forfft_ng%d_%d_x2.bin" % (n, s)])
        _rel(oracle.revfft(n, n, g["revfft/revfft_ng%d_%d_x.bin" % (n, s)]), g["revfft/revfft_ng%d_%d_x2.bin" % (n, s)])
    finally:
        oracle.set_fft_order(0)
    assert oracle.get_fft_order() == 0


def test_radix_schedule_spread_is_float64_rounding(oracle):
    """Two 3-step ng=32 runs under the two schedules differ at float64 rounding
    only (delta, gamma and p most, being small residual fields)."""
    import importlib.util
    import os
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "oracle_spread.py")
    spec = importlib.util.spec_from_file_location("oracle_spread", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    sp = mod.spread(32, 4, 3)
    assert all(0.0 < v < 1e-10 for v in sp.values()), sp
    assert sp["qs"] < 1e-14
