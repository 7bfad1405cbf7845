"""End-to-end pins of the oracle: the initial-condition generators and the
complete vstrip -> balinit -> swto3d -> nhswps run (reference src/test.rs:11-43),
whose monitor.asc/ecomp.asc text the reference compares token by token."""
import numpy as np
import pytest

from conftest import golden


def _r8(a, skip=1):
    return a[skip:]


@pytest.mark.parametrize("ng", [18, 32, 64])
def test_vstrip(oracle, ng):
    ref = golden("sta2dfft")["vstrip/qq_init_%d.r8" % ng][1:]
    got = oracle.vstrip(ng)
    np.testing.assert_allclose(got, ref, rtol=0, atol=1e-13)


@pytest.mark.parametrize("ng,nz", [(18, 2), (32, 4)])
def test_balinit(oracle, ng, nz):
    g = golden("sta2dfft")
    qq0 = g["balinit/%d_%d_qq_init.r8" % (ng, nz)][1:]
    sw = g["balinit/%d_%d_sw_init.r8" % (ng, nz)].reshape(3, ng * ng + 1)[:, 1:]
    qq, dd, gg = oracle.balinit(ng, nz, qq0)
    for got, ref in zip((qq, dd, gg), sw):
        np.testing.assert_allclose(got, ref, rtol=0, atol=1e-11)


def test_swto3d(oracle):
    g = golden("sta2dfft")
    sw = g["swto3d/18_2_sw_init.r8"].reshape(3, 18 * 18 + 1)[:, 1:]
    q3, d3, g3 = oracle.swto3d(2, *sw)
    for got, name in ((q3, "qq"), (d3, "dd"), (g3, "gg")):
        np.testing.assert_array_equal(got, g["swto3d/18_2_%s_init.r8" % name][1:])


def _tokens(raw):
    return bytes(raw).decode().split()


@pytest.mark.parametrize("ng,nz,dt,tsim", [(32, 4, 1.0 / 32, 1.0), (18, 4, 1.0 / 18, 2.0)])
def test_complete(oracle, ng, nz, dt, tsim):
    qq0 = oracle.vstrip(ng)
    qq, dd, gg = oracle.balinit(ng, nz, qq0)
    q3, d3, g3 = oracle.swto3d(nz, qq, dd, gg)
    monitor, ecomp, sweeps = oracle.run_nhswps(ng, nz, dt, 0.25, tsim, q3, d3, g3)
    g = golden("complete")
    ref_m = _tokens(g["%d_%d/monitor.asc" % (ng, nz)])
    ref_e = _tokens(g["%d_%d/ecomp.asc" % (ng, nz)])
    got_m = " ".join(monitor).split()
    got_e = " ".join(ecomp).split()
    assert len(got_m) == len(ref_m) and len(got_e) == len(ref_e)
    # printed to 5-9 decimals: compare numerically at one unit of the last digit
    np.testing.assert_allclose(np.array(got_m, float), np.array(ref_m, float), rtol=0, atol=1.01e-6)
    np.testing.assert_allclose(np.array(got_e, float), np.array(ref_e, float), rtol=0, atol=1.01e-9)
