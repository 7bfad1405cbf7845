"""GPU parity: the CUDA path (through the C ABI) against the reference's golden
vectors and the CPU oracle.

Tolerances: the reference's own (1e-10 absolute for the spectral and nhswps
functions, 1e-13 for transforms and slices, scaled by the fixture's magnitude
where the reference compares bit-exactly).  Multi-step runs against the FP64
oracle: the FP64 path within 3x the oracle's own float64 rounding spread (the
oracle run again with its second radix schedule, field by field); SW_MIXED within
the 1e-5 rel-L2 of its contract; SW_FP32 within its measured, documented bounds.
"""
import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu
FIELDS = ["u", "v", "w", "z", "zx", "zy", "r", "ri", "aa", "zeta", "pn", "dpn", "ps", "qs", "ds", "gs"]


def _close(a, b, tol):
    a = np.ravel(np.asarray(a), order="F")
    b = np.ravel(np.asarray(b), order="F")
    err = np.abs(a - b).max()
    assert err <= tol, "max abs err %.3e > %.1e" % (err, tol)


def _rel(a, b, tol=1e-13):
    scale = max(np.abs(b).max(), 1e-300)
    _close(np.asarray(a) / scale, np.asarray(b) / scale, tol)


def rel_l2(a, b):
    a = np.ravel(a, order="F")
    b = np.ravel(b, order="F")
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


# ---- stafft / sta2dfft --------------------------------------------------------
@pytest.mark.parametrize("n,s", [(n, s) for n in (12, 15, 16, 18, 24) for s in (1, 2)])
def test_forfft_revfft_golden(sw, n, s):
    g = golden("stafft")
    _, trig = sw.stafft.initfft(n)
    fac = sw.stafft.factorisen(n)
    x = g["forfft/forfft_ng%d_%d_x.bin" % (n, s)].copy()
    _rel(sw.stafft.forfft(n, n, x, trig, fac), g["forfft/forfft_ng%d_%d_x2.bin" % (n, s)])
    x = g["revfft/revfft_ng%d_%d_x.bin" % (n, s)].copy()
    _rel(sw.stafft.revfft(n, n, x, trig, fac), g["revfft/revfft_ng%d_%d_x2.bin" % (n, s)])


@pytest.mark.parametrize("n", [32, 96, 160, 256, 384, 512])
def test_fft_config_sizes_vs_oracle(sw, oracle, n):
    """Batch (nz+1)*n = 17n columns, N(0,1) inputs (seed 2)."""
    m = 17 * n
    rng = np.random.default_rng(2)
    x = rng.standard_normal(m * n)
    ref = oracle.forfft(m, n, x)
    got = sw.stafft.forfft(m, n, x.copy())
    _rel(got, ref, 1e-14 * np.sqrt(n))
    back = sw.stafft.revfft(m, n, got.copy())
    _rel(back, x, 1e-14 * np.sqrt(n))


def test_ptospc_spctop_golden(sw):
    g = golden("sta2dfft")
    sp = sw.Spectral(32, 4)
    _rel(sp.ptospc(g["ptospc/ptospc_ng32_rvar.bin"]), g["ptospc/ptospc_ng32_svar2.bin"])
    _rel(sp.spctop(g["spctop/spctop_ng32_svar.bin"]), g["spctop/spctop_ng32_rvar2.bin"])


@pytest.mark.parametrize("which,case,ng", [("x", 1, 32), ("x", 2, 24), ("y", 1, 32), ("y", 2, 24)])
def test_deriv_golden(sw, which, case, ng):
    g = golden("sta2dfft")
    sp = sw.Spectral(ng, 4)
    var = g["deriv/%sderiv_%d_var.bin" % (which, case)]
    out = sp.xderiv(var) if which == "x" else sp.yderiv(var)
    _close(out, g["deriv/%sderiv_%d_der2.bin" % (which, case)], 0.0)


@pytest.mark.parametrize("name", ["hlap", "glap", "rlap", "helm", "c2g2", "simp", "rope", "fope", "filt",
                                  "diss", "opak", "rdis", "etdv", "htdv", "ap", "etd1", "htd1", "theta",
                                  "weight", "hrkx", "hrky", "rk", "spmf"])
def test_init_spectral_golden(sw, name):
    sp = sw.Spectral(32, 4)
    ref = golden("spectral")["init_spectral/32_4_%s.bin" % name]
    _rel(np.ravel(getattr(sp, name), order="F"), ref, 1e-15)


# ---- spectral ---------------------------------------------------------------------
@pytest.mark.parametrize("ng,nz", [(18, 2), (30, 4), (48, 6)])
def test_main_invert_golden(sw, ng, nz):
    g = golden("spectral")
    k = "main_invert/%d_%d_" % (ng, nz)
    sp = sw.Spectral(ng, nz)
    r, u, v, zeta = sp.main_invert(g[k + "qs.bin"], g[k + "ds.bin"], g[k + "gs.bin"])
    for name, got in (("r", r), ("u", u), ("v", v), ("zeta", zeta)):
        _close(got, g[k + name + ".bin"], 1e-10)


@pytest.mark.parametrize("fn", ["jacob", "divs"])
@pytest.mark.parametrize("ng,nz", [(30, 4), (48, 6)])
def test_jacob_divs_golden(sw, fn, ng, nz):
    g = golden("spectral")
    k = "%s/%d_%d_" % (fn, ng, nz)
    sp = sw.Spectral(ng, nz)
    _close(getattr(sp, fn)(g[k + "aa.bin"], g[k + "bb.bin"]), g[k + "cs.bin"], 1e-10)


@pytest.mark.parametrize("ng,nz", [(18, 2), (30, 4)])
def test_ptospc3d_spctop3d_deal3d_golden(sw, ng, nz):
    g = golden("spectral")
    sp = sw.Spectral(ng, nz)
    k = "ptospc3d/%d_%d_" % (ng, nz)
    _close(sp.ptospc3d(g[k + "fp.bin"], g[k + "fs.bin"].copy(), 0, nz - 1), g[k + "fs2.bin"], 1e-10)
    k = "spctop3d/%d_%d_" % (ng, nz)
    _close(sp.spctop3d(g[k + "fs.bin"], g[k + "fp.bin"].copy(), 0, nz - 1), g[k + "fp2.bin"], 1e-10)
    k = "deal3d/%d_%d_" % (ng, nz)
    _close(sp.deal3d(g[k + "fp.bin"].copy()), g[k + "fp2.bin"], 1e-10)


@pytest.mark.parametrize("ng,nz", [(18, 2), (32, 4)])
def test_deal2d_golden(sw, ng, nz):
    g = golden("spectral")
    k = "deal2d/%d_%d_" % (ng, nz)
    _close(sw.Spectral(ng, nz).deal2d(g[k + "fp.bin"].copy()), g[k + "fp2.bin"], 1e-10)


@pytest.mark.parametrize("ng,nz", [(18, 2), (48, 4)])
def test_spec1d_golden(sw, ng, nz):
    g = golden("spectral")
    k = "spec1d/%d_%d_" % (ng, nz)
    sp = sw.Spectral(ng, nz)
    spec = sp.spec1d(g[k + "ss.bin"])
    _close(spec[: sp.kmax + 1], g[k + "spec2.bin"][: sp.kmax + 1], 1e-13)


# ---- nhswps -------------------------------------------------------------------------
def gpu_state(sw, group, case, ng, nz, t=0.0):
    g = golden("nhswps")
    sp = sw.Spectral(ng, nz)
    fields = {}
    for name in FIELDS:
        for key in ("%s/%s_%s.bin" % (group, case, name), "%s/%s/%s.bin" % (group, case, name)):
            if key in g:
                fields[name] = g[key]
    return sw.State(sp, t=t, **fields)


def expect(group, case, name):
    g = golden("nhswps")
    for key in ("%s/%s_%s2.bin" % (group, case, name), "%s/%s/%s2.bin" % (group, case, name)):
        if key in g:
            return g[key]
    raise KeyError(name)


@pytest.mark.parametrize("ng,nz", [(18, 2), (32, 4)])
def test_vertical_golden(sw, ng, nz):
    st = gpu_state(sw, "vertical", "%d_%d" % (ng, nz), ng, nz)
    sw.nhswps.vertical(st)
    for name in ("z", "zx", "zy", "w", "aa"):
        _close(st.get(name), expect("vertical", "%d_%d" % (ng, nz), name), 1e-10)


@pytest.mark.parametrize("ng,nz", [(18, 2), (32, 4)])
def test_coeffs_golden(sw, ng, nz):
    case = "%d_%d" % (ng, nz)
    st = gpu_state(sw, "coeffs", case, ng, nz)
    outs = sw.nhswps.coeffs(st)
    g = golden("nhswps")
    for name, got in zip(("sigx", "sigy", "cpt1", "cpt2"), outs):
        _close(got, g["coeffs/%s_%s2.bin" % (case, name)], 1e-10)


@pytest.mark.parametrize("ng,nz", [(18, 2), (32, 4)])
def test_cpsource_golden(sw, ng, nz):
    case = "%d_%d" % (ng, nz)
    st = gpu_state(sw, "cpsource", case, ng, nz)
    _close(sw.nhswps.cpsource(st), golden("nhswps")["cpsource/%s_sp02.bin" % case], 1e-12)


@pytest.mark.parametrize("ng,nz", [(18, 2), (32, 4)])
def test_source_golden(sw, ng, nz):
    case = "%d_%d" % (ng, nz)
    st = gpu_state(sw, "source", case, ng, nz)
    outs = sw.nhswps.source(st)
    g = golden("nhswps")
    for name, got in zip(("sqs", "sds", "sgs"), outs):
        ref = g["source/%s_%s2.bin" % (case, name)]
        _close(got, ref, 1e-13 * max(1.0, np.abs(ref).max()))


@pytest.mark.parametrize("ng,nz", [(24, 4), (32, 4)])
def test_psolve_golden(sw, oracle, ng, nz):
    case = "%d_%d" % (ng, nz)
    st = gpu_state(sw, "psolve", case, ng, nz)
    it, errp = sw.nhswps.psolve(st)
    ost = oracle.State(ng, nz, {k: np.ravel(st.get(k), order="F") for k in FIELDS})
    # same sweep count as the oracle on the same input
    ost2 = oracle.State(ng, nz, {k: v for k, v in _inputs("psolve", case).items()})
    status, oit, oerr = oracle.psolve(oracle.Spectral(ng, nz), ost2)
    assert status == 0 and it == oit
    for name in ("z", "zx", "zy", "w", "aa", "ri", "pn", "ps", "dpn"):
        _close(st.get(name), expect("psolve", case, name), 1e-10)


def _inputs(group, case):
    g = golden("nhswps")
    out = {}
    for name in FIELDS:
        for key in ("%s/%s_%s.bin" % (group, case, name), "%s/%s/%s.bin" % (group, case, name)):
            if key in g:
                out[name] = g[key]
    return out


@pytest.mark.parametrize("ng,nz,t0", [(18, 6, 5.555_555_555_555_555E-2), (24, 4, 0.624_999_999_999_999_9)])
def test_advance_golden(sw, ng, nz, t0):
    case = "%d_%d" % (ng, nz)
    st = gpu_state(sw, "advance", case, ng, nz, t=t0)
    st.ggen = True
    sw.nhswps.advance(st)
    for name in FIELDS:
        _close(st.get(name), expect("advance", case, name), 1e-10)
    assert abs(st.t - (t0 + 1.0 / ng)) < 1e-12


# ---- multi-step runs against the FP64 oracle (config: ng=32, nz=4, vstrip -> balinit,
# q + N(0, 1e-3) seed 1, delta = gamma = 0, 10 steps) ---------------------------------
def _config0(sw, oracle, precision, steps):
    ng, nz = 32, 4
    qq0 = oracle.vstrip(ng)
    qb, _, _ = oracle.balinit(ng, nz, qq0)
    rng = np.random.default_rng(1)
    q3 = np.tile(qb, nz + 1) + rng.normal(0.0, 1.0e-3, ng * ng * (nz + 1))
    z3 = np.zeros_like(q3)
    sp = sw.Spectral(ng, nz, precision=precision)
    st = sw.nhswps.initial_state(sp, q3, z3, z3)
    st.ggen = True
    osp, ost = oracle.initial_state(ng, nz, q3, z3, z3)
    for _ in range(steps):
        sw.nhswps.advance(st)
        status, _, _ = oracle.advance(osp, ost, ggen=True)
        assert status == 0
    return st, ost


def _h(f, nz):
    """h = z(nz)/HBAR - 1 per horizontal point."""
    return f[-f.size // (nz + 1):] / 0.4 - 1.0


_SPREAD = {}


def _config0_spread(oracle, steps):
    """rel-L2 between two oracle runs of the configuration that differ only in the
    radix schedule of their transforms: the float64 rounding floor of this run."""
    if steps not in _SPREAD:
        ng, nz = 32, 4
        qq0 = oracle.vstrip(ng)
        qb, _, _ = oracle.balinit(ng, nz, qq0)
        rng = np.random.default_rng(1)
        q3 = np.tile(qb, nz + 1) + rng.normal(0.0, 1.0e-3, ng * ng * (nz + 1))
        z3 = np.zeros_like(q3)
        runs = []
        for order in (0, 1):
            oracle.set_fft_order(order)
            try:
                osp, ost = oracle.initial_state(ng, nz, q3, z3, z3)
                for _ in range(steps):
                    assert oracle.advance(osp, ost, ggen=True)[0] == 0
            finally:
                oracle.set_fft_order(0)
            runs.append(ost.f)
        _SPREAD[steps] = {k: rel_l2(runs[1][k], runs[0][k]) for k in runs[0]}
    return _SPREAD[steps]


def test_fp64_ten_steps_vs_oracle(sw, oracle):
    """The FP64 path after 10 steps against the oracle, every field within 3x the
    oracle's own rounding spread (measured here: 9e-16 on qs, 8e-15 on u, 2e-12 on
    pn, 3e-12 on delta, 5e-12 on gamma).  delta, gamma and p are small residual fields
    whose relative rounding error is the largest."""
    st, ost = _config0(sw, oracle, sw.SW_FP64, 10)
    spread = _config0_spread(oracle, 10)
    for k in ("qs", "ds", "gs", "u", "v", "z", "pn"):
        err = rel_l2(st.get(k), ost.f[k])
        assert err <= 3.0 * max(spread[k], 1e-16), "%s rel-L2 %.3e > 3 x spread %.3e" % (k, err, spread[k])


def test_mixed_ten_steps_vs_oracle(sw, oracle):
    """SW_MIXED (float32 correction sweeps with stop rule 1e-7, float32 transforms for
    the dealiased products of the pressure set-up and source) within its 1e-5 rel-L2
    contract on every field, the pressure included."""
    st, ost = _config0(sw, oracle, sw.SW_MIXED, 10)
    for k in ("qs", "ds", "gs", "u", "v", "z", "pn"):
        err = rel_l2(st.get(k), ost.f[k])
        assert err <= 1e-5, "%s rel-L2 %.3e" % (k, err)


def test_fp32_ten_steps_vs_oracle(sw, oracle):
    """SW_FP32 (float32 transforms and physical fields) at ng=32: within 1e-5 on
    every field but the pressure, whose float32 iteration stops at 1e-6 or on
    stagnation (bound 1e-4).  Its error grows with ng (test_gpu_batching, ng=256)."""
    st, ost = _config0(sw, oracle, sw.SW_FP32, 10)
    for k, tol in (("qs", 1e-5), ("ds", 1e-5), ("gs", 1e-5), ("u", 1e-5), ("v", 1e-5), ("z", 1e-5), ("pn", 1e-4)):
        err = rel_l2(st.get(k), ost.f[k])
        assert err <= tol, "%s rel-L2 %.3e > %.0e" % (k, err, tol)


@pytest.mark.parametrize("precision", ["fp64", "mixed", "fp32"])
def test_nonfinite_state_reports_diverged(sw, precision):
    """A NaN put into qs from the host ends the pressure iteration with
    SW_ERR_PSOLVE_DIVERGED (a deliberate deviation: the reference's `while errp >
    toler` leaves the loop on a NaN as if converged, psolve.rs:88), in graph and
    host-driven steps, and the context stays usable: a valid state then advances."""
    import ctypes
    prec = {"fp64": sw.SW_FP64, "mixed": sw.SW_MIXED, "fp32": sw.SW_FP32}[precision]
    ng, nz = 32, 4
    qq = sw.vstrip.pv_strip(ng)
    rng = np.random.default_rng(4)
    q3 = np.tile(qq, nz + 1) + rng.normal(0.0, 1.0e-3, ng * ng * (nz + 1))
    z3 = np.zeros_like(q3)
    L = sw._native.lib()
    for graphs in (1, 0):
        sp = sw.Spectral(ng, nz, precision=prec)
        sw._native.check(L.sw_set_graphs(sp.ctx, graphs))
        st = sw.nhswps.initial_state(sp, q3, z3, z3)
        good = st.get("qs").copy()
        bad = good.copy()
        bad[3, 5, 2] = np.nan
        st.set("qs", bad)
        assert L.sw_advance(sp.ctx, 1, 1) == sw._native.SW_ERR_PSOLVE_DIVERGED
        for k in FIELDS:  # a fresh state, as nhswps makes one (pressure first guess 0)
            st.set(k, np.zeros(sp.n3))
        st = sw.nhswps.initial_state(sp, q3, z3, z3)
        sw._native.check(L.sw_advance(sp.ctx, 2, 1))
        assert np.all(np.isfinite(st.get("gs")))
        sp.close()


def test_graph_steps_match_host_driven_steps(sw):
    """A step run as one CUDA graph (device-side pressure loops) gives the same
    fields, bit for bit, as the host-driven path."""
    import ctypes
    ng, nz = 32, 4
    qq = sw.vstrip.pv_strip(ng)
    rng = np.random.default_rng(3)
    q3 = np.tile(qq, nz + 1) + rng.normal(0.0, 1.0e-3, ng * ng * (nz + 1))
    z3 = np.zeros_like(q3)
    out = []
    for graphs in (1, 0):
        sp = sw.Spectral(ng, nz)
        sw._native.check(sw._native.lib().sw_set_graphs(sp.ctx, graphs))
        st = sw.nhswps.initial_state(sp, q3, z3, z3)
        st.ggen = True
        sw.nhswps.advance(st, nsteps=3)
        out.append({k: st.get(k) for k in ("qs", "ds", "gs", "pn", "dpn", "w")})
        out[-1]["sweeps"] = sw.nhswps.last_sweeps(sp)
    for k in ("qs", "ds", "gs", "pn", "dpn", "w"):
        assert np.array_equal(out[0][k], out[1][k]), k
    assert out[0]["sweeps"] == out[1]["sweeps"]


def test_psolve_iteration_cap_raises(sw):
    """An unreachable sweep cap returns SW_ERR_PSOLVE_MAXITER (the reference quits,
    src/nhswps/psolve.rs:360-366), with the GPU context still usable."""
    st = gpu_state(sw, "psolve", "24_4", 24, 4)
    with pytest.raises(sw.SwError) as e:
        sw.nhswps.psolve(st, nitmax=1)
    assert e.value.status == sw._native.SW_ERR_PSOLVE_MAXITER
    it, errp = sw.nhswps.psolve(gpu_state(sw, "psolve", "24_4", 24, 4))
    assert it > 1 and errp <= 1e-9


def test_ensemble_members_match_single_runs(sw):
    """Members of one batched context evolve exactly like separate single runs
    (each member its own seed; no coupling between members)."""
    ng, nz, M, steps = 32, 4, 3, 2
    qq = sw.vstrip.pv_strip(ng)
    inits = []
    for m in range(M):
        rng = np.random.default_rng(100 + m)
        inits.append(np.tile(qq, nz + 1) + rng.normal(0.0, 1.0e-3, ng * ng * (nz + 1)))
    z3 = np.zeros_like(inits[0])
    ens = sw.Spectral(ng, nz, nmembers=M)
    states = [sw.nhswps.initial_state(ens, q, z3, z3, member=m, invert=False) for m, q in enumerate(inits)]
    sw.nhswps.main_invert_all(ens)
    states[0].ggen = True
    sw.nhswps.advance(states[0], nsteps=steps)
    for m in range(M):
        single = sw.Spectral(ng, nz)
        st = sw.nhswps.initial_state(single, inits[m], z3, z3)
        st.ggen = True
        sw.nhswps.advance(st, nsteps=steps)
        for k in ("qs", "ds", "gs", "pn", "u"):
            err = rel_l2(states[m].get(k), st.get(k))
            assert err <= 1e-12, "member %d %s rel-L2 %.3e" % (m, k, err)


@pytest.mark.parametrize("ng,nz", [(18, 2), (32, 4)])
def test_balinit_on_device_matches_golden(sw, ng, nz):
    """sw_balinit (the fixed-point iteration on the device) against the
    reference's sw_init.r8 of the same qq_init (src/balinit.rs:21-435), at the
    oracle's tolerance for this fixture."""
    g = golden("sta2dfft")
    qq0 = g["balinit/%d_%d_qq_init.r8" % (ng, nz)][1:]
    ref = g["balinit/%d_%d_sw_init.r8" % (ng, nz)].reshape(3, ng * ng + 1)[:, 1:]
    got = sw.balinit.balance(ng, nz, qq0)
    for a, b, name in zip(got, ref, ("qq", "dd", "gg")):
        _close(a, b, 1e-11)


def test_balinit_rejects_float32_context(sw):
    sp = sw.Spectral(32, 4, precision=sw.SW_FP32)
    with pytest.raises(sw.SwError) as e:
        sw.balinit.balance(32, 4, np.zeros(32 * 32), spectral=sp)
    assert e.value.status == sw._native.SW_ERR_STATE


@pytest.mark.parametrize("ng,nz,dt,tsim", [(32, 4, 1.0 / 32, 1.0), (18, 4, 1.0 / 18, 2.0)])
def test_nhswps_end_to_end(sw, tmp_path, ng, nz, dt, tsim):
    """vstrip -> balinit -> swto3d -> nhswps through the package (reference
    src/test.rs:29-40): monitor.asc and ecomp.asc match the reference's files to
    their printed precision, and the f32 snapshots have the reference's size."""
    params = sw.parameters.Parameters()
    params.numerical.grid_resolution = ng
    params.numerical.vertical_layers = nz
    params.numerical.time_step = dt
    params.numerical.duration = tsim
    params.environment.output_directory = str(tmp_path)
    sw.vstrip.init_pv_strip(params)
    sw.balinit.balinit(params)
    sw.swto3d.swto3d(params)
    sw.nhswps.nhswps(params)
    g = golden("complete")
    for name, tol in (("monitor.asc", 1.01e-6), ("ecomp.asc", 1.01e-9)):
        ref = np.array(bytes(g["%d_%d/%s" % (ng, nz, name)]).decode().split(), float)
        got = np.array(open(tmp_path / name).read().split(), float)
        assert got.shape == ref.shape, name
        np.testing.assert_allclose(got, ref, rtol=0, atol=tol, err_msg=name)
    for rel in ("3d/ql.r4", "2d/q.r4", "2d/h.r4"):
        key = "%d_%d/%s" % (ng, nz, rel)
        assert (tmp_path / rel).stat().st_size == g[key].size * 4, rel
    # the q snapshot frames agree with the reference's f32 output
    ref = g["%d_%d/2d/q.r4" % (ng, nz)]
    got = np.fromfile(tmp_path / "2d/q.r4", dtype="<f4")
    assert np.abs(got - ref).max() <= 2e-5 * max(1.0, np.abs(ref).max())


def test_d2fft_class_golden(sw):
    """sta2dfft's D2FFT (src/sta2dfft.rs:37-184) through the package's class: its
    trig tables equal initfft's, ptospc / spctop and the derivatives with the
    domain's own wavenumbers equal the reference's golden outputs, and a foreign
    wavenumber array is refused rather than ignored."""
    g = golden("sta2dfft")
    d = sw.sta2dfft.D2FFT(32, 32)
    f, trig = sw.stafft.initfft(32)
    assert np.array_equal(d.xtrig, trig) and list(d.xfactors) == list(f)
    s = np.zeros(32 * 32)
    _rel(d.ptospc(g["ptospc/ptospc_ng32_rvar.bin"], s), g["ptospc/ptospc_ng32_svar2.bin"])
    r = np.zeros(32 * 32)
    _rel(d.spctop(g["spctop/spctop_ng32_svar.bin"], r), g["spctop/spctop_ng32_rvar2.bin"])
    for which, case, ng in (("x", 1, 32), ("x", 2, 24), ("y", 1, 32), ("y", 2, 24)):
        dd = d if ng == 32 else sw.sta2dfft.D2FFT(ng, ng)
        var = g["deriv/%sderiv_%d_var.bin" % (which, case)]
        rk = g["deriv/%sderiv_%d_rk%s.bin" % (which, case, which)]
        out = np.zeros(ng * ng)
        (dd.xderiv if which == "x" else dd.yderiv)(rk, var, out)
        _close(out, g["deriv/%sderiv_%d_der2.bin" % (which, case)], 0.0)
    with pytest.raises(ValueError):
        d.xderiv(2.0 * d.kx, g["deriv/xderiv_1_var.bin"], np.zeros(32 * 32))
