"""Workload of the bounds-check test (tests/test_gpu_bounds_check.py): the hot
path on small grids through the C ABI, returning the results as named float64
arrays.  Run as a script with SW_CUDA_LIB_VARIANT=bc it exercises the
bounds-check debug build (libswcuda_bc.so) in a child process and saves the
arrays to the .npz given as its argument; any call that returns an error status
(an access outside the registered allocations included) raises."""
import ctypes
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _package():
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from conftest import load_package
    return load_package()


def _ensemble(sw, ng, nz, M, prec, seed0):
    qq = sw.vstrip.pv_strip(ng)
    sp = sw.Spectral(ng, nz, precision=prec, nmembers=M)
    z3 = np.zeros(ng * ng * (nz + 1))
    for m in range(M):
        rng = np.random.default_rng(seed0 + m)
        q3 = np.tile(qq, nz + 1) + rng.normal(0.0, 1.0e-3, ng * ng * (nz + 1))
        sw.nhswps.initial_state(sp, q3, z3, z3, member=m, invert=False)
    sw.nhswps.main_invert_all(sp)
    return sp


def _get(sw, sp, member, key):
    a = np.zeros(sp.n3)
    sw._native.check(sw._native.lib().sw_state_get(sp.ctx, sw._native.FIELD_INDEX[key], member,
                                                   sw._native.dptr(a), sp.n3))
    return a


def run(sw):
    import torch
    L = sw._native.lib()
    out = {}
    # steps of every precision on a two-member ensemble: graph-launched, then host-driven
    for name, prec in (("fp64", sw.SW_FP64), ("mixed", sw.SW_MIXED), ("fp32", sw.SW_FP32)):
        sp = _ensemble(sw, 32, 4, 2, prec, 7)
        sw._native.check(L.sw_advance(sp.ctx, 2, 1))
        sw._native.check(L.sw_set_graphs(sp.ctx, 0))
        sw._native.check(L.sw_advance(sp.ctx, 1, 1))
        for k in ("qs", "ds", "gs", "pn"):
            out["%s_%s" % (name, k)] = _get(sw, sp, 1, k)
        sp.close()
    # the reference's one-function-at-a-time entry points (their own kernels, not
    # the fused step's), on a float64 and a float32 context
    for name, prec in (("fn64", sw.SW_FP64), ("fn32", sw.SW_FP32)):
        sp = _ensemble(sw, 32, 4, 1, prec, 11)
        st = sw.State(sp, member=0)
        sw.nhswps.vertical(st)
        sig = sw.nhswps.coeffs(st)
        sp0 = sw.nhswps.cpsource(st)
        sw.nhswps.psolve(st)
        src = sw.nhswps.source(st)
        out["%s_sigx" % name] = sig[0]
        out["%s_sp0" % name] = sp0
        out["%s_sgs" % name] = src[2]
        out["%s_pn" % name] = _get(sw, sp, 0, "pn")
        sp.close()
    # an uneven ensemble: two (ng, nz) groups advanced by one graph launch per step
    draws = [(32, 4), (48, 4), (32, 4)]
    ens = sw.nhswps.Ensemble([d[0] for d in draws], [d[1] for d in draws], precision=sw.SW_MIXED)
    for k, (ng, nz) in enumerate(draws):
        qq = sw.vstrip.pv_strip(ng)
        rng = np.random.default_rng(300 + k)
        q3 = np.tile(qq, nz + 1) + rng.normal(0.0, 1.0e-3, ng * ng * (nz + 1))
        ens.initial_state(k, q3, np.zeros_like(q3), np.zeros_like(q3))
    ens.invert_all()
    ens.advance(2)
    for k in range(len(draws)):
        out["mixed_ens%d_gs" % k] = ens.state(k).get("gs").ravel(order="F")
    ens.close()
    # a length served by the generic tile pass, and the savegrid outputs
    sp = _ensemble(sw, 48, 8, 1, sw.SW_FP64, 3)
    sw._native.check(L.sw_advance(sp.ctx, 1, 1))
    st = sw.State.__new__(sw.State)
    object.__setattr__(st, "spectral", sp)
    object.__setattr__(st, "member", 0)
    energies, spec, f3, f2 = sw.nhswps.savegrid_data(st)
    out["ng48_gs"] = _get(sw, sp, 0, "gs")
    out["ng48_energies"] = np.asarray(energies, dtype=np.float64)
    out["ng48_spectra"] = np.asarray(spec, dtype=np.float64).ravel()
    out["ng48_f3"] = np.concatenate([np.asarray(f3[k], dtype=np.float64) for k in sorted(f3)])
    out["ng48_f2"] = np.concatenate([np.asarray(f2[k], dtype=np.float64) for k in sorted(f2)])
    sp.close()
    # batched 2-D transforms on caller buffers (n = 96 generic, n = 256 register-staged)
    for ng in (96, 256):
        sp = sw.Spectral(ng, 2)
        torch.manual_seed(ng)
        a = torch.randn(3 * ng * ng, dtype=torch.float64, device="cuda")
        b = torch.empty_like(a)
        c = torch.empty_like(a)
        sw._native.check(L.sw_fft2d_dev(sp.ctx, 0, 3, ctypes.c_void_p(a.data_ptr()), ctypes.c_void_p(b.data_ptr())))
        sw._native.check(L.sw_fft2d_dev(sp.ctx, 1, 3, ctypes.c_void_p(b.data_ptr()), ctypes.c_void_p(c.data_ptr())))
        sw._native.check(L.sw_sync(sp.ctx))
        out["fft2d_%d_in" % ng] = a.cpu().numpy()
        out["fft2d_%d_spec" % ng] = b.cpu().numpy()
        out["fft2d_%d_back" % ng] = c.cpu().numpy()
        sp.close()
    torch.cuda.synchronize()
    return out


if __name__ == "__main__":
    res = run(_package())
    np.savez(sys.argv[1], **res)
    print("bounds-check workload ok: %d arrays" % len(res))
