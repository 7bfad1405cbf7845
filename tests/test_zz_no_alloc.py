"""The allocation-free 2-D transform entry point, sw_fft2d_noalloc.

It exists for callers that cannot allocate device memory where they transform
(a plugin inside a framework that owns the device memory, code recorded into
someone else's CUDA graph, allocation-free real-time loops).  The test calls it
through the C ABI with caller-owned device buffers and checks it against the
context-based sw_fft2d_dev and the FP64 oracle on two calls in a row (forward,
then reverse) for lengths served by both tile passes, with more planes than its
fixed scratch holds at once, plus the rejection of bad sizes and arguments.  This
file is collected last so that a failure here cannot stop the rest of the GPU
suite from running.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


# (ng, planes): the generic tile pass (64, 96, 512, 1024) and the register-staged
# n = 256 pass; 256 with 40 planes and 1024 with 3 planes exceed what the 16 MiB
# scratch holds at once (31 and 1 planes), so those calls run in chunks
CASES = [(64, 5), (96, 4), (256, 40), (512, 3), (1024, 3)]


@pytest.mark.parametrize("ng,planes", CASES)
def test_noalloc_matches_context_transform_and_oracle(sw, oracle, ng, planes):
    import torch
    L = sw._native.lib()
    sp = sw.Spectral(ng, 2)
    torch.manual_seed(ng)
    a = torch.randn(planes * ng * ng, dtype=torch.float64, device="cuda")
    ref = torch.empty_like(a)
    got = torch.empty_like(a)
    stream = torch.cuda.current_stream().cuda_stream
    torch.cuda.synchronize()
    # call 1: forward (ptospc)
    sw._native.check(L.sw_fft2d_dev(sp.ctx, 0, planes, _ptr(a), _ptr(ref)))
    sw._native.check(L.sw_sync(sp.ctx))
    sw._native.check(L.sw_fft2d_noalloc(ng, 0, planes, _ptr(a), _ptr(got), ctypes.c_void_p(stream)))
    torch.cuda.synchronize()
    r, g = ref.cpu().numpy(), got.cpu().numpy()
    assert np.abs(g - r).max() <= 1e-13 * np.abs(r).max()
    # the last plane against the FP64 oracle's ptospc (independent butterflies)
    n2 = ng * ng
    osp = oracle.Spectral(ng, 2)
    last = slice((planes - 1) * n2, planes * n2)
    o = osp.ptospc(a.cpu().numpy()[last])
    assert np.abs(g[last] - o).max() <= 1e-13 * np.abs(o).max()
    # call 2: reverse (spctop) of the forward result
    back_ref = torch.empty_like(a)
    back = torch.empty_like(a)
    sw._native.check(L.sw_fft2d_dev(sp.ctx, 1, planes, _ptr(ref), _ptr(back_ref)))
    sw._native.check(L.sw_sync(sp.ctx))
    sw._native.check(L.sw_fft2d_noalloc(ng, 1, planes, _ptr(got), _ptr(back), ctypes.c_void_p(stream)))
    torch.cuda.synchronize()
    r, g = back_ref.cpu().numpy(), back.cpu().numpy()
    assert np.abs(g - r).max() <= 1e-13 * np.abs(r).max()
    assert np.abs(g - a.cpu().numpy()).max() <= 1e-12  # round trip restores the input
    sp.close()


def test_noalloc_rejects_bad_arguments(sw):
    import torch
    L = sw._native.lib()
    buf = torch.zeros(16, dtype=torch.float64, device="cuda")
    st = L.sw_fft2d_noalloc(2048, 0, 1, _ptr(buf), _ptr(buf), None)
    assert st == sw._native.SW_ERR_ARG
    assert b"1024" in L.sw_last_error()
    assert L.sw_fft2d_noalloc(34, 0, 1, _ptr(buf), _ptr(buf), None) == sw._native.SW_ERR_FACTORISE
    assert L.sw_fft2d_noalloc(33, 0, 1, _ptr(buf), _ptr(buf), None) == sw._native.SW_ERR_ARG
    assert L.sw_fft2d_noalloc(64, 2, 1, _ptr(buf), _ptr(buf), None) == sw._native.SW_ERR_ARG
    assert L.sw_fft2d_noalloc(64, 0, 0, _ptr(buf), _ptr(buf), None) == sw._native.SW_ERR_ARG
