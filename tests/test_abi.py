"""CPU checks of the C ABI: the library builds for sm_100a, loads without a GPU
and exports every entry point include/sw_cuda.h declares."""
import ctypes
import os

import pytest

from conftest import PKG_DIR, load_package


def _lib_path():
    return os.path.join(PKG_DIR, "libswcuda.so")


def test_library_exports_header_symbols():
    sw = load_package()
    assert os.path.exists(_lib_path()), "build libswcuda.so first (python shallow-water_b200/build.py)"
    lib = ctypes.CDLL(_lib_path())
    declared = sw._native.declared_symbols()
    assert len(declared) >= 40
    missing = [s for s in declared if not hasattr(lib, s)]
    assert not missing, missing
    # every declared symbol has a ctypes signature in the binding
    assert set(declared) <= set(sw._native._SIGS), set(declared) - set(sw._native._SIGS)


def test_host_only_entry_points(sw):
    """factorisen/initfft run on the host and need no device."""
    assert sw.stafft.factorisen(16) == [0, 2, 0, 0, 0]
    assert sw.stafft.factorisen(8640) == [3, 1, 1, 0, 1]
    with pytest.raises(sw.SwError) as e:
        sw.stafft.factorisen(14)
    assert e.value.status == sw._native.SW_ERR_FACTORISE


def test_initfft_matches_golden(sw):
    import numpy as np
    from conftest import golden
    for n in (18, 30, 32):
        _, trig = sw.stafft.initfft(n)
        np.testing.assert_allclose(trig, golden("stafft")["initfft/%d_trig.bin" % n], rtol=0, atol=1e-13)


def test_no_device_reports_error(sw):
    """Without a GPU, creating a context fails loudly (no CPU fallback)."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = ctypes.c_void_p()
    st = sw._native.lib().sw_ctx_create(32, 4, 1, 0, 0, ctypes.byref(h))
    assert st != 0
