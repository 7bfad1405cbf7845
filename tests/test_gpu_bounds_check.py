"""The bounds-check debug build, libswcuda_bc.so (-DSW_BOUNDS_CHECK; built by
__graft_entry__.build() and `python shallow-water_b200/build.py --bounds-check`).

In that build every device access through the library's shared access helpers is
checked against the registered device allocations and its alignment; a failing
access is skipped (so the debug build never touches memory outside them) and the
entry point returns SW_ERR_CUDA with the first failing address.  It stands in for
a memory checker on the kernels' index arithmetic.

The workload (tests/bc_workload.py: steps of every precision, graph-launched and
host-driven, on a two-member ensemble; the one-function-at-a-time entry points
vertical, coeffs, cpsource, psolve and source; an uneven ensemble of two grids; a
generic-length grid with savegrid; 2-D transforms of caller buffers at n = 96 and
256) runs in a child process on the debug build, because this process has the
plain library loaded.  Every call must
succeed, and the results must equal the plain library's to rounding: the checks
add branches around the accesses, and the compiler may then contract a product and
a sum into one rounding at other places than in the plain build.  Bounds: 1e-10
for float64 results (measured 1.3e-12 on gamma, a small residual field, at ng=48),
1e-6 for the mixed and float32 runs, 1e-4 for the float32 per-function psolve, whose
stop rule (1e-6 or stagnation) may end one sweep apart."""
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_bounds_check_build_runs_the_hot_path_clean(sw, tmp_path):
    lib_bc = os.path.join(ROOT, "shallow-water_b200", "libswcuda_bc.so")
    assert os.path.exists(lib_bc), "libswcuda_bc.so not built (python shallow-water_b200/build.py --bounds-check)"
    out = str(tmp_path / "bc.npz")
    env = dict(os.environ, SW_CUDA_LIB_VARIANT="bc")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "tests", "bc_workload.py"), out], env=env,
                       capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-4000:]
    got = dict(np.load(out))
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import bc_workload
    ref = bc_workload.run(sw)
    assert set(got) == set(ref)
    for k in ref:
        a, b = got[k], ref[k]
        scale = max(np.abs(b).max(), 1e-300)
        # float32 pressure iterations may stop one sweep apart (stop rule 1e-6)
        tol = 1e-4 if k.startswith("fn32_") else 1e-6 if k.startswith(("mixed_", "fp32_")) else 1e-10
        assert np.abs(a - b).max() <= tol * scale, (k, np.abs(a - b).max() / scale)
