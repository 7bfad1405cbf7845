"""Float64 rounding spread of a multi-step oracle run: rel-L2 between two runs of
the oracle that differ only in the radix schedule of their transforms
(oracle.set_fft_order 0 and 1).  The GPU tests judge the FP64 path against 3x
this spread; the table of the ng=256 test (SPREAD_256 in test_gpu_batching.py)
was made with

    python tests/golden/oracle_spread.py 256 16 10

Input: the vstrip PV strip on every level + N(0, 1e-3) per point (seed 1),
delta = gamma = 0, `steps` advance steps.
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)


def spread(ng, nz, steps):
    from oracle import oracle as orc
    qq = orc.vstrip(ng)
    rng = np.random.default_rng(1)
    q3 = np.tile(qq, nz + 1) + rng.normal(0.0, 1.0e-3, ng * ng * (nz + 1))
    z3 = np.zeros_like(q3)
    runs = []
    for order in (0, 1):
        orc.set_fft_order(order)
        try:
            sp, st = orc.initial_state(ng, nz, q3, z3, z3)
            for _ in range(steps):
                assert orc.advance(sp, st, ggen=True)[0] == 0
        finally:
            orc.set_fft_order(0)
        runs.append(st.f)
    return {k: float(np.linalg.norm(runs[1][k] - runs[0][k]) / max(np.linalg.norm(runs[0][k]), 1e-300))
            for k in ("qs", "u", "v", "z", "pn", "ds", "gs")}


if __name__ == "__main__":
    ng, nz, steps = (int(a) for a in sys.argv[1:4])
    print({k: "%.2e" % v for k, v in spread(ng, nz, steps).items()})
