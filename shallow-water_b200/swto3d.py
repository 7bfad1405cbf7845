"""Replicate the 2-D balanced fields over the nz+1 levels (reference src/swto3d.rs:10-39)."""
import os

import numpy as np


def swto3d_arrays(nz, qq, dd, gg):
    return tuple(np.tile(np.asarray(a, np.float64).reshape(-1, order="F"), nz + 1) for a in (qq, dd, gg))


def swto3d(parameters):
    ng = parameters.numerical.grid_resolution
    nz = parameters.numerical.vertical_layers
    d = str(parameters.environment.output_directory)
    raw = np.fromfile(os.path.join(d, "sw_init.r8"), dtype="<f8").reshape(3, ng * ng + 1)[:, 1:]
    for name, arr in zip(("qq", "dd", "gg"), swto3d_arrays(nz, *raw)):
        np.concatenate([[0.0], arr]).astype("<f8").tofile(os.path.join(d, name + "_init.r8"))
