"""PV-strip initial condition (reference src/vstrip.rs:8-124), host set-up code.

Builds the strip on a 16*ng grid and restricts it to ng x ng by repeated
nine-point averaging, exactly as the reference does, vectorised over y.
"""
import os

import numpy as np


def pv_strip(ng, strip_width=0.4, a2=0.02, a3=-0.01):
    """Zero-mean PV anomaly qq(ng, ng), flat in Fortran order (iy + ng*ix)."""
    ngu = 16 * ng
    qmax = 4.0 * np.pi
    hwid = strip_width / 2.0
    glu = 2.0 * np.pi / ngu
    x = glu * np.arange(ngu, dtype=np.float64) - np.pi
    y = glu * np.arange(ngu, dtype=np.float64) - np.pi
    y1 = -hwid
    y2 = hwid + a2 * np.sin(2.0 * x) + a3 * np.sin(3.0 * x)          # per column i
    prod = (y2[None, :] - y[:, None]) * (y[:, None] - y1)             # qa[j, i]
    qa = np.where(prod > 0.0, 4.0 * qmax * prod / (y2[None, :] - y1) ** 2, 0.0)
    ngh = ngu
    while ngh > ng:
        nguf = ngh
        ngh //= 2
        iy = np.arange(ngh)
        qod2 = qa[2 * iy, nguf - 1].copy()
        qev2 = np.empty(ngh + 1)
        qev2[1:] = qa[2 * iy + 1, nguf - 1]
        qev2[0] = qa[nguf - 1, nguf - 1]
        for ix in range(ngh):
            mix = 2 * (ix + 1)
            qod1 = qa[2 * iy, mix - 2].copy()
            qod0 = qa[2 * iy, mix - 1].copy()
            qev1 = np.empty(ngh + 1)
            qev0 = np.empty(ngh + 1)
            qev1[1:] = qa[2 * iy + 1, mix - 2]
            qev0[1:] = qa[2 * iy + 1, mix - 1]
            qev1[0] = qev1[ngh]
            qev0[0] = qev0[ngh]
            qa[:ngh, ix] = (0.0625 * (qev0[1:] + qev0[:-1] + qev2[1:] + qev2[:-1])
                            + 0.125 * (qev1[1:] + qev1[:-1] + qod0 + qod2) + 0.25 * qod1)
            qod2 = qod0
            qev2 = qev0
    block = qa[:ng, :ng]
    qavg = 0.0
    for ix in range(ng):
        for v in block[:, ix]:
            qavg += v
    qavg /= ng * ng
    return np.ascontiguousarray((block - qavg).reshape(-1, order="F"))


def init_pv_strip(parameters):
    """Write qq_init.r8 (8-byte header + field) and header-less zero dd/gg (vstrip.rs:108-121)."""
    num = parameters.numerical
    ng = num.grid_resolution
    d = str(parameters.environment.output_directory)
    os.makedirs(d, exist_ok=True)
    qq = pv_strip(ng, num.strip_width, num.a2, num.a3)
    np.concatenate([[0.0], qq]).astype("<f8").tofile(os.path.join(d, "qq_init.r8"))
    np.zeros(ng * ng, dtype="<f8").tofile(os.path.join(d, "dd_init.r8"))
    np.zeros(ng * ng, dtype="<f8").tofile(os.path.join(d, "gg_init.r8"))
