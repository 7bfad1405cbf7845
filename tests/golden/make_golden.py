"""Pack the reference's golden test vectors into compressed ``.npz`` fixtures.

The reference (rse-standrewscs/shallow-water, Rust) ships its unit-test
fixtures as raw binary files next to the code that uses them:

* ``*.bin``  big-endian float64, Fortran order (``src/utils.rs:81-107``)
* ``*.r8``   little-endian float64 with one 8-byte header word per record
             (``src/vstrip.rs:108-121``, ``src/balinit.rs:423-435``)
* ``*.r4``   little-endian float32 frames ``[t, field...]``
             (``src/nhswps/mod.rs:654-663``)
* ``*.asc``  text output (``monitor.asc``/``ecomp.asc``)

This script reads them from a checkout of the reference and writes one
``.npz`` per reference module into this directory, converted to native
float64 arrays (float32 for ``.r4``), flat, keyed by the fixture's path
relative to its ``testdata`` directory.  Text files are stored as uint8
byte arrays.  The large ``advance/128_16`` bench-only state is skipped.

Usage:  python tests/golden/make_golden.py [REFERENCE_ROOT]
"""
import os
import sys

import numpy as np

GROUPS = {
    "stafft": "src/stafft/testdata",
    "sta2dfft": "src/testdata",          # ptospc/spctop/deriv/init2dfft + IC files
    "spectral": "src/spectral/testdata",
    "nhswps": "src/nhswps/testdata",
}
SKIP_DIRS = ("128_16", "complete")


def _read(path):
    raw = open(path, "rb").read()
    if path.endswith(".bin"):
        return np.frombuffer(raw, dtype=">f8").astype(np.float64)
    if path.endswith(".r8"):
        return np.frombuffer(raw, dtype="<f8").astype(np.float64)
    if path.endswith(".r4"):
        return np.frombuffer(raw, dtype="<f4").astype(np.float32)
    return np.frombuffer(raw, dtype=np.uint8).copy()


def pack(root, outdir):
    for name, rel in GROUPS.items():
        base = os.path.join(root, rel)
        arrays = {}
        for dirpath, _, files in os.walk(base):
            if any(s in dirpath for s in SKIP_DIRS):
                continue
            for f in sorted(files):
                p = os.path.join(dirpath, f)
                key = os.path.relpath(p, base).replace(os.sep, "/")
                arrays[key] = _read(p)
        np.savez_compressed(os.path.join(outdir, name + ".npz"), **arrays)
        print(name, len(arrays), "arrays")
    # end-to-end outputs (src/test.rs:11-43): monitor/ecomp text and r4 frames
    arrays = {}
    base = os.path.join(root, "src/testdata/complete")
    for dirpath, _, files in os.walk(base):
        for f in sorted(files):
            p = os.path.join(dirpath, f)
            arrays[os.path.relpath(p, base).replace(os.sep, "/")] = _read(p)
    np.savez_compressed(os.path.join(outdir, "complete.npz"), **arrays)
    print("complete", len(arrays), "arrays")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py REFERENCE_CHECKOUT")
    pack(sys.argv[1], os.path.dirname(os.path.abspath(__file__)))
