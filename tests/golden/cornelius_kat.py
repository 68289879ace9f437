"""Cornelius known-answer vectors.

The reference ships freezeout/cornelius-c++-1.3/output_{3d,4d}.dat, written
by its example_cornelius.cpp: 10^4 cubes (3D) and hypercubes (4D) whose corner
values are glibc rand()/RAND_MAX drawn in sequence from the default seed
(2D first, then 3D, then 4D), threshold 0.5, unit spacing; each element is
printed as centroid then normal at the ostream default precision (6
significant digits, "%g"), space-separated with a trailing space.

`random_cubes(dim)` regenerates those inputs; `format_elements` prints an
element array the same way.  Run as a script (where the reference tree is
available) to refresh tests/golden/cornelius_kat.json with the element counts
and SHA-256 of the reference files.
"""
import ctypes
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_KAT = os.path.join(os.environ.get("VH_REFERENCE", "/root/reference"), "freezeout/cornelius-c++-1.3")
RAND_MAX = 2147483647


def random_cubes(dim: int, n: int = 10000) -> np.ndarray:
    libc = ctypes.CDLL("libc.so.6")
    libc.rand.restype = ctypes.c_int
    libc.srand(1)
    skip = {2: 0, 3: 4 * n, 4: 4 * n + 8 * n}[dim]
    for _ in range(skip):
        libc.rand()
    per = 2 ** dim
    vals = np.array([libc.rand() / float(RAND_MAX) for _ in range(per * n)], dtype=np.float64)
    return vals.reshape(n, per)


def format_elements(el: np.ndarray) -> str:
    return "".join(" ".join("%g" % v for v in row) + " \n" for row in el)


def main():
    out = {}
    for dim in (3, 4):
        path = os.path.join(REF_KAT, f"output_{dim}d.dat")
        with open(path, "rb") as f:
            data = f.read()
        out[f"{dim}d"] = {"elements": data.count(b"\n"), "sha256": hashlib.sha256(data).hexdigest(),
                          "source": f"freezeout/cornelius-c++-1.3/output_{dim}d.dat"}
    with open(os.path.join(HERE, "cornelius_kat.json"), "w") as f:
        json.dump(out, f, indent=1)
    print(json.dumps(out, indent=1))


if __name__ == "__main__":
    sys.exit(main())
