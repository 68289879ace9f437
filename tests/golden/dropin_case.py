"""Drop-in end-to-end case: the reference's own run() (HydroPlugin.cpp:74-321,
stock macros: theta 1.1, conformal a = 13.8997, shear only) on the lattice of
tests/golden/dropin_conf/ with initial-condition type 13 (an energy-density
vector, HydroWrapper.cpp:20-23).  The vector is a Gaussian blob,
20 GeV/fm^3 * exp(-r^2 / (2 * 1.5^2)) on the 41x41 grid.

Run as a script where the reference build (oracle/_ref) exists to regenerate
tests/golden/dropin_surface.json: row count and SHA-256 of the reference's
surface.dat for this case (the text itself is ~600 kB and not committed), and
the SHA-256 of every field dump the reference's run() writes
(outputDynamicalQuantities, HydroPlugin.cpp:40-71)."""
import ctypes as C
import hashlib
import json
import os
import shutil
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
CONF = os.path.join(HERE, "dropin_conf")
GOLDEN = os.path.join(HERE, "dropin_surface.json")
NX = NY = 41
DX = 0.2


def e_vector() -> np.ndarray:
    x = (np.arange(NX) - (NX - 1) / 2.0) * DX
    X, Y = np.meshgrid(x, x, indexing="ij")
    e = 20.0 * np.exp(-(X ** 2 + Y ** 2) / (2 * 1.5 ** 2))
    return np.ascontiguousarray(e.T.reshape(-1))   # index i + nx*j


def main():
    lib = C.CDLL(os.path.join(HERE, "..", "..", "oracle", "_ref", "libvhref_stock.so"))
    lib.vhref_threads(1)
    lib.vhref_load_conf(CONF.encode())
    e = e_vector()
    out = tempfile.mkdtemp()
    lib.vhref_run_vector.argtypes = [C.c_char_p, C.c_void_p, C.c_int]
    lib.vhref_run_vector(out.encode(), e.ctypes.data, len(e))
    with open(os.path.join(out, "surface.dat"), "rb") as f:
        d = f.read()
    dumps = {}
    for name in sorted(os.listdir(out)):
        if name != "surface.dat":
            with open(os.path.join(out, name), "rb") as f:
                dumps[name] = hashlib.sha256(f.read()).hexdigest()
    shutil.rmtree(out)
    with open(GOLDEN, "w") as f:
        json.dump({"rows": d.count(b"\n"), "sha256": hashlib.sha256(d).hexdigest(), "bytes": len(d),
                   "dumps": dumps,
                   "source": "reference run(), stock macros, tests/golden/dropin_conf, IC type 13 "
                             "(tests/golden/dropin_case.py)"}, f, indent=1)
    print("wrote", GOLDEN)


if __name__ == "__main__":
    sys.exit(main())
