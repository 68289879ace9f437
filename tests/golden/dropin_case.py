"""Drop-in end-to-end case: the reference's own run() (HydroPlugin.cpp:74-321,
stock macros: theta 1.1, conformal a = 13.8997, shear only) on the lattice of
tests/golden/dropin_conf/ (2+1D, 41x41) and tests/golden/dropin_conf_3d/ (3+1D,
25x25x11) with initial-condition type 13 (an energy-density vector,
HydroWrapper.cpp:20-23): Gaussian blobs, 20 GeV/fm^3 * exp(-r^2 / (2 * 1.5^2))
in 2+1D and 20 GeV/fm^3 * exp(-r^2 / (2 * 1.2^2) - eta^2 / (2 * 0.9^2)) in 3+1D.

Run as a script where the reference build (oracle/_ref) exists to regenerate
tests/golden/dropin_surface.json and dropin_surface_3d.json: row count and
SHA-256 of the reference's surface.dat for each case (the text itself is ~600 kB and not committed), and
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

# case -> configuration directory, golden file, Gaussian blob of the IC vector:
# peak (GeV/fm^3) * exp(-(x^2 + y^2) / (2 w^2) - eta^2 / (2 w_eta^2))
CASES = {
    "2p1d": {"conf": os.path.join(HERE, "dropin_conf"), "golden": os.path.join(HERE, "dropin_surface.json"),
             "n": (41, 41, 1), "dx": 0.2, "deta": 0.1, "peak": 20.0, "w": 1.5, "w_eta": None},
    "3p1d": {"conf": os.path.join(HERE, "dropin_conf_3d"), "golden": os.path.join(HERE, "dropin_surface_3d.json"),
             "n": (25, 25, 11), "dx": 0.3, "deta": 0.3, "peak": 20.0, "w": 1.2, "w_eta": 0.9},
}
CONF = CASES["2p1d"]["conf"]
GOLDEN = CASES["2p1d"]["golden"]


def e_vector(case: str = "2p1d") -> np.ndarray:
    """the initial energy density, interior index i + nx*(j + ny*k)
    (InitialConditions.cpp:1606-1617)"""
    c = CASES[case]
    nx, ny, nz = c["n"]
    x = (np.arange(nx) - (nx - 1) / 2.0) * c["dx"]
    y = (np.arange(ny) - (ny - 1) / 2.0) * c["dx"]
    z = (np.arange(nz) - (nz - 1) / 2.0) * c["deta"]
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    e = c["peak"] * np.exp(-(X ** 2 + Y ** 2) / (2 * c["w"] ** 2))
    if c["w_eta"]:
        e = e * np.exp(-Z ** 2 / (2 * c["w_eta"] ** 2))
    return np.ascontiguousarray(e.reshape(-1))


def make_golden(case: str):
    c = CASES[case]
    lib = C.CDLL(os.path.join(HERE, "..", "..", "oracle", "_ref", "libvhref_stock.so"))
    lib.vhref_threads(1)
    lib.vhref_load_conf(c["conf"].encode())
    e = e_vector(case)
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
    with open(c["golden"], "w") as f:
        json.dump({"rows": d.count(b"\n"), "sha256": hashlib.sha256(d).hexdigest(), "bytes": len(d),
                   "dumps": dumps,
                   "source": f"reference run(), stock macros, {os.path.basename(c['conf'])}, IC type 13 "
                             f"(tests/golden/dropin_case.py, case {case})"}, f, indent=1)
    print("wrote", c["golden"], d.count(b"\n"), "rows")


def main():
    for case in (sys.argv[1:] or list(CASES)):
        make_golden(case)


if __name__ == "__main__":
    sys.exit(main())
