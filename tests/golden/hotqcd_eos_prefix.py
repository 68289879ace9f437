"""Writes tests/golden/hotqcd_eos_prefix.npy: the first 2000 records (e, P, s,
T; e up to 37.7 GeV/fm^3) of the reference's shipped equation of state,
EoS/hrg_hotqcd_eos_binary.dat (HotQCD lattice matched to a hadron resonance
gas; 100 000 records of 4 doubles, read by EquationOfState.cpp:292-327).

The GPU box has no copy of the reference tree, so the device tests on the
shipped EoS run on this prefix, which covers every energy density the test
events reach (their initial peak is 30 GeV/fm^3).  On the CPU, where the full
table is present, tests/test_oracle_vs_reference.py checks the oracle against
the reference's own code on the full table, and that the evolution on the
prefix equals the evolution on the full table bit for bit.

    python tests/golden/hotqcd_eos_prefix.py   # needs VH_REFERENCE or /root/reference
"""
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "hotqcd_eos_prefix.npy")
ROWS = 2000


def full_table_path() -> str:
    return os.path.join(os.environ.get("VH_REFERENCE", "/root/reference"), "EoS", "hrg_hotqcd_eos_binary.dat")


def load_full() -> np.ndarray:
    return np.fromfile(full_table_path(), dtype=np.float64).reshape(-1, 4)


def load_prefix() -> np.ndarray:
    return np.load(OUT)


if __name__ == "__main__":
    np.save(OUT, np.ascontiguousarray(load_full()[:ROWS]))
    print("wrote", OUT)
