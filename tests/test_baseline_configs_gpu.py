"""Bit-for-bit parity with the oracle on the benchmark configurations
themselves, not reduced lattices, and on the reference's shipped EoS.

* plain 2+1D Gubser flow, 101x101, the whole event: 300 RK2 steps with a
  freezeout block (T_F = 0.15 GeV) every fo_factor steps; every field at steps
  100, 200 and 300 and every element's 20 columns of every block;
* plain 3+1D Glauber event at its full 131x131x61 lattice (the headline
  workload): 6 RK2 steps and 3 freezeout blocks, every field and element;
* the HotQCD/HRG table the reference ships (EoS/hrg_hotqcd_eos_binary.dat,
  its first 2000 records committed in tests/golden/hotqcd_eos_prefix.npy;
  tests/test_oracle_vs_reference.py pins the oracle to the reference on the
  full table and the prefix to the full table), on a fused and a phase-split
  lattice, with the table sound-speed shortcut on and off.

The oracle (oracle/vh_oracle.c, cornelius_oracle.c) equals the reference's
own code bit for bit (tests/test_oracle_vs_reference.py)."""
import os
import sys

import numpy as np
import pytest

import vh
from oracle import OracleEvent

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import hotqcd_eos_prefix as HQ  # noqa: E402

FIELDS_14 = list(range(14)) + [100, 101, 102, 103, 200, 201]
FIELDS_15 = list(range(15)) + [100, 101, 102, 103, 200, 201]


def _bad_fields(cfg, gpu, orc, fields):
    bad = {}
    for f in fields:
        A, B = vh.face_cells(cfg, gpu.field(f)), vh.face_cells(cfg, orc.field(f))
        n = int(np.count_nonzero(A.view(np.uint64) != B.view(np.uint64)))
        if n:
            bad[f] = n
    return bad


def _block(gpu, orc, tag):
    ne, na = gpu.freezeout()
    el_g = gpu.surface()
    el_o, na_o = orc.freezeout()
    assert na == na_o, (tag, na, na_o)
    assert ne == len(el_o), (tag, ne, len(el_o))
    np.testing.assert_array_equal(el_g.view(np.uint64), el_o.view(np.uint64), err_msg=str(tag))
    return ne


def test_gubser_101_whole_event_with_freezeout():
    cfg = vh.gubser_config()
    assert (cfg.nx, cfg.ny, cfg.nz, cfg.T_freezeout_GeV) == (101, 101, 1, 0.15)
    st = vh.gubser_ic(cfg)
    gpu, orc = vh.Event(cfg), OracleEvent(cfg)
    gpu.set_initial(st)
    orc.set_initial(st)
    fac = cfg.fo_factor
    done, elements = 0, 0
    while done < 300:
        elements += _block(gpu, orc, ("block at step", done))
        gpu.step(fac)
        assert orc.step(fac) == 0
        done += fac
        if done % 100 == 0:
            gpu.sync()
            bad = _bad_fields(cfg, gpu, orc, FIELDS_14)
            assert not bad, f"after {done} steps, bit-differing cells per field: {bad}"
    assert elements > 10000
    assert gpu.powf_misses() == 0
    gpu.close()


def test_glauber_131x131x61_steps_and_freezeout():
    cfg = vh.glauber_config()
    assert (cfg.nx, cfg.ny, cfg.nz) == (131, 131, 61)
    rows = vh.synthetic_eos_table()
    st = vh.glauber_ic(cfg, rows)
    gpu, orc = vh.Event(cfg, rows), OracleEvent(cfg, rows)
    gpu.set_initial(st)
    orc.set_initial(st)
    assert gpu.launches_per_step() == 10          # the phase-split stage of the benchmark
    elements = 0
    for blk in range(3):
        elements += _block(gpu, orc, ("block", blk))
        gpu.step(2)
        assert orc.step(2) == 0
        gpu.sync()
        bad = _bad_fields(cfg, gpu, orc, FIELDS_15)
        assert not bad, f"after {2 * (blk + 1)} steps, bit-differing cells per field: {bad}"
    assert elements > 100000
    gpu.close()


@pytest.mark.parametrize("dims", [(19, 17, 7), (41, 39, 21)], ids=["fused", "split"])
@pytest.mark.parametrize("shortcut", ["on", "off"])
def test_hotqcd_table_bitexact(dims, shortcut, monkeypatch):
    if shortcut == "off":
        monkeypatch.setenv("VH_CS2_SHORTCUT", "0")
    rows = HQ.load_prefix()
    cfg = vh.glauber_config(*dims)
    cfg.dx = cfg.dy = 0.7 if dims[0] < 30 else 0.35
    cfg.dz = 0.5 if dims[0] < 30 else 0.2
    cfg.dt = 0.05 if dims[0] < 30 else 0.025
    st = vh.glauber_ic(cfg, rows)
    gpu, orc = vh.Event(cfg, rows), OracleEvent(cfg, rows)
    gpu.set_initial(st)
    orc.set_initial(st)
    assert gpu.launches_per_step() == (10 if dims[0] > 30 else 2)
    for blk in range(3):
        _block(gpu, orc, ("block", blk))
        gpu.step(3)
        assert orc.step(3) == 0
        gpu.sync()
        bad = _bad_fields(cfg, gpu, orc, FIELDS_15)
        assert not bad, f"block {blk}: bit-differing cells per field: {bad}"
    gpu.close()
