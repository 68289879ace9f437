"""The device freezeout (Cornelius cube scan + surface append) against the
oracle and against the reference's Cornelius known-answer files.

Surface elements are compared as raw IEEE-754 bit patterns: the device
performs the reference's arithmetic in the reference's order, so the element
count, order and all 20 columns must match exactly."""
import hashlib
import json
import os
import sys

import numpy as np
import pytest

import vh
from oracle import OracleEvent

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import cornelius_kat as K  # noqa: E402


@pytest.mark.parametrize("dim", [3, 4])
def test_device_cornelius_known_answers(dim):
    with open(os.path.join(HERE, "golden", "cornelius_kat.json")) as f:
        gold = json.load(f)[f"{dim}d"]
    cubes = K.random_cubes(dim)
    el, counts = vh.cornelius_surfaces(dim, cubes, 0.5, np.ones(dim))
    assert len(el) == gold["elements"]
    assert hashlib.sha256(K.format_elements(el).encode()).hexdigest() == gold["sha256"]


def _run_blocks(cfg, rows, st, blocks):
    gpu, orc = vh.Event(cfg, rows), OracleEvent(cfg, rows)
    gpu.set_initial(st)
    orc.set_initial(st)
    total = 0
    for b in range(blocks):
        ne, na = gpu.freezeout()
        el_g = gpu.surface()
        el_o, na_o = orc.freezeout()
        assert na == na_o, (b, na, na_o)
        assert ne == len(el_o), (b, ne, len(el_o))
        np.testing.assert_array_equal(el_g.view(np.uint64), el_o.view(np.uint64), err_msg=f"block {b}")
        total += ne
        gpu.step(cfg.fo_factor)
        orc.step(cfg.fo_factor)
    gpu.sync()
    return total


# the element buffer's first size: the library's estimate, or one so small
# that blocks overflow it and are emitted again into a larger buffer
CAPS = [None, "1", "200"]


@pytest.mark.parametrize("initial_cap", CAPS)
def test_freezeout_gubser_2p1d_bitexact(initial_cap, monkeypatch):
    if initial_cap:
        monkeypatch.setenv("VH_FO_INITIAL_CAP", initial_cap)
    cfg = vh.gubser_config(41, 37)
    cfg.T_freezeout_GeV = 0.2
    assert _run_blocks(cfg, None, vh.gubser_ic(cfg), 5) > 0


@pytest.mark.parametrize("initial_cap", CAPS)
def test_freezeout_glauber_3p1d_bitexact(initial_cap, monkeypatch):
    if initial_cap:
        monkeypatch.setenv("VH_FO_INITIAL_CAP", initial_cap)
    cfg = vh.glauber_config(21, 19, 7)
    cfg.dx = cfg.dy = 0.6
    cfg.dz = 0.5
    cfg.dt = 0.05
    rows = vh.synthetic_eos_table()
    assert _run_blocks(cfg, rows, vh.glauber_ic(cfg, rows), 4) > 0
