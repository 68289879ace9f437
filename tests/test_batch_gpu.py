"""Batched evolution (vh_batch_*): members of different sizes advanced with one
launch per RK phase must equal, bit for bit, the oracle and the single-event
path, for every launch configuration the autotuner can pick."""
import numpy as np
import pytest

import vh
from oracle import OracleEvent

pytestmark = pytest.mark.gpu

FIELDS_15 = list(range(15)) + [100, 101, 102, 103, 200, 201]


def _bits(a):
    return np.ascontiguousarray(a).view(np.uint64)


def _diff(cfg, a, b):
    return int(np.count_nonzero(_bits(vh.face_cells(cfg, a)) != _bits(vh.face_cells(cfg, b))))


def _compare(cfg, x, y):
    bad = {}
    for f in FIELDS_15:
        n = _diff(cfg, x.field(f), y.field(f))
        if n:
            bad[f] = n
    return bad


def _hotspot_members(sizes, rows, seed0=11):
    cfgs = [vh.hotspot_config(n) for n in sizes]
    ics = [vh.hotspot_ic(c, rows, seed=seed0 + i) for i, c in enumerate(cfgs)]
    return cfgs, ics


def _events(cfgs, ics, rows):
    evs = []
    for c, st in zip(cfgs, ics):
        e = vh.Event(c, rows)
        e.set_initial(st)
        evs.append(e)
    return evs


def test_batch_matches_oracle():
    rows = vh.synthetic_eos_table()
    cfgs, ics = _hotspot_members([21, 33, 40], rows)
    evs = _events(cfgs, ics, rows)
    b = vh.Batch(evs)
    b.step(6)
    t = b.tuning()
    assert t.stage_ms > 0
    for c, st, e in zip(cfgs, ics, evs):
        e.sync()
        o = OracleEvent(c, rows)
        o.set_initial(st)
        assert o.step(6) == 0
        bad = _compare(c, e, o)
        assert not bad, f"{c.nx}x{c.ny}: bit-differing cells per field {bad} (tuning {t.describe()})"
        assert e.progress()[0] == 6
        assert e.powf_misses() == 0


@pytest.mark.parametrize("fused", [False, True])
@pytest.mark.parametrize("tx,persistent", [(32, False), (32, True), (8, False), (128, True), (64, False), (16, True)])
def test_every_tuning_equals_single_event_path(fused, tx, persistent):
    rows = vh.synthetic_eos_table()
    cfgs, ics = _hotspot_members([19, 27], rows, seed0=3)
    evs = _events(cfgs, ics, rows)
    ref = _events(cfgs, ics, rows)
    b = vh.Batch(evs)
    b.set_tuning(vh.make_tuning(fused, tx, persistent))
    b.step(3)
    for c, e, r in zip(cfgs, evs, ref):
        r.step(3)
        e.sync()
        r.sync()
        bad = _compare(c, e, r)
        assert not bad, f"{c.nx}x{c.ny} fused={fused} {tx}x{128 // tx} persistent={persistent}: {bad}"


def test_mixed_2d_3d_batch_and_interleaved_single_steps():
    rows = vh.synthetic_eos_table()
    g = vh.glauber_config(13, 11, 5)
    g.dx = g.dy = 0.5
    g.dz = 0.4
    g.dt = 0.05
    h = vh.hotspot_config(23)
    cfgs = [g, h]
    ics = [vh.glauber_ic(g, rows), vh.hotspot_ic(h, rows, seed=5)]
    evs = _events(cfgs, ics, rows)
    ref = _events(cfgs, ics, rows)
    b = vh.Batch(evs)
    b.step(3)
    evs[0].step(2)           # a member may be stepped alone between batch steps
    b.step(2)
    ref[0].step(7)
    ref[1].step(5)
    for c, e, r in zip(cfgs, evs, ref):
        e.sync()
        r.sync()
        bad = _compare(c, e, r)
        assert not bad, f"{c.nx}x{c.ny}x{c.nz}: {bad}"
    assert evs[0].progress()[0] == 7 and evs[1].progress()[0] == 5


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_inactive_member_is_frozen(precision):
    """an inactive member does not move (its tiles are skipped in every phase,
    the mixed face-once flux included) and resumes where it stopped: its
    state equals that of the same event stepped as often in a batch of its
    own, and the other members equal a batch without it"""
    rows = vh.synthetic_eos_table()
    cfgs, ics = _hotspot_members([17, 25, 21], rows, seed0=21)
    if precision == "mixed":
        cfgs = [c.copy(precision=vh.VH_PREC_MIXED) for c in cfgs]
    evs = _events(cfgs, ics, rows)
    b = vh.Batch(evs)
    b.step(2)
    evs[1].sync()
    before = evs[1].field(vh.VH_F_E).copy()
    b.set_active(1, False)
    b.step(3)
    evs[1].sync()
    assert np.array_equal(_bits(evs[1].field(vh.VH_F_E)), _bits(before))
    assert evs[1].progress()[0] == 2
    b.set_active(1, True)
    b.step(1)
    ref_a = _events([cfgs[0], cfgs[2]], [ics[0], ics[2]], rows)
    ref_b = _events([cfgs[1]], [ics[1]], rows)
    ba, bb = vh.Batch(ref_a), vh.Batch(ref_b)
    ba.step(6)
    bb.step(3)
    for c, e, r in ((cfgs[0], evs[0], ref_a[0]), (cfgs[1], evs[1], ref_b[0]), (cfgs[2], evs[2], ref_a[1])):
        e.sync()
        r.sync()
        assert e.status()[0] == 0
        assert not _compare(c, e, r)
    if precision == "fp64":
        singles = _events(cfgs, ics, rows)
        for c, e, r, n in zip(cfgs, evs, singles, [6, 3, 6]):
            r.step(n)
            r.sync()
            assert not _compare(c, e, r)


def test_freezeout_of_batched_member():
    rows = vh.synthetic_eos_table()
    cfgs, ics = _hotspot_members([31, 29], rows, seed0=40)
    evs = _events(cfgs, ics, rows)
    ref = _events(cfgs, ics, rows)
    b = vh.Batch(evs)
    for e, r in zip(evs, ref):
        e.freezeout()
        r.freezeout()
    for _ in range(3):
        b.step(2)
        for e, r in zip(evs, ref):
            r.step(2)
            ne, na = e.freezeout()
            me, ma = r.freezeout()
            assert (ne, na) == (me, ma)
            assert np.array_equal(_bits(e.surface()), _bits(r.surface()))


def test_batch_rejects_mixed_eos():
    rows = vh.synthetic_eos_table()
    a = vh.Event(vh.hotspot_config(15), rows)
    c = vh.Event(vh.gubser_config(15, 15))
    a.set_initial(vh.hotspot_ic(a.cfg, rows, seed=1))
    c.set_initial(vh.gubser_ic(c.cfg))
    with pytest.raises(vh.VhError):
        vh.Batch([a, c])
    with pytest.raises(vh.VhError):
        vh.Batch([a, a])


def test_launch_count_and_phase_timing():
    rows = vh.synthetic_eos_table()
    cfgs, ics = _hotspot_members([41, 61], rows, seed0=60)
    evs = _events(cfgs, ics, rows)
    b = vh.Batch(evs)
    t = b.autotune()
    per = b.launches_per_step()
    assert per == (3 if t.fused else 9)
    b.phase_timing(True)
    b.step(2)
    ph = b.phase_times()
    b.phase_timing(False)
    assert sum(n for _, n in ph.values()) == 2 * (per - 1)
    assert all(ms > 0 for ms, _ in ph.values())
