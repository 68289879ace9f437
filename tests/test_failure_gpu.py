"""Failure reporting without a GPU fault: where the reference prints and
exits (a NaN energy density, EnergyMomentumTensor.cpp:197-203; a NaN
regulation factor, FullyDiscreteKurganovTadmorScheme.cpp:849), the device
records the first failing cell and step and the host reads VH_ERR_NAN; the
context stays usable and other events are unaffected."""
import numpy as np
import pytest

import vh

pytestmark = pytest.mark.gpu
VH_ERR_NAN = 4


def _poisoned(cfg, st):
    e = st.e.copy()
    e[len(e) // 2] = np.nan
    return vh.InitialState(e, st.p, st.u, st.pi, st.Pi)


def test_nan_is_reported_not_faulted():
    cfg = vh.gubser_config(21, 19)
    st = vh.gubser_ic(cfg)
    ev = vh.Event(cfg)
    ev.set_initial(_poisoned(cfg, st))
    ev.step(2)
    rc, step, cell = ev.status()
    assert rc == VH_ERR_NAN and step == 0
    ncx, ncy = cfg.nx + 4, cfg.ny + 4
    assert 0 <= cell < ncx * ncy * (cfg.nz + 4)
    # the context still works: a fresh initial state evolves cleanly
    ok = vh.Event(cfg)
    ok.set_initial(st)
    ok.step(3)
    assert ok.status()[0] == 0
    ev.set_initial(st)                   # a new initial state clears the event's error
    ev.step(1)
    assert ev.status()[0] == 0


def test_failing_batch_member_is_isolated():
    rows = vh.synthetic_eos_table()
    cfgs = [vh.hotspot_config(n) for n in (23, 29)]
    sts = [vh.hotspot_ic(c, rows, seed=70 + i) for i, c in enumerate(cfgs)]
    evs = [vh.Event(c, rows) for c in cfgs]
    evs[0].set_initial(_poisoned(cfgs[0], sts[0]))
    evs[1].set_initial(sts[1])
    ref = vh.Event(cfgs[1], rows)
    ref.set_initial(sts[1])
    b = vh.Batch(evs)
    b.step(3)
    ref.step(3)
    assert evs[0].status()[0] == VH_ERR_NAN
    assert evs[1].status()[0] == 0 and ref.status()[0] == 0
    a, r = evs[1].field(vh.VH_F_E), ref.field(vh.VH_F_E)
    assert np.array_equal(a.view(np.uint64), r.view(np.uint64))


def test_failed_batch_member_is_not_advanced():
    """a member whose device flagged an error is no longer computed while the
    batch goes on (its root solves would otherwise grind on garbage): its
    error and its energy density stay those of the failing step, and the
    other members advance as usual"""
    rows = vh.synthetic_eos_table()
    cfgs = [vh.hotspot_config(n) for n in (23, 29)]
    sts = [vh.hotspot_ic(c, rows, seed=80 + i) for i, c in enumerate(cfgs)]
    evs = [vh.Event(c, rows) for c in cfgs]
    evs[0].set_initial(_poisoned(cfgs[0], sts[0]))
    evs[1].set_initial(sts[1])
    b = vh.Batch(evs)
    b.step(2)
    assert evs[0].status()[0] == VH_ERR_NAN
    rc0, step0, cell0 = evs[0].status()
    frozen = evs[0].field(vh.VH_F_E).copy()
    b.step(3)
    assert evs[0].status() == (rc0, step0, cell0)
    assert np.array_equal(evs[0].field(vh.VH_F_E).view(np.uint64), frozen.view(np.uint64))
    ref = vh.Event(cfgs[1], rows)
    ref.set_initial(sts[1])
    ref.step(5)
    assert evs[1].status()[0] == 0
    assert np.array_equal(evs[1].field(vh.VH_F_E).view(np.uint64), ref.field(vh.VH_F_E).view(np.uint64))
