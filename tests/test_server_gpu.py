"""The event server (vh_server_*): events submitted together, admitted by
memory, advanced in batches (or alone, above the solo size) and frozen out at
their own cadence must give exactly the surfaces and step counts of each event
run alone with the same cadence (FP64 is bit-exact through batching)."""
import numpy as np
import pytest

import vh

pytestmark = pytest.mark.gpu


def _events(rows):
    out = []
    for i, n in enumerate((21, 33, 41, 27)):
        c = vh.hotspot_config(n)
        c.fo_factor = 5
        out.append((c, vh.hotspot_ic(c, rows, seed=100 + i)))
    g = vh.glauber_config(15, 13, 5)
    g.dx = g.dy = 0.5
    g.dz = 0.4
    g.dt = 0.05
    g.fo_factor = 4
    out.append((g, vh.glauber_ic(g, rows, b=3.0)))
    return out


@pytest.mark.parametrize("hbm_fraction,solo_cells", [(0.5, None), (1e-9, None), (0.5, 1000), (0.5, 1)])
def test_server_matches_single_event_runs(hbm_fraction, solo_cells):
    """solo_cells 1000 steps the 33^2 and 41^2 events alone beside a batch of
    the other three; 1 steps every event alone"""
    rows = vh.synthetic_eos_table()
    evs = _events(rows)
    srv = vh.Server(rows, hbm_fraction=hbm_fraction, max_steps=60, solo_cells=solo_cells)
    for tag, (c, st) in enumerate(evs):
        srv.submit(c, st, tag)
    srv.wait(300)
    done = {d.tag: d for d in srv.poll()}
    assert sorted(done) == list(range(len(evs)))
    stats = srv.stats()
    assert stats["done"] == len(evs) and stats["queued"] == 0 and stats["active"] == 0
    if hbm_fraction < 1e-6:
        assert stats["batch_builds"] >= len(evs)      # admitted one at a time
    if solo_cells == 1:
        assert stats["batch_builds"] == 0
    for tag, (c, st) in enumerate(evs):
        d = done[tag]
        assert d.t_submit <= d.t_admit <= d.t_done
        surf = srv.take_surface(tag)
        steps, ref, status = vh.run_like_server(c, rows, st, max_steps=60)
        assert d.status == status == 0
        assert d.steps == steps
        assert surf.shape == ref.shape and d.n_elements == len(ref)
        assert np.array_equal(surf.view(np.uint64), ref.view(np.uint64))
    srv.close()


def test_server_batches_each_kind_apart():
    """events of different precision and EoS kind are served side by side,
    one batch per kind; FP64 members equal their single runs bit for bit, the
    mixed member its single mixed run within the batch-vs-single rounding"""
    rows = vh.synthetic_eos_table()
    a = vh.hotspot_config(17)
    b = vh.hotspot_config(19).copy(precision=vh.VH_PREC_MIXED)
    g = vh.gubser_config(15, 15)
    for c in (a, b, g):
        c.fo_factor = 4
    ics = [vh.hotspot_ic(a, rows, seed=1), vh.hotspot_ic(b, rows, seed=2), vh.gubser_ic(g)]
    srv = vh.Server(rows, max_steps=20)
    for tag, (c, st) in enumerate(zip((a, b, g), ics)):
        srv.submit(c, st, tag)
    srv.wait(120)
    done = {d.tag: d for d in srv.poll()}
    assert srv.stats()["batch_builds"] == 3
    for tag, (c, st) in enumerate(zip((a, b, g), ics)):
        steps, ref, status = vh.run_like_server(c, rows, st, max_steps=20)
        surf = srv.take_surface(tag)
        assert done[tag].status == status == 0 and done[tag].steps == steps
        assert surf.shape == ref.shape
        if c.precision == vh.VH_PREC_FP64:
            assert np.array_equal(surf.view(np.uint64), ref.view(np.uint64))
        else:
            scale = np.maximum(np.max(np.abs(ref), axis=0), 1e-300)
            assert np.max(np.abs(surf - ref) / scale) < 1e-5
    srv.close()


def test_server_device_generated_events():
    """events submitted as generator parameters (initial state made on the
    device at admission) equal the same events run alone"""
    rows = vh.synthetic_eos_table()
    h = [vh.hotspot_config(n) for n in (29, 37)]
    for c in h:
        c.fo_factor = 5
    g = vh.glauber_config(21, 19, 7)
    g.dx = g.dy = 0.5
    g.dz = 0.4
    g.dt = 0.05
    g.fo_factor = 4
    srv = vh.Server(rows, max_steps=40)
    srv.submit_hotspots(h[0], 0, seed=5)
    srv.submit_hotspots(h[1], 1, seed=6)
    srv.submit_glauber(g, 2, b=2.0)
    srv.wait(300)
    done = {d.tag: d for d in srv.poll()}
    inits = [(h[0], lambda ev: ev.init_hotspots(seed=5)), (h[1], lambda ev: ev.init_hotspots(seed=6)),
             (g, lambda ev: ev.init_glauber(b=2.0))]
    for tag, (c, init) in enumerate(inits):
        steps, ref, status = vh.run_like_server(c, rows, init, max_steps=40)
        surf = srv.take_surface(tag)
        assert done[tag].status == status == 0 and done[tag].steps == steps
        assert surf.shape == ref.shape and np.array_equal(surf.view(np.uint64), ref.view(np.uint64))
    srv.close()
