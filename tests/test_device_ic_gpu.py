"""Initial conditions generated on the device (vh_event_init_glauber,
vh_event_init_hotspots) against the host generators, and the evolution from
them against the oracle started from the same (downloaded) state."""
import numpy as np
import pytest

import vh
from oracle import OracleEvent

pytestmark = pytest.mark.gpu


def _close(a, b, tol=1e-13):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)) <= tol


def _state(cfg, ev):
    e = vh.interior(cfg, ev.field(vh.VH_F_E)).ravel()
    p = vh.interior(cfg, ev.field(vh.VH_F_P)).ravel()
    u = np.stack([vh.interior(cfg, ev.field(vh.VH_F_UT + c)).ravel() for c in range(4)])
    return e, p, u


def test_device_glauber_matches_host():
    rows = vh.synthetic_eos_table()
    cfg = vh.glauber_config(41, 37, 11)
    ev = vh.Event(cfg, rows)
    ev.init_glauber(b=5.0)
    ref = vh.glauber_ic(cfg, rows, b=5.0)
    e, p, u = _state(cfg, ev)
    assert _close(e, ref.e) and _close(p, ref.p) and np.array_equal(u, ref.u)
    assert ev.progress()[0] == 0


def test_device_hotspots_match_host_and_evolve_like_the_oracle():
    rows = vh.synthetic_eos_table()
    cfg = vh.hotspot_config(45)
    ev = vh.Event(cfg, rows)
    ev.init_hotspots(seed=12)
    ref = vh.hotspot_ic(cfg, rows, seed=12)
    e, p, u = _state(cfg, ev)
    # the hottest spots lie beyond the EoS table, where p(e) is the table's last
    # segment extrapolated and a last-bit difference in e grows ~100-fold
    assert _close(e, ref.e) and _close(p, ref.p, 1e-12) and np.array_equal(u, ref.u)
    orc = OracleEvent(cfg, rows)
    orc.set_initial(vh.InitialState(e, p, u, None, np.zeros_like(e)))
    ev.step(4)
    assert orc.step(4) == 0
    ev.sync()
    for f in list(range(15)) + [100, 101, 102, 103, 200, 201]:
        A, B = vh.face_cells(cfg, ev.field(f)), vh.face_cells(cfg, orc.field(f))
        assert np.count_nonzero(A.view(np.uint64) != B.view(np.uint64)) == 0, f


def test_device_ic_argument_checks():
    rows = vh.synthetic_eos_table()
    ev = vh.Event(vh.glauber_config(9, 9, 5), rows)
    with pytest.raises(vh.VhError):
        ev.init_hotspots(seed=1)                  # hotspot events are 2+1D
    with pytest.raises(vh.VhError):
        ev.init_glauber(R=-1.0)
