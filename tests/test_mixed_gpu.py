"""Mixed precision (VH_PREC_MIXED): FP32 limiter, flux and source arithmetic
with FP64 accumulation and root solve, against the FP64 path (bit-identical
to the oracle and the reference).

The reference's scheme is chaotic in the dilute edge region: its discrete
switches (the e <= 0.1 inversion branch, EnergyMomentumTensor.cpp:188-191;
the e < e_reg regulation threshold; the u^tau > 1e3 reset) turn any
perturbation into O(1) local differences, so a relative change of 2^-50 in
the initial energy density alone grows to ~8 % relative L-infinity in e after
the Gubser event's 300 steps.  The mixed path is therefore checked (a) to
1e-4 relative L-infinity (max |a - b| / max |b|) before that growth sets in,
and (b) at the end of the event against the FP64 path's own sensitivity: its
error must stay within a small factor of what a one-ulp-scale perturbation of
the FP64 run produces."""
import numpy as np
import pytest

import vh
from oracle import OracleEvent

pytestmark = pytest.mark.gpu


def rel_linf(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def _run(cfg, rows, st, steps, mixed):
    c = cfg.copy(precision=vh.VH_PREC_MIXED if mixed else vh.VH_PREC_FP64)
    ev = vh.Event(c, rows)
    ev.set_initial(st)
    ev.step(steps)
    ev.sync()
    return ev


def _errors(cfg, ev, orc):
    out = {}
    for name, fid in [("e", vh.VH_F_E), ("ut", vh.VH_F_UT), ("ux", vh.VH_F_UT + 1), ("uy", vh.VH_F_UT + 2),
                      ("pixx", 8), ("pixy", 9), ("piyy", 11), ("pinn", 13)]:
        out[name] = rel_linf(vh.interior(cfg, ev.field(fid)), vh.interior(cfg, orc.field(fid)))
    return out


def test_gubser_mixed_vs_fp64():
    cfg = vh.gubser_config()
    st = vh.gubser_ic(cfg)
    err = _errors(cfg, _run(cfg, None, st, 30, True), _run(cfg, None, st, 30, False))
    assert max(err.values()) <= 1e-4, err


def test_gubser_mixed_error_within_fp64_sensitivity():
    """the full Gubser event (101 x 101, 300 steps)"""
    cfg = vh.gubser_config()
    st = vh.gubser_ic(cfg)
    bumped = vh.gubser_ic(cfg)
    bumped.e = bumped.e * (1 + 2.0 ** -50)
    ref = _run(cfg, None, st, 300, False)
    mixed = _errors(cfg, _run(cfg, None, st, 300, True), ref)
    floor = _errors(cfg, _run(cfg, None, bumped, 300, False), ref)
    assert floor["e"] > 1e-3, floor           # the chaotic growth this test is built around
    for k in ("e", "ut", "ux", "uy"):
        assert mixed[k] <= 3 * floor[k], (k, mixed, floor)


def test_glauber_mixed_vs_oracle():
    cfg = vh.glauber_config(27, 25, 9)
    cfg.dx = cfg.dy = 0.5
    cfg.dz = 0.4
    cfg.dt = 0.05
    rows = vh.synthetic_eos_table()
    st = vh.glauber_ic(cfg, rows)
    ev = _run(cfg, rows, st, 40, True)
    orc = OracleEvent(cfg, rows)
    orc.set_initial(st)
    assert orc.step(40) == 0
    err = _errors(cfg, ev, orc)
    err["Pi"] = rel_linf(vh.interior(cfg, ev.field(14)), vh.interior(cfg, orc.field(14)))
    assert err["e"] <= 1e-4, err
    assert ev.status()[0] == 0


def _surface_sums(ev, steps, fo_every):
    ev.freezeout()
    tot = np.zeros(4)
    count = 0
    for _ in range(steps // fo_every):
        ev.step(fo_every)
        n, _ = ev.freezeout()
        if n:
            s = ev.surface()
            tot += s[:, 4:8].sum(axis=0)
            count += n
    return count, tot


def test_freezeout_surface_mixed_vs_fp64():
    cfg = vh.gubser_config()
    st = vh.gubser_ic(cfg)
    bumped = vh.gubser_ic(cfg)
    bumped.e = bumped.e * (1 + 2.0 ** -50)
    res = {}
    for key, prec, ic in (("fp64", vh.VH_PREC_FP64, st), ("mixed", vh.VH_PREC_MIXED, st),
                          ("fp64_bumped", vh.VH_PREC_FP64, bumped)):
        ev = vh.Event(cfg.copy(precision=prec))
        ev.set_initial(ic)
        res[key] = _surface_sums(ev, 300, 10)
    n64, s64 = res["fp64"]
    assert n64 > 0
    for key in ("mixed", "fp64_bumped"):
        n, s = res[key]
        res[key] = (abs(n - n64) / n64, float(np.max(np.abs(s - s64)) / np.max(np.abs(s64))))
    dn, ds = res["mixed"]
    fn, fs = res["fp64_bumped"]
    assert dn <= max(0.005, 3 * fn), res
    assert ds <= max(1e-4, 3 * fs), res


def test_batched_mixed_matches_single_mixed():
    rows = vh.synthetic_eos_table()
    cfgs = [vh.hotspot_config(n).copy(precision=vh.VH_PREC_MIXED) for n in (25, 33)]
    ics = [vh.hotspot_ic(c, rows, seed=9 + i) for i, c in enumerate(cfgs)]
    evs, ref = [], []
    for c, st in zip(cfgs, ics):
        for lst in (evs, ref):
            e = vh.Event(c, rows)
            e.set_initial(st)
            lst.append(e)
    b = vh.Batch(evs)
    b.step(20)
    for c, e, r in zip(cfgs, evs, ref):
        r.step(20)
        e.sync()
        r.sync()
        # the same mixed arithmetic in differently shaped kernels (the single
        # event runs the face-parallel stage): FMA contraction may differ
        assert rel_linf(vh.interior(c, e.field(vh.VH_F_E)), vh.interior(c, r.field(vh.VH_F_E))) <= 1e-5
    with pytest.raises(vh.VhError):
        x = vh.Event(vh.hotspot_config(15), rows)
        x.set_initial(vh.hotspot_ic(x.cfg, rows, seed=1))
        vh.Batch([evs[0], x])


def test_mixed_split_face_once_vs_fp64():
    """a lattice above the fused/split threshold (2^15 cells): the mixed split
    stage evaluates each face once; after 20 steps its error against the FP64
    path must stay within 1e-4 relative L-infinity in e (the velocity, whose
    largest deviations sit in the dilute edge, within 1e-2)"""
    cfg = vh.glauber_config(81, 81, 41)
    rows = vh.synthetic_eos_table()
    st = vh.glauber_ic(cfg, rows)
    mixed = _run(cfg, rows, st, 20, True)
    ref = _run(cfg, rows, st, 20, False)
    assert mixed.launches_per_step() == 10          # the phase-split form ran
    err = _errors(cfg, mixed, ref)
    assert err["e"] <= 1e-4, err
    assert max(err[k] for k in ("ut", "ux", "uy")) <= 1e-2, err


_REPRO = r"""
import hashlib, sys
import vh
rows = vh.synthetic_eos_table()
h = hashlib.sha256()
# a single event on the phase-split stage (face-once FP32 flux)
cfg = vh.glauber_config(65, 65, 33).copy(precision=vh.VH_PREC_MIXED)
cfg.dx = cfg.dy = 0.3
cfg.dz = 0.3
cfg.dt = 0.03
ev = vh.Event(cfg, rows)
ev.set_initial(vh.glauber_ic(cfg, rows))
ev.step(12)
ev.sync()
rc = ev.status()[0]
for f in list(range(15)) + [100, 101, 102, 103, 200, 201]:
    h.update(vh.face_cells(cfg, ev.field(f)).tobytes())
# an autotuned batch of lumpy 2+1D events of three sizes
evs = []
for i, n in enumerate((61, 81, 101, 81)):
    c = vh.hotspot_config(n).copy(precision=vh.VH_PREC_MIXED)
    e = vh.Event(c, rows)
    e.set_initial(vh.hotspot_ic(c, rows, seed=i))
    evs.append((c, e))
b = vh.Batch([e for _, e in evs])
b.autotune()
b.step(15)
for c, e in evs:
    e.sync()
    rc = rc or e.status()[0]
    for f in list(range(15)) + [100, 101, 102, 103, 200, 201]:
        h.update(vh.face_cells(c, e.field(f)).tobytes())
print("HASH", rc, h.hexdigest())
"""


def test_mixed_results_same_in_every_process_and_with_poisoned_memory():
    """the mixed path gives the same bits in separate processes, also when
    every event buffer starts filled with NaNs or with the finite sentinel
    1.4e301 (VH_POISON_ALLOC=1 / 2): no kernel reads event memory that no
    kernel wrote (a finite sentinel is not swallowed by the fmin/fmax of the
    limiter and the wave speed, as a NaN would be)"""
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = []
    for poison in ("", "", "1", "2"):
        env = dict(os.environ, PYTHONPATH=os.pathsep.join([os.path.join(root, "cpu-vh_b200"), root]))
        env.pop("VH_POISON_ALLOC", None)
        if poison:
            env["VH_POISON_ALLOC"] = poison
        r = subprocess.run([sys.executable, "-c", _REPRO], env=env, capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr[-2000:]
        out.append([ln for ln in r.stdout.splitlines() if ln.startswith("HASH")][-1])
    assert out[0].split()[1] == "0", out[0]
    assert len(set(out)) == 1, out


def test_mixed_face_forms_agree():
    """the face-once flux over line pieces (along y and eta, the default) and
    over 32 x 8 face tiles (VH_FACE_FORM=tiles) compute every face and every
    cell update with the same arithmetic: the same bits (child processes:
    the form is chosen once per process)"""
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    child = _REPRO.split("# an autotuned batch")[0] + 'print("HASH", rc, h.hexdigest())\n'
    out = []
    for form in ("tiles", "lines"):
        env = dict(os.environ, VH_FACE_FORM=form,
                   PYTHONPATH=os.pathsep.join([os.path.join(root, "cpu-vh_b200"), root]))
        env.pop("VH_POISON_ALLOC", None)
        r = subprocess.run([sys.executable, "-c", child], env=env, capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr[-2000:]
        out.append([ln for ln in r.stdout.splitlines() if ln.startswith("HASH")][-1])
    assert out[0].split()[1] == "0" and out[0] == out[1], out
