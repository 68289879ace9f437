"""Bit-for-bit parity of the fused CUDA RK2 step with the C oracle.

The oracle (oracle/vh_oracle.c) is itself checked bit for bit against the
reference's own sources in tests/test_oracle_vs_reference.py.  The CUDA path
must reproduce every interior and face-ghost value exactly (compared as raw
IEEE-754 bit patterns), over many steps, for both equations of state."""
import numpy as np
import pytest

import vh
from oracle import OracleEvent

pytestmark = pytest.mark.gpu

FIELDS_14 = list(range(14)) + [100, 101, 102, 103, 200, 201]
FIELDS_15 = list(range(15)) + [100, 101, 102, 103, 200, 201]


def _bitdiff(cfg, a, b):
    A, B = vh.face_cells(cfg, a), vh.face_cells(cfg, b)
    return int(np.count_nonzero(A.view(np.uint64) != B.view(np.uint64)))


def _compare(cfg, gpu, orc, fields):
    bad = {}
    for f in fields:
        n = _bitdiff(cfg, gpu.field(f), orc.field(f))
        if n:
            bad[f] = n
    return bad


@pytest.mark.parametrize("nx,ny,steps", [(41, 37, [1, 5, 30]), (101, 101, [1, 20])])
def test_gubser_conformal_bitexact(nx, ny, steps):
    cfg = vh.gubser_config(nx, ny)
    st = vh.gubser_ic(cfg)
    gpu, orc = vh.Event(cfg), OracleEvent(cfg)
    gpu.set_initial(st)
    orc.set_initial(st)
    done = 0
    for s in steps:
        gpu.step(s - done)
        assert orc.step(s - done) == 0
        done = s
        gpu.sync()
        bad = _compare(cfg, gpu, orc, FIELDS_14)
        assert not bad, f"after {s} steps, bit-differing cells per field: {bad}"
    assert gpu.powf_misses() == 0


@pytest.mark.parametrize("dims,steps", [((27, 25, 9), [1, 4, 12]), ((21, 19, 1), [1, 10])])
def test_glauber_table_bulk_bitexact(dims, steps):
    nx, ny, nz = dims
    cfg = vh.glauber_config(nx, ny, nz)
    cfg.dx = cfg.dy = 0.5
    cfg.dz = 0.4
    cfg.dt = 0.05
    rows = vh.synthetic_eos_table()
    st = vh.glauber_ic(cfg, rows)
    gpu, orc = vh.Event(cfg, rows), OracleEvent(cfg, rows)
    gpu.set_initial(st)
    orc.set_initial(st)
    done = 0
    for s in steps:
        gpu.step(s - done)
        assert orc.step(s - done) == 0
        done = s
        gpu.sync()
        bad = _compare(cfg, gpu, orc, FIELDS_15)
        assert not bad, f"after {s} steps, bit-differing cells per field: {bad}"


_SPLIT_CHECK = r"""
import sys, numpy as np
import vh
from oracle import OracleEvent
cfg = vh.glauber_config(65, 65, 63)
cfg.dx = cfg.dy = 0.3
cfg.dz = 0.25
cfg.dt = 0.03
rows = vh.synthetic_eos_table()
st = vh.glauber_ic(cfg, rows)
gpu, orc = vh.Event(cfg, rows), OracleEvent(cfg, rows)
gpu.set_initial(st)
orc.set_initial(st)
fields = list(range(15)) + [100, 101, 102, 103, 200, 201]
bad = 0
for n in (1, 2):
    gpu.step(n)
    assert orc.step(n) == 0
    gpu.sync()
    for f in fields:
        A, B = vh.face_cells(cfg, gpu.field(f)), vh.face_cells(cfg, orc.field(f))
        bad += int(np.count_nonzero(A.view(np.uint64) != B.view(np.uint64)))
print("LAUNCHES", gpu.launches_per_step(), "BAD", bad)
"""


@pytest.mark.parametrize("env", [{}, {"VH_FLUX_FORM": "staged"}, {"VH_FLUX_STAGED": "0"}, {"VH_STAGE_MODE": "fused"},
                                 {"VH_STAGE_MODE": "fused", "VH_STAGE_FACES": "0"}],
                         ids=["split-slopes", "split-staged", "split-global", "fused-faces", "fused-one-thread"])
def test_large_lattice_forms_bitexact(env):
    """above 2^15 cells the stage runs phase-split, its flux reading a
    shared-memory tile with the half slopes computed once per tile by default
    (or each cell computing its own: staged); below, fused with one thread per
    face; every form must equal the oracle bit for bit on the same lattice (run
    in a child process: the form is chosen once per process)"""
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    e = dict(os.environ, **env)
    e["PYTHONPATH"] = os.pathsep.join([os.path.join(root, "cpu-vh_b200"), os.path.join(root, "oracle"), root])
    out = subprocess.run([sys.executable, "-c", _SPLIT_CHECK], env=e, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    line = [l for l in out.stdout.splitlines() if l.startswith("LAUNCHES")][-1].split()
    assert int(line[1]) == (2 if env.get("VH_STAGE_MODE") == "fused" else 10)
    assert int(line[3]) == 0, line


@pytest.mark.parametrize("case", ["gubser", "glauber"])
def test_thermal_vorticity_bitexact(case):
    """thermal vorticity and velocity after the initial condition and after
    steps equal the oracle's (itself equal to the reference's) on the interior"""
    if case == "gubser":
        cfg, rows = vh.gubser_config(41, 37), None
        st = vh.gubser_ic(cfg)
    else:
        cfg = vh.glauber_config(27, 25, 9)
        cfg.dx = cfg.dy = 0.5
        cfg.dz = 0.4
        cfg.dt = 0.05
        rows = vh.synthetic_eos_table()
        st = vh.glauber_ic(cfg, rows)
    gpu, orc = vh.Event(cfg, rows), OracleEvent(cfg, rows)
    gpu.set_initial(st)
    orc.set_initial(st)
    gpu.vorticity(True)
    for n in (0, 1, 4):
        if n:
            gpu.step(n)
            assert orc.step(n) == 0
        orc.vorticity()
        gpu.sync()
        for f in list(range(vh.VH_F_W, vh.VH_F_W + 6)) + list(range(vh.VH_F_BETA, vh.VH_F_BETA + 4)):
            a, b = vh.interior(cfg, gpu.field(f)), vh.interior(cfg, orc.field(f))
            assert np.count_nonzero(np.ascontiguousarray(a).view(np.uint64) !=
                                    np.ascontiguousarray(b).view(np.uint64)) == 0, (case, n, f)


@pytest.mark.parametrize("case", ["gubser", "glauber", "glauber-split"])
def test_dynamical_sources_bitexact(case):
    """dynamical sources entering the evolution: single event (fused and
    split lattices) and batch members equal the oracle bit for bit"""
    if case == "gubser":
        cfg, rows = vh.gubser_config(41, 37), None
        st = vh.gubser_ic(cfg)
    else:
        cfg = vh.glauber_config(27, 25, 9) if case == "glauber" else vh.glauber_config(41, 39, 21)
        cfg.dx = cfg.dy = 0.5
        cfg.dz = 0.4
        cfg.dt = 0.05
        rows = vh.synthetic_eos_table()
        st = vh.glauber_ic(cfg, rows)
    N = cfg.nx * cfg.ny * cfg.nz
    rng = np.random.default_rng(9)
    src = rng.normal(0.0, 0.5, size=(4, N)) * np.abs(st.e)[None, :] / (1.0 + np.abs(st.e).max())
    gpu, orc = vh.Event(cfg, rows), OracleEvent(cfg, rows)
    gpu.set_initial(st)
    orc.set_initial(st)
    gpu.set_sources(src)
    orc.set_sources(src)
    gpu.step(3)
    assert orc.step(3) == 0
    gpu.sync()
    fields = FIELDS_15 if cfg.bulk else FIELDS_14
    bad = _compare(cfg, gpu, orc, fields)
    assert not bad, bad
    # the same through a batch, sources set after the batch was built
    mem = vh.Event(cfg, rows)
    mem.set_initial(st)
    b = vh.Batch([mem])
    mem.set_sources(src)
    b.step(3)
    mem.sync()
    assert not _compare(cfg, mem, orc, fields)


@pytest.mark.parametrize("case", ["gubser", "glauber", "glauber-split"])
def test_regulation_factors_bitexact(case):
    """the kept regulation factors equal the oracle's (itself equal to the
    reference's regFacShear / regFacBulk), fused and split forms"""
    if case == "gubser":
        cfg, rows = vh.gubser_config(41, 37), None
        st = vh.gubser_ic(cfg)
    else:
        cfg = vh.glauber_config(27, 25, 9) if case == "glauber" else vh.glauber_config(41, 39, 21)
        cfg.dx = cfg.dy = 0.5
        cfg.dz = 0.4
        cfg.dt = 0.05
        rows = vh.synthetic_eos_table()
        st = vh.glauber_ic(cfg, rows)
    gpu, orc = vh.Event(cfg, rows), OracleEvent(cfg, rows)
    gpu.set_initial(st)
    orc.set_initial(st)
    gpu.keep_regulation(True)
    gpu.step(3)
    assert orc.step(3) == 0
    gpu.sync()
    for f in ((400, 401) if cfg.bulk else (400,)):
        a, b = vh.interior(cfg, gpu.field(f)), vh.interior(cfg, orc.field(f))
        assert np.count_nonzero(np.ascontiguousarray(a).view(np.uint64) !=
                                np.ascontiguousarray(b).view(np.uint64)) == 0, (case, f)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_table_sound_speed_shortcut_is_exact(precision, monkeypatch):
    """the kernels take the table sound speed as 1/3 up to the bound the
    library proves for the table; with the shortcut off (VH_CS2_SHORTCUT=0,
    read when a step is issued) the source terms and root solves evaluate the
    reference's expression everywhere, and every value is the same bit for bit
    -- single events (split stage) and batch members"""
    cfg = vh.glauber_config(41, 37, 23)
    cfg.dx = cfg.dy = 0.5
    cfg.dz = 0.4
    cfg.dt = 0.05
    if precision == "mixed":
        cfg = cfg.copy(precision=vh.VH_PREC_MIXED)
    rows = vh.synthetic_eos_table()
    st = vh.glauber_ic(cfg, rows, b=4.0)
    h = vh.hotspot_config(27).copy(precision=cfg.precision)
    hst = vh.hotspot_ic(h, rows, seed=3)

    def run():
        ev = vh.Event(cfg, rows)
        ev.set_initial(st)
        ev.step(8)
        ev.sync()
        m = vh.Event(h, rows)
        m.set_initial(hst)
        b = vh.Batch([m])
        b.step(6)
        m.sync()
        b.close()
        return ev, m

    a, am = run()
    monkeypatch.setenv("VH_CS2_SHORTCUT", "0")
    b, bm = run()
    assert a.launches_per_step() == 10
    assert not {f: n for f in FIELDS_15 if (n := _bitdiff(cfg, a.field(f), b.field(f)))}
    assert not {f: n for f in FIELDS_15 if (n := _bitdiff(h, am.field(f), bm.field(f)))}
