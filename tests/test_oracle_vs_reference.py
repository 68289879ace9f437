"""The C oracle against the reference's own sources (oracle/_ref) and
against the reference's Cornelius known-answer files.

Runs on CPU.  The reference libraries exist only where the reference tree was
available when __graft_entry__.build() ran; those tests skip elsewhere.  The
known-answer test uses the committed golden hashes and runs everywhere."""
import ctypes as C
import hashlib
import json
import os
import sys
import tempfile

import numpy as np
import pytest

import vh
import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import cornelius_kat as K  # noqa: E402

FIELDS = lambda nq: list(range(nq)) + [100, 101, 102, 103, 200, 201]  # noqa: E731


def _same(cfg, a, b):
    A, B = vh.face_cells(cfg, a), vh.face_cells(cfg, b)
    return int(np.count_nonzero(A.view(np.uint64) != B.view(np.uint64)))


def small_glauber():
    cfg = vh.glauber_config(21, 19, 7)
    cfg.dx = cfg.dy = 0.6
    cfg.dz = 0.5
    cfg.dt = 0.05
    rows = vh.synthetic_eos_table()
    return cfg, rows, vh.glauber_ic(cfg, rows)


def small_hotspots():
    """a lumpy 2+1D event whose edge cells hit the e floor and the u^tau > 1e3
    velocity reset (EnergyMomentumTensor.cpp:205-232)"""
    cfg = vh.hotspot_config(41)
    rows = vh.synthetic_eos_table()
    return cfg, rows, vh.hotspot_ic(cfg, rows, seed=3)


def small_gubser():
    cfg = vh.gubser_config(31, 27)
    return cfg, None, vh.gubser_ic(cfg)


CASES = {"gubser": small_gubser, "glauber": small_glauber, "hotspots": small_hotspots}


@pytest.mark.parametrize("case,variant", [("gubser", "conf"), ("glauber", "table"), ("hotspots", "table")])
def test_kt_steps_bitexact_vs_reference(case, variant):
    if not O.ref_available(variant):
        pytest.skip("reference build not present")
    cfg, rows, st = CASES[case]()
    ref = O.RefEvent(variant, cfg, rows, threads=1)
    orc = O.OracleEvent(cfg, rows)
    ref.set_initial(st)
    orc.set_initial(st)
    for n in (1, 6):
        ref.step(n)
        assert orc.step(n) == 0
        for f in FIELDS(orc.nq):
            assert _same(cfg, ref.field(f), orc.field(f)) == 0, (case, f)


def test_reference_threads_agree_after_ghost_fix():
    if not O.ref_available("table"):
        pytest.skip("reference build not present")
    cfg, rows, st = small_glauber()
    out = []
    for th in (1, 4):
        ref = O.RefEvent("table", cfg, rows, threads=th)
        ref.set_initial(st)
        ref.step(5)
        out.append([ref.field(f) for f in FIELDS(15)])
    for a, b in zip(*out):
        assert _same(cfg, a, b) == 0


def _parse_surface(path):
    with open(path) as f:
        rows = [list(map(float, ln.split())) for ln in f if ln.strip()]
    return np.array(rows).reshape(-1, 20)


@pytest.mark.parametrize("case,variant", [("gubser", "conf"), ("glauber", "table")])
def test_freezeout_matches_reference(case, variant):
    if not O.ref_available(variant):
        pytest.skip("reference build not present")
    cfg, rows, st = small_gubser() if case == "gubser" else small_glauber()
    if case == "gubser":
        cfg.T_freezeout_GeV = 0.2      # a surface that crosses the small grid
    ref = O.RefEvent(variant, cfg, rows, threads=1)
    orc = O.OracleEvent(cfg, rows)
    ref.set_initial(st)
    orc.set_initial(st)
    with tempfile.TemporaryDirectory() as d:
        for blk in range(3):
            path = os.path.join(d, f"s{blk}.dat")
            above_ref = ref.freezeout(path)
            el_orc, above_orc = orc.freezeout()
            el_ref = _parse_surface(path)
            assert above_ref == above_orc
            assert el_ref.shape == el_orc.shape, (blk, el_ref.shape, el_orc.shape)
            assert el_ref.shape[0] > 0
            np.testing.assert_array_equal(el_ref.view(np.uint64), el_orc.view(np.uint64))
            ref.step(cfg.fo_factor)
            orc.step(cfg.fo_factor)


@pytest.mark.parametrize("dim", [3, 4])
def test_cornelius_known_answers(dim):
    with open(os.path.join(HERE, "golden", "cornelius_kat.json")) as f:
        gold = json.load(f)[f"{dim}d"]
    L = O.oracle_lib()
    L.vho_cornelius_batch.argtypes = [C.c_int, C.c_void_p, C.c_int, C.c_double, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]
    cubes = K.random_cubes(dim)
    out = np.zeros((40000, 2 * dim))
    counts = np.zeros(len(cubes), dtype=np.int32)
    dx = np.ones(4)
    n = L.vho_cornelius_batch(dim, cubes.ctypes.data, len(cubes), 0.5, dx.ctypes.data, out.ctypes.data, len(out),
                              counts.ctypes.data)
    assert n == gold["elements"]
    txt = K.format_elements(out[:n]).encode()
    assert hashlib.sha256(txt).hexdigest() == gold["sha256"]


W_FIELDS = list(range(300, 306)) + list(range(310, 314))


@pytest.mark.parametrize("case,variant", [("gubser", "conf"), ("glauber", "table")])
def test_vorticity_bitexact_vs_reference(case, variant):
    """thermal vorticity and velocity (Vorticity.cpp:6-171) after the initial
    condition and after steps, as the driver computes them, on the interior
    (the reference's ghost-cell routine also copies w and beta into the ghost
    layers during the RK stages, i.e. the previous step's values; nothing reads
    them)"""
    if not O.ref_available(variant):
        pytest.skip("reference build not present")
    cfg, rows, st = CASES[case]()
    ref = O.RefEvent(variant, cfg, rows, threads=1)
    orc = O.OracleEvent(cfg, rows)
    ref.set_initial(st)
    orc.set_initial(st)
    for n in (0, 1, 3):
        if n:
            ref.step(n)
            assert orc.step(n) == 0
        ref.vorticity()
        orc.vorticity()
        for f in W_FIELDS:
            a, b = vh.interior(cfg, ref.field(f)), vh.interior(cfg, orc.field(f))
            assert np.count_nonzero(a.view(np.uint64) != b.view(np.uint64)) == 0, (case, n, f)
        assert np.any(orc.field(303) != 0) or n == 0


@pytest.mark.parametrize("case,variant", [("gubser", "conf"), ("glauber", "table")])
def test_dynamical_sources_bitexact_vs_reference(case, variant):
    """the Source arrays (SourceTerms.cpp:584-587) entering the evolution"""
    if not O.ref_available(variant):
        pytest.skip("reference build not present")
    cfg, rows, st = CASES[case]()
    N = cfg.nx * cfg.ny * cfg.nz
    rng = np.random.default_rng(5)
    src = rng.normal(0.0, 0.5, size=(4, N)) * np.abs(st.e)[None, :] / (1.0 + np.abs(st.e).max())
    ref = O.RefEvent(variant, cfg, rows, threads=1)
    orc = O.OracleEvent(cfg, rows)
    ref.set_initial(st)
    orc.set_initial(st)
    ref.set_sources(src)
    orc.set_sources(src)
    ref.step(4)
    assert orc.step(4) == 0
    for f in FIELDS(orc.nq):
        assert _same(cfg, ref.field(f), orc.field(f)) == 0, (case, f)


@pytest.mark.parametrize("case,variant", [("gubser", "conf"), ("glauber", "table")])
def test_regulation_factors_bitexact_vs_reference(case, variant):
    """regFacShear / regFacBulk after steps (FullyDiscreteKurganovTadmorScheme.cpp:835-855)"""
    if not O.ref_available(variant):
        pytest.skip("reference build not present")
    cfg, rows, st = CASES[case]()
    ref = O.RefEvent(variant, cfg, rows, threads=1)
    orc = O.OracleEvent(cfg, rows)
    ref.set_initial(st)
    orc.set_initial(st)
    ref.step(3)
    assert orc.step(3) == 0
    for f in ((400, 401) if cfg.bulk else (400,)):
        a, b = vh.interior(cfg, ref.field(f)), vh.interior(cfg, orc.field(f))
        assert np.count_nonzero(a.view(np.uint64) != b.view(np.uint64)) == 0, (case, f)


# ------------------------------------------------- the shipped HotQCD EoS
import hotqcd_eos_prefix as HQ  # noqa: E402


def hotqcd_glauber():
    """a small 3+1D Glauber event (bulk on) on the reference's shipped EoS"""
    cfg = vh.glauber_config(19, 17, 7)
    cfg.dx = cfg.dy = 0.7
    cfg.dz = 0.5
    cfg.dt = 0.05
    return cfg


@pytest.mark.skipif(not os.path.exists(HQ.full_table_path()), reason="the reference's EoS file is not here")
def test_hotqcd_table_oracle_vs_reference():
    """the oracle on the reference's shipped 100 000-record HotQCD table
    (loaded as EquationOfState.cpp:292-327 loads it) equals the reference's
    own code: steps and freezeout blocks"""
    if not O.ref_available("table"):
        pytest.skip("reference build not present")
    full = HQ.load_full()
    cfg = hotqcd_glauber()
    st = vh.glauber_ic(cfg, full)
    # one thread: the reference's cells-above count (checkForCellsAboveTc,
    # FreezeOut.cpp:368-378) increments a shared counter inside `omp parallel
    # for` without a reduction, so with more threads it loses increments
    ref = O.RefEvent("table", cfg, full, threads=1)
    orc = O.OracleEvent(cfg, full)
    ref.set_initial(st)
    orc.set_initial(st)
    with tempfile.TemporaryDirectory() as d:
        for blk in range(4):
            path = os.path.join(d, f"s{blk}.dat")
            above_ref = ref.freezeout(path)
            el_orc, above_orc = orc.freezeout()
            assert above_ref == above_orc
            np.testing.assert_array_equal(_parse_surface(path).view(np.uint64), el_orc.view(np.uint64))
            ref.step(3)
            assert orc.step(3) == 0
            for f in FIELDS(orc.nq):
                assert _same(cfg, ref.field(f), orc.field(f)) == 0, (blk, f)


@pytest.mark.skipif(not os.path.exists(HQ.full_table_path()), reason="the reference's EoS file is not here")
def test_hotqcd_prefix_evolves_like_the_full_table():
    """the committed 2000-record prefix gives the same evolution as the full
    table for the test events (energy densities stay inside the prefix), and
    the prefix equals the first records of the shipped file"""
    full, pre = HQ.load_full(), HQ.load_prefix()
    np.testing.assert_array_equal(pre, full[:len(pre)])
    cfg = hotqcd_glauber()
    st = vh.glauber_ic(cfg, full)
    assert np.array_equal(st.e, vh.glauber_ic(cfg, pre).e)
    a, b = O.OracleEvent(cfg, full), O.OracleEvent(cfg, pre)
    a.set_initial(st)
    b.set_initial(st)
    for n in (2, 8):
        assert a.step(n) == 0 and b.step(n) == 0
        e = vh.interior(cfg, a.field(100))
        assert e.max() * 0.197326938 < pre[-3, 0]
        for f in FIELDS(a.nq):
            assert _same(cfg, a.field(f), b.field(f)) == 0, (n, f)
