"""Host-side pieces that need no GPU: the C ABI exports, the rhic-conf
parsers of the C++ drop-in against the reference's own parsers, the host EoS
against the oracle, and the initial-condition generators."""
import ctypes as C
import os
import re
import tempfile

import numpy as np
import pytest

import vh
import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def _declared(header):
    with open(os.path.join(ROOT, "include", header)) as f:
        txt = re.sub(r"/\*.*?\*/", "", f.read(), flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(vh_\w+)\s*\(", txt, flags=re.M)))


def test_c_abi_exports_every_declared_symbol():
    names = _declared("vh_b200.h")
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(vh.lib, n)]
    assert not missing, missing


def test_event_create_without_device_fails_cleanly():
    if vh.lib.vh_device_available():
        pytest.skip("a GPU is present")
    cfg = vh.gubser_config(9, 9)
    with pytest.raises(vh.VhError) as ei:
        vh.Event(cfg)
    assert ei.value.code == 7   # VH_ERR_NODEVICE


def test_event_create_rejects_a_lattice_beyond_32_bit_cell_indices():
    # checked before the device is looked for, so this runs on any host
    cfg = vh.gubser_config(9, 9)
    cfg.nx, cfg.ny, cfg.nz = 2000, 2000, 600
    with pytest.raises(vh.VhError) as ei:
        vh.Event(cfg)
    assert ei.value.code == 1   # VH_ERR_ARG


class Lat(C.Structure):
    _fields_ = [(n, C.c_int) for n in ("nx", "ny", "nz", "ncx", "ncy", "ncz", "nt", "fo")] + \
               [(n, C.c_double) for n in ("dx", "dy", "dz", "dt", "theta")]


class Hyd(C.Structure):
    _fields_ = [("t0", C.c_double), ("etabar", C.c_double), ("TF", C.c_double), ("piNS", C.c_int),
                ("Treg", C.c_double), ("doFO", C.c_int)]


class Ic(C.Structure):
    _fields_ = [("type", C.c_int), ("A", C.c_int), ("nsrc", C.c_int)] + \
               [(n, C.c_double) for n in ("e0", "snn", "b", "alpha", "var", "mean")] + [("src", C.c_int)]


def _mine(d):
    lib = C.CDLL(os.path.join(ROOT, "cpu-vh_b200", "libcpu-vh_lib.so"))
    L, H, I = Lat(), Hyd(), Ic()
    getattr(lib, "_Z21readLatticeParametersPKcPv")(d.encode(), C.byref(L))
    getattr(lib, "_Z19readHydroParametersPKcPv")(d.encode(), C.byref(H))
    getattr(lib, "_Z30readInitialConditionParametersPKcPv")(d.encode(), C.byref(I))
    return bytes(L), bytes(H), bytes(I)


def _theirs(d):
    lib = C.CDLL(os.path.join(ROOT, "oracle", "_ref", "libvhref_stock.so"))
    L, H, I = Lat(), Hyd(), Ic()
    lib.vhref_read_parameters(d.encode(), C.byref(L), C.byref(H), C.byref(I))
    return bytes(L), bytes(H), bytes(I)


@pytest.mark.parametrize("case", ["dropin", "messy"])
def test_properties_parsers_match_reference(case):
    if not O.ref_available("stock"):
        pytest.skip("reference build not present")
    if case == "dropin":
        d = os.path.join(HERE, "golden", "dropin_conf")
        return_dir = d
    else:
        return_dir = tempfile.mkdtemp()
        with open(os.path.join(return_dir, "lattice.properties"), "w") as f:
            f.write("numLatticePointsX = 131\n  ny=\t131 \nnz=61\n300\ndx = 0.15\ndy=0.15\n\tdz=0.2\ndt=0.015\nFO = 3\nextra=1\n")
        with open(os.path.join(return_dir, "hydro.properties"), "w") as f:
            f.write("t0=0.6\r\netas=0.08\r\nTF=0.150\r\npiNS=1\r\nTreg=0.1\r\nFO=0\r\n")
        with open(os.path.join(return_dir, "ic.properties"), "w") as f:
            f.write("type=2\nn=0\nA=197\ne0=30\nsnn=42\nb=7.0\nalpha=0.5\nvar=1.69\nmean=3.0\n")
    assert _mine(return_dir) == _theirs(return_dir)


def test_host_eos_matches_oracle():
    rows = vh.synthetic_eos_table()
    cfg = vh.glauber_config(9, 9, 3)
    orc = O.OracleEvent(cfg, rows)
    xs = np.concatenate([np.geomspace(1e-6, 400.0, 2000), [0.0, 0.0643, 1e-15]])
    for what, f in ((0, orc.L.vho_eos_p), (1, orc.L.vho_eos_cs2), (2, orc.L.vho_eos_T)):
        a = np.array([vh.eos_eval(cfg, rows, what, x) for x in xs])
        b = np.array([f(orc.h, x) for x in xs])
        np.testing.assert_array_equal(a.view(np.uint64), b.view(np.uint64))
    for T in (0.05, 0.5, 0.76, 1.2):
        assert vh.eos_eval(cfg, rows, 3, T) == orc.L.vho_eos_e(orc.h, T)
    conf = vh.gubser_config(9, 9)
    oc = O.OracleEvent(conf)
    for x in np.geomspace(1e-6, 300.0, 500):
        assert vh.eos_eval(conf, None, 2, x) == oc.L.vho_eos_T(oc.h, x)


def test_synthetic_table_is_monotone_and_crossover():
    rows = vh.synthetic_eos_table()
    e, p, s, T = rows.T
    assert np.all(np.diff(e) > 0) and np.all(np.diff(p) > 0) and np.all(np.diff(T) > 0)
    assert np.allclose(np.diff(e), np.diff(e)[0])
    cs2 = np.gradient(p, e)
    Tc = T[np.argmin(cs2[5:-5]) + 5]
    assert 0.13 < Tc < 0.19 and cs2.min() < 0.2


def test_initial_conditions():
    cfg = vh.glauber_config(41, 41, 11)
    rows = vh.synthetic_eos_table()
    st = vh.glauber_ic(cfg, rows)
    e = st.e.reshape(11, 41, 41)
    assert np.all(np.isfinite(e)) and e.min() >= 1e-3
    assert abs(e.max() - (30.0 / vh.HBARC + 1e-3)) < 1e-9
    np.testing.assert_allclose(e, e[::-1, ::-1, ::-1], rtol=1e-12)   # b along x: point symmetric
    g = vh.gubser_config(31, 31)
    sg = vh.gubser_ic(g)
    c = 15 + 31 * 15
    T0 = vh.eos_eval(g, None, 2, sg.e[c]) * vh.HBARC
    assert abs(T0 - 0.3) < 1e-6
    assert np.all(np.isfinite(sg.pi)) and abs(sg.u[1][c]) == 0.0
    h1 = vh.hotspot_ic(vh.gubser_config(61, 61), None, seed=7)
    h2 = vh.hotspot_ic(vh.gubser_config(61, 61), None, seed=7)
    h3 = vh.hotspot_ic(vh.gubser_config(61, 61), None, seed=8)
    assert np.array_equal(h1.e, h2.e) and not np.array_equal(h1.e, h3.e)


def test_table_sound_speed_is_one_third_up_to_the_bound():
    """the kernels take the table sound speed as 1/3 without evaluating it up
    to the bound the library proves for the table (vh_eos_eval what = 4): the
    oracle's full evaluation of the reference's expression gives exactly 1/3
    on a dense sample up to that bound -- at the table's nodes, between them,
    below the table where the pressure is floored and above it where the last
    segment is extrapolated -- and tables without the properties the proof
    needs (rising pressure, slopes in (0, 2.9]) get no bound"""
    rows = vh.synthetic_eos_table()
    cfg = vh.glauber_config(9, 9, 3)
    hi = vh.eos_eval(cfg, rows, 4, 0.0)
    e = rows[:, 0] / 0.197326938
    d = e[1] - e[0]
    assert hi >= e[-1]
    orc = O.OracleEvent(cfg, rows)
    rng = np.random.default_rng(7)
    xs = np.concatenate([rng.uniform(-1e3, hi, 100000), np.geomspace(1e-12, hi, 5000), e, e + d / 2,
                         e + d * (1 - 1e-12), e[-1] + d * np.arange(1, 200), [hi, -1e6, 0.0, 1e-300]])
    cs = np.array([orc.L.vho_eos_cs2(orc.h, float(x)) for x in xs])
    assert np.count_nonzero(cs != 1.0 / 3.0) == 0
    for bad in ("flat", "falling", "steep"):
        r = rows.copy()
        if bad == "flat":
            r[700, 1] = r[699, 1]
        elif bad == "falling":
            r[700, 1] = r[699, 1] * 0.999
        else:
            r[:, 1] *= 10.0
        assert vh.eos_eval(cfg, r, 4, 0.0) == -np.inf, bad
    assert vh.eos_eval(vh.gubser_config(9, 9), None, 4, 0.0) == -np.inf


def _same_bits(a, b):
    a, b = np.ascontiguousarray(a, dtype=np.float64), np.ascontiguousarray(b, dtype=np.float64)
    return a.shape == b.shape and np.array_equal(a.view(np.uint64), b.view(np.uint64))


def test_oracle_workload_generators_equal_the_library_bit_for_bit():
    """the CPU side (oracle/workload_gen.c, which the reference's own libraries
    link) makes the benchmark's inputs bit for bit as the library does, so the
    reference arm runs on the same inputs without loading the CUDA library"""
    rows = O.synthetic_eos_rows()
    assert _same_bits(rows, vh.synthetic_eos_table())
    g = vh.glauber_config(23, 21, 9)
    og = O.glauber_workload(23, 21, 9)
    for k in ("nx", "ny", "nz", "dx", "dy", "dz", "dt", "t0", "etabar", "bulk", "eos_kind", "theta"):
        assert getattr(g, k) == getattr(og, k), k

    def press(e, cfg=g):
        return np.array([vh.eos_eval(cfg, rows, 0, x) for x in e])

    a, b = vh.glauber_ic(g, rows), O.glauber_state(og, press)
    assert _same_bits(a.e, b.e) and _same_bits(a.p, b.p) and _same_bits(a.u, b.u)
    h, oh = vh.hotspot_config(41), O.hotspot_workload(41)
    for seed in (0, 7):
        a, b = vh.hotspot_ic(h, rows, seed=seed), O.hotspot_state(oh, lambda e: press(e, h), seed)
        assert _same_bits(a.e, b.e) and _same_bits(a.p, b.p) and _same_bits(a.u, b.u)
    gu, ogu = vh.gubser_config(31, 27), O.gubser_workload(31, 27)
    a, b = vh.gubser_ic(gu), O.gubser_state(ogu)
    assert _same_bits(a.e, b.e) and _same_bits(a.p, b.p) and _same_bits(a.u, b.u) and _same_bits(a.pi, b.pi)


@pytest.mark.skipif(not O.ref_available("table"), reason="the reference's own sources were not built here")
def test_reference_pressure_of_the_initial_state_equals_the_library():
    """the reference arm gives the reference its initial state with the
    reference's own EoS pressure; it equals the library's host EoS"""
    rows = O.synthetic_eos_rows()
    cfg = O.glauber_workload(15, 13, 5)
    ref = O.RefEvent("table", cfg, rows)
    st = O.glauber_state(cfg, ref.pressure)
    g = vh.glauber_config(15, 13, 5)
    assert _same_bits(st.p, vh.glauber_ic(g, rows).p)


def test_no_kernel_name_in_two_floating_point_modes():
    """the mixed-precision translation unit (vh_mixed.cu: FMA contraction,
    fast FP32 division) and the FP64 ones (vh_kt.cu, vh_batch.cu: no
    contraction) must not instantiate a kernel of the same name: two device
    functions behind one launch stub leave it to the runtime which one runs
    (a template without the precision among its parameters did, and the
    mixed results then differed between processes)"""
    import subprocess
    build = os.path.join(ROOT, "cpu-vh_b200", "_build")
    if not os.path.exists(os.path.join(build, "vh_mixed.o")):
        pytest.skip("library objects not built here")

    def kernels(obj):
        out = subprocess.run(["nm", "-C", os.path.join(build, obj)], capture_output=True, text=True, check=True).stdout
        return {ln.split(" ", 2)[2] for ln in out.splitlines()
                if " W " in ln and "_kernel" in ln and ln.split(" ", 2)[2].startswith("void vh::")}

    mixed = kernels("vh_mixed.o")
    assert mixed, "no kernels found in vh_mixed.o"
    for obj in ("vh_kt.o", "vh_batch.o"):
        both = mixed & kernels(obj)
        assert not both, (obj, sorted(both)[:5])
