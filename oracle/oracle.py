"""TEST INFRASTRUCTURE ONLY: Python access to the CPU oracles.

* OracleEvent wraps liboracle_vh.so, the C restatement of the cpu-vh hot path
  (vh_oracle.c, cornelius_oracle.c).  It is built from this directory's
  sources by `make -C oracle` (the tests build it on demand with gcc).
* RefEvent wraps oracle/_ref/libvhref_<variant>.so, the reference's own
  sources compiled in place by oracle/ref.mk; it exists only where the
  reference tree was available at build time.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may use
this module, and only as the checker or the timed CPU baseline.
"""
from __future__ import annotations

import contextlib
import ctypes as C
import os
import subprocess
import sys

from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "liboracle_vh.so")
REF_DIR = os.path.join(HERE, "_ref")
_dp = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")


_libc = C.CDLL(None)
_libc.fflush.argtypes = [C.c_void_p]


@contextlib.contextmanager
def _stdout_to_stderr():
    """C-level stdout (fd 1) goes to stderr inside the block."""
    sys.stdout.flush()
    _libc.fflush(None)
    saved = os.dup(1)
    os.dup2(2, 1)
    try:
        yield
    finally:
        _libc.fflush(None)
        os.dup2(saved, 1)
        os.close(saved)


def build_oracle(force: bool = False) -> str:
    srcs = [os.path.join(HERE, f) for f in ("vh_oracle.c", "cornelius_oracle.c", "workload_gen.c")
            if os.path.exists(os.path.join(HERE, f))]
    newest = max(os.path.getmtime(s) for s in srcs)
    if force or not os.path.exists(ORACLE_LIB) or os.path.getmtime(ORACLE_LIB) < newest:
        subprocess.run(["make", "-s", "-C", HERE, "liboracle_vh.so", "CC_HOST=gcc"], check=True)
    return ORACLE_LIB


_olib = None


def oracle_lib():
    global _olib
    if _olib is None:
        _olib = C.CDLL(build_oracle())
        L = _olib
        L.vho_create.restype = C.c_void_p
        L.vho_create.argtypes = [C.c_int] * 3 + [C.c_double] * 7 + [C.c_int, C.c_double, C.c_double, C.c_int]
        L.vho_set_conformal.argtypes = [C.c_void_p, C.c_double]
        L.vho_set_zeta.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_double, C.c_double]
        L.vho_set_table.argtypes = [C.c_void_p, _dp, C.c_int]
        L.vho_set_ic.argtypes = [C.c_void_p, _dp, _dp, _dp, C.c_void_p, C.c_void_p]
        L.vho_step.argtypes = [C.c_void_p, C.c_int]
        L.vho_get.argtypes = [C.c_void_p, C.c_int, _dp]
        L.vho_destroy.argtypes = [C.c_void_p]
        L.vho_vorticity.argtypes = [C.c_void_p]
        L.vho_set_sources.argtypes = [C.c_void_p] + [C.c_void_p] * 4
        for f in ("vho_eos_p", "vho_eos_T", "vho_eos_cs2", "vho_eos_e"):
            getattr(L, f).argtypes = [C.c_void_p, C.c_double]
            getattr(L, f).restype = C.c_double
        L.vho_fo_eF.argtypes = [C.c_void_p]
        L.vho_fo_eF.restype = C.c_double
        L.vho_time.argtypes = [C.c_void_p]
        L.vho_time.restype = C.c_double
        L.vho_steps_done.argtypes = [C.c_void_p]
        if hasattr(L, "vho_freezeout"):
            L.vho_freezeout.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]
            L.vho_freezeout.restype = C.c_int
    return _olib


def _p(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float64).ctypes.data_as(C.c_void_p)


class OracleEvent:
    """The C restatement driven like vh.Event (same config structure)."""

    def __init__(self, cfg, eos_rows=None):
        L = oracle_lib()
        self.L, self.cfg = L, cfg
        self.h = L.vho_create(cfg.nx, cfg.ny, cfg.nz, cfg.dx, cfg.dy, cfg.dz, cfg.dt, cfg.t0, cfg.etabar, cfg.theta,
                              cfg.bulk, cfg.T_reg_GeV, cfg.T_freezeout_GeV, cfg.fo_factor)
        if cfg.eos_kind == 1:
            rows = np.ascontiguousarray(eos_rows, dtype=np.float64)
            L.vho_set_table(self.h, rows, len(rows))
        else:
            L.vho_set_conformal(self.h, cfg.eos_factor)
        L.vho_set_zeta(self.h, cfg.zeta_law, cfg.zeta_norm, cfg.zeta_T0_GeV, cfg.zeta_width_GeV)
        self.nq = 15 if cfg.bulk else 14

    def set_initial(self, st):
        self._keep = [np.ascontiguousarray(x, dtype=np.float64) if x is not None else None
                      for x in (st.e, st.p, np.asarray(st.u).reshape(-1), None if st.pi is None else np.asarray(st.pi).reshape(-1), st.Pi)]
        e, p, u, pi, Pi = self._keep
        self.L.vho_set_ic(self.h, e, p, u, _p(pi) if pi is not None else None, _p(Pi) if Pi is not None else None)

    def step(self, n=1):
        return self.L.vho_step(self.h, n)

    def vorticity(self):
        """thermal vorticity and velocity of the current state (fields 300+, 310+)"""
        self.L.vho_vorticity(self.h)

    def set_sources(self, src):
        """dynamical sources: (4, N) interior array (t, x, y, eta) or None"""
        if src is None:
            self.L.vho_set_sources(self.h, None, None, None, None)
            return
        self._src = np.ascontiguousarray(src, dtype=np.float64)
        self.L.vho_set_sources(self.h, *[_p(self._src[c]) for c in range(4)])

    def field(self, fid):
        ncx, ncy, ncz = self.cfg.nx + 4, self.cfg.ny + 4, self.cfg.nz + 4
        out = np.zeros(ncx * ncy * ncz)
        rc = self.L.vho_get(self.h, fid, out)
        assert rc == 0, fid
        return out

    def freezeout(self, cap=None):
        n_el, n_ab = C.c_int(), C.c_int()
        cap = cap or max(1024, 40 * self.cfg.nx * self.cfg.ny * max(1, self.cfg.nz))
        buf = np.zeros((cap, 20))
        rc = self.L.vho_freezeout(self.h, buf.ctypes.data_as(C.c_void_p), cap, C.byref(n_el), C.byref(n_ab))
        assert rc == 0, rc
        return buf[:n_el.value].copy(), n_ab.value

    def close(self):
        if self.h:
            self.L.vho_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()


# --------------------------------------------------------------- workloads
# The benchmark's workloads described without the CUDA library: a plain
# configuration record (the fields of vh_config that the oracles read) and
# the seeded generators of workload_gen.c, which both liboracle_vh.so and the
# oracle/_ref libraries export, so the reference can be given its inputs
# while only its own library is loaded.

@dataclass
class WorkloadConfig:
    nx: int
    ny: int
    nz: int
    dx: float
    dy: float
    dz: float
    dt: float
    t0: float
    etabar: float
    theta: float = 1.8
    bulk: int = 0
    eos_kind: int = 0                 # 0 conformal, 1 table
    eos_factor: float = 15.6269
    T_reg_GeV: float = 0.1
    T_freezeout_GeV: float = 0.15
    fo_factor: int = 2
    zeta_law: int = 0                 # 0 the reference's law, 1 Gaussian in T [GeV]
    zeta_norm: float = 0.0
    zeta_T0_GeV: float = 0.0
    zeta_width_GeV: float = 0.0


def gubser_workload(nx=101, ny=101) -> WorkloadConfig:
    """Config "plain 2+1D Gubser": 101^2, dx = 0.1 fm, tau0 = 1, dtau = 0.01,
    eta/s = 0.2, conformal a = 15.6269, theta = 1.8, T_F = 0.15 GeV"""
    return WorkloadConfig(nx, ny, 1, 0.1, 0.1, 0.1, 0.01, 1.0, 0.2)


def glauber_workload(nx=131, ny=131, nz=61) -> WorkloadConfig:
    """Config "plain 3+1D Glauber": 131^2 x 61, dx = dy = 0.15, deta = 0.2,
    tau0 = 0.6, dtau = 0.015, eta/s = 0.08, table EoS, Gaussian zeta/s"""
    return WorkloadConfig(nx, ny, nz, 0.15, 0.15, 0.2, 0.015, 0.6, 0.08, bulk=1, eos_kind=1,
                          zeta_law=1, zeta_norm=0.05, zeta_T0_GeV=0.17, zeta_width_GeV=0.02)


def hotspot_workload(n=101) -> WorkloadConfig:
    """a 2+1D lumpy event of the batched workload: n x n, dx = 0.1 fm,
    tau0 = 0.6, dtau = 0.01, otherwise as the Glauber event"""
    c = glauber_workload(n, n, 1)
    c.dx = c.dy = c.dz = 0.1
    c.t0, c.dt = 0.6, 0.01
    return c


@dataclass
class WorkloadState:
    e: np.ndarray
    p: np.ndarray
    u: np.ndarray          # (4, N)
    pi: np.ndarray | None  # (10, N)
    Pi: np.ndarray | None  # (N,)


def _gen_sigs(L):
    if getattr(L, "_vhg_ready", False):
        return L
    L.vhg_eos_synthetic_table.argtypes = [C.c_int] + [C.c_double] * 6 + [_dp]
    L.vhg_ic_glauber.argtypes = [C.c_int] * 3 + [C.c_double] * 10 + [_dp, _dp]
    L.vhg_ic_hotspots.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_uint64] + [C.c_double] * 6 + [_dp, _dp]
    L.vhg_ic_gubser.argtypes = [C.c_int, C.c_int] + [C.c_double] * 7 + [_dp, _dp, _dp, C.c_void_p]
    L._vhg_ready = True
    return L


def synthetic_eos_rows(lib=None, nrows=2000, T_lo=0.05, e_max=60.0, a=15.6269, dip=0.2, Tc=0.16, w=0.04):
    """the 2000-row crossover EoS table (rows e, P, s, T)"""
    L = _gen_sigs(lib or oracle_lib())
    rows = np.zeros((nrows, 4))
    assert L.vhg_eos_synthetic_table(nrows, T_lo, e_max, a, dip, Tc, w, rows) == 0
    return rows


def glauber_state(cfg, pressure, lib=None, R=6.38, a=0.535, sigma_nn=4.2, b=7.0, e0=30.0, eta_flat=3.0,
                  eta_sigma=1.3) -> WorkloadState:
    """optical-Glauber initial state; pressure(e) -> p is the EoS of the
    caller's library"""
    L = _gen_sigs(lib or oracle_lib())
    N = cfg.nx * cfg.ny * cfg.nz
    e, u = np.zeros(N), np.zeros(4 * N)
    assert L.vhg_ic_glauber(cfg.nx, cfg.ny, cfg.nz, cfg.dx, cfg.dy, cfg.dz, R, a, sigma_nn, b, e0, eta_flat,
                            eta_sigma, e, u) == 0
    return WorkloadState(e, pressure(e), u.reshape(4, N), None, np.zeros(N) if cfg.bulk else None)


def hotspot_state(cfg, pressure, seed, lib=None, mean_spots=200.0, w=0.4, k_gamma=1.6, amp=20.0, R=6.38,
                  a=0.535) -> WorkloadState:
    L = _gen_sigs(lib or oracle_lib())
    N = cfg.nx * cfg.ny
    e, u = np.zeros(N), np.zeros(4 * N)
    assert L.vhg_ic_hotspots(cfg.nx, cfg.ny, cfg.dx, cfg.dy, seed, mean_spots, w, k_gamma, amp, R, a, e, u) == 0
    return WorkloadState(e, pressure(e), u.reshape(4, N), None, np.zeros(N) if cfg.bulk else None)


def gubser_state(cfg, lib=None, q=1.0, T0_GeV=0.3) -> WorkloadState:
    L = _gen_sigs(lib or oracle_lib())
    N = cfg.nx * cfg.ny
    e, p, u, pi = np.zeros(N), np.zeros(N), np.zeros(4 * N), np.zeros(10 * N)
    assert L.vhg_ic_gubser(cfg.nx, cfg.ny, cfg.dx, cfg.dy, cfg.t0, cfg.eos_factor, cfg.etabar, q, T0_GeV, e, p, u,
                           pi.ctypes.data_as(C.c_void_p)) == 0
    return WorkloadState(e, p, u.reshape(4, N), pi.reshape(10, N), None)


def ref_lib_path(variant: str) -> str:
    return os.path.join(REF_DIR, f"libvhref_{variant}.so")


def ref_available(variant: str) -> bool:
    return os.path.exists(ref_lib_path(variant))


def load_gen_lib(path: str):
    """a library exporting the workload generators (oracle/_ref or the oracle)"""
    return _gen_sigs(C.CDLL(path))


def shipped_runs_here() -> bool:
    """the *_shipped libraries are built for Sapphire Rapids class x86-64
    (AVX-512 incl. FP16, AMX): only load them on a host that has those"""
    try:
        flags = set(open("/proc/cpuinfo").read().split())
    except OSError:
        return False
    return {"avx512f", "avx512bw", "avx512vl", "avx512_fp16", "amx_tile"} <= flags


def shipped_build_flags() -> str:
    """how the *_shipped reference libraries were compiled (oracle/ref.mk)"""
    p = os.path.join(REF_DIR, "shipped_flags.txt")
    return open(p).read().strip() if os.path.exists(p) else "unknown"


class RefEvent:
    """The reference's own code (oracle/_ref), single-threaded unless asked.

    The reference keeps its state in process globals, so only one RefEvent per
    variant library may be live at a time.  Its diagnostics (printf to
    stdout) are sent to stderr while it runs, so that a caller's stdout stays
    its own."""

    def __init__(self, variant, cfg, eos_rows=None, threads=1):
        path = os.path.join(REF_DIR, f"libvhref_{variant}.so")
        L = C.CDLL(path)
        self.L, self.cfg = L, cfg
        L.vhref_threads.argtypes = [C.c_int]
        L.vhref_threads(threads)
        L.vhref_setup.argtypes = [C.c_int] * 5 + [C.c_double] * 8 + [C.c_int]
        L.vhref_setup(cfg.nx, cfg.ny, cfg.nz, 100000, cfg.fo_factor, cfg.dx, cfg.dy, cfg.dz, cfg.dt, cfg.t0, cfg.etabar,
                      cfg.T_freezeout_GeV, cfg.T_reg_GeV, 0)
        if eos_rows is not None:
            L.vhref_load_eos_table.argtypes = [_dp, C.c_int]
            rows = np.ascontiguousarray(eos_rows, dtype=np.float64)
            L.vhref_load_eos_table(rows, len(rows))
        L.vhref_set_ic_arrays.argtypes = [_dp] * 5
        L.vhref_get.argtypes = [C.c_int, _dp]
        L.vhref_step.argtypes = [C.c_int]
        L.vhref_time_steps.argtypes = [C.c_int]
        L.vhref_time_steps.restype = C.c_double
        L.vhref_freezeout.argtypes = [C.c_char_p]
        L.vhref_run_full.argtypes = [C.c_char_p]
        L.vhref_theta.restype = C.c_double
        for f in ("vhref_eos_pressure", "vhref_eos_temperature", "vhref_eos_cs2", "vhref_eos_energy"):
            getattr(L, f).argtypes = [C.c_double]
            getattr(L, f).restype = C.c_double
        L.vhref_eos_pressure_n.argtypes = [_dp, _dp, C.c_long]

    def pressure(self, e):
        """the reference's equilibrium pressure of the energy densities e"""
        e = np.ascontiguousarray(e, dtype=np.float64)
        p = np.zeros_like(e)
        self.L.vhref_eos_pressure_n(e, p, len(e))
        return p

    def set_initial(self, st):
        N = self.cfg.nx * self.cfg.ny * self.cfg.nz
        pi = np.zeros(10 * N) if st.pi is None else np.ascontiguousarray(st.pi, dtype=np.float64).reshape(-1)
        Pi = np.zeros(N) if st.Pi is None else np.ascontiguousarray(st.Pi, dtype=np.float64)
        self.L.vhref_set_ic_arrays(np.ascontiguousarray(st.e), np.ascontiguousarray(st.p),
                                   np.ascontiguousarray(st.u, dtype=np.float64).reshape(-1), pi, Pi)
        with _stdout_to_stderr():
            self.L.vhref_init()

    def step(self, n=1):
        with _stdout_to_stderr():
            self.L.vhref_step(n)

    def vorticity(self):
        with _stdout_to_stderr():
            self.L.vhref_vorticity()

    def set_sources(self, src):
        self._src = np.ascontiguousarray(src, dtype=np.float64)
        self.L.vhref_set_sources.argtypes = [_dp] * 4
        self.L.vhref_set_sources(*[np.ascontiguousarray(self._src[c]) for c in range(4)])

    def time_steps(self, n):
        with _stdout_to_stderr():
            return self.L.vhref_time_steps(n)

    def field(self, fid):
        ncx, ncy, ncz = self.cfg.nx + 4, self.cfg.ny + 4, self.cfg.nz + 4
        out = np.zeros(ncx * ncy * ncz)
        assert self.L.vhref_get(fid, out) == 0, fid
        return out

    def freezeout(self, path):
        with _stdout_to_stderr():
            return self.L.vhref_freezeout(path.encode())
