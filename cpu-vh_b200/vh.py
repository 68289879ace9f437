"""ctypes bindings for libvh_b200.so, the C ABI of the B200 KT + freezeout path.

The library is the product; this module only marshals numpy arrays across the
C ABI declared in include/vh_b200.h.  It never falls back to a CPU
implementation: if the shared library is missing, importing this module
raises.

Workload presets mirror the synthetic configurations the path is measured on:

  gubser_2p1d   101x101x1, dx=0.1 fm, tau0=1.0, dtau=0.01, conformal a=15.6269,
                eta/s=0.2, theta=1.8, T0=0.3 GeV at the origin, q=1/fm,
                pi^{mu nu} at its Navier-Stokes value, T_F=0.15 GeV.
  glauber_3p1d  131x131x61, dx=dy=0.15 fm, deta=0.2, tau0=0.6, dtau=0.015,
                2000-row synthetic crossover EoS table, eta/s=0.08, Gaussian
                zeta/s, optical Glauber Au+Au b=7 fm, peak 30 GeV/fm^3,
                plateau |eta|<1.5 with Gaussian tails sigma=1.3.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libvh_b200.so")

if not os.path.exists(LIB_PATH):
    raise ImportError(f"libvh_b200.so not built at {LIB_PATH}; run `make -C cpu-vh_b200` "
                      "(or __graft_entry__.build())")

lib = C.CDLL(LIB_PATH)

VH_OK = 0
VH_EOS_CONFORMAL, VH_EOS_TABLE = 0, 1
VH_ZETA_REFERENCE, VH_ZETA_GAUSSIAN = 0, 1
VH_PREC_FP64, VH_PREC_MIXED = 0, 1
VH_F_UT, VH_F_UPT, VH_F_E, VH_F_P = 100, 110, 200, 201
VH_F_W, VH_F_BETA, VH_F_REGFAC = 300, 310, 400
VH_FO_COLUMNS = 20
PHASES = ("source", "flux_x", "flux_y", "flux_eta", "final", "fused")
HBARC = 0.197326938

FO_COLUMN_NAMES = ["tau", "x", "y", "eta", "ds0", "ds1", "ds2", "ds3", "ux", "uy", "un",
                   "e", "T", "P", "pixx", "pixy", "pixn", "piyy", "piyn", "Pi"]


class VhConfig(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
                ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double),
                ("dt", C.c_double), ("t0", C.c_double), ("etabar", C.c_double),
                ("T_freezeout_GeV", C.c_double), ("T_reg_GeV", C.c_double),
                ("fo_factor", C.c_int), ("theta", C.c_double), ("eos_kind", C.c_int),
                ("eos_factor", C.c_double), ("bulk", C.c_int), ("zeta_law", C.c_int),
                ("zeta_norm", C.c_double), ("zeta_T0_GeV", C.c_double),
                ("zeta_width_GeV", C.c_double), ("precision", C.c_int)]

    def nq(self) -> int:
        return 15 if self.bulk else 14

    def padded(self):
        return (self.nx + 4, self.ny + 4, self.nz + 4)

    def copy(self, **kw) -> "VhConfig":
        c = VhConfig()
        C.pointer(c)[0] = self
        for k, v in kw.items():
            setattr(c, k, v)
        return c


_dp = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_cfgp = C.POINTER(VhConfig)
_evp = C.c_void_p


def _sig(name, res, args):
    f = getattr(lib, name)
    f.restype = res
    f.argtypes = args
    return f


_sig("vh_config_default", C.c_int, [_cfgp])
_sig("vh_config_nq", C.c_int, [_cfgp])
_sig("vh_last_error", C.c_char_p, [])
_sig("vh_device_available", C.c_int, [])
_sig("vh_event_create", C.c_int, [_cfgp, C.c_void_p, C.c_int, C.POINTER(_evp)])
_sig("vh_event_destroy", C.c_int, [_evp])
_sig("vh_event_set_initial", C.c_int, [_evp, _dp, _dp, _dp, C.c_void_p, C.c_void_p])
_sig("vh_event_set_initial_device", C.c_int, [_evp, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p])
_sig("vh_event_step", C.c_int, [_evp, C.c_int])
_sig("vh_event_status", C.c_int, [_evp, C.POINTER(C.c_int), C.POINTER(C.c_longlong)])
_sig("vh_event_progress", C.c_int, [_evp, C.POINTER(C.c_int), C.POINTER(C.c_double)])
_sig("vh_event_get_field", C.c_int, [_evp, C.c_int, _dp])
_sig("vh_event_freezeout", C.c_int, [_evp, C.POINTER(C.c_int), C.POINTER(C.c_int)])
_sig("vh_event_fetch_surface", C.c_int, [_evp, C.c_void_p, C.c_int, C.POINTER(C.c_int)])
_sig("vh_event_stream", C.c_int, [_evp, C.POINTER(C.c_void_p)])
_sig("vh_event_kernel_launches", C.c_int, [_evp, C.POINTER(C.c_int)])
_sig("vh_event_phase_timing", C.c_int, [_evp, C.c_int])
_sig("vh_event_vorticity", C.c_int, [_evp, C.c_int])
_sig("vh_event_set_sources", C.c_int, [_evp] + [C.c_void_p] * 4)
_sig("vh_event_keep_regulation", C.c_int, [_evp, C.c_int])
_sig("vh_event_init_glauber", C.c_int, [_evp] + [C.c_double] * 7)
_sig("vh_event_init_hotspots", C.c_int, [_evp, C.c_ulonglong] + [C.c_double] * 6)
_sig("vh_event_phase_times", C.c_int, [_evp, C.POINTER(C.c_double), C.POINTER(C.c_longlong)])
_btp = C.c_void_p
_sig("vh_batch_create", C.c_int, [C.POINTER(C.c_void_p), C.c_int, C.POINTER(_btp)])
_sig("vh_batch_destroy", C.c_int, [_btp])
_sig("vh_batch_size", C.c_int, [_btp, C.POINTER(C.c_int)])
_sig("vh_batch_step", C.c_int, [_btp, C.c_int])
_sig("vh_batch_set_active", C.c_int, [_btp, C.c_int, C.c_int])
_sig("vh_batch_kernel_launches", C.c_int, [_btp, C.POINTER(C.c_int)])
_sig("vh_batch_phase_timing", C.c_int, [_btp, C.c_int])
_sig("vh_batch_phase_times", C.c_int, [_btp, C.POINTER(C.c_double), C.POINTER(C.c_longlong)])
_sig("vh_batch_stream", C.c_int, [_btp, C.POINTER(C.c_void_p)])
_sig("vh_event_device_field", C.c_int, [_evp, C.c_int, C.POINTER(C.c_void_p)])
_sig("vh_event_energy_of_T", C.c_int, [_evp, C.c_double, C.POINTER(C.c_double)])
_sig("vh_event_powf_misses", C.c_int, [_evp, C.POINTER(C.c_ulonglong)])
_sig("vh_cornelius_surfaces", C.c_int, [C.c_int, C.c_void_p, C.c_int, C.c_double, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.POINTER(C.c_int)])
_sig("vh_device_math_check", C.c_int, [C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p])
_sig("vh_eos_synthetic_table", C.c_int, [C.c_int] + [C.c_double] * 6 + [_dp])
_sig("vh_eos_eval", C.c_double, [_cfgp, C.c_void_p, C.c_int, C.c_int, C.c_double])
_sig("vh_ic_gubser", C.c_int, [_cfgp, C.c_double, C.c_double, _dp, _dp, _dp, C.c_void_p])
_sig("vh_ic_glauber", C.c_int, [_cfgp, C.c_void_p, C.c_int] + [C.c_double] * 7 + [_dp, _dp, _dp])
_sig("vh_ic_hotspots", C.c_int, [_cfgp, C.c_void_p, C.c_int, C.c_uint64] + [C.c_double] * 6 + [_dp, _dp, _dp])


class VhError(RuntimeError):
    def __init__(self, code: int, where: str):
        msg = lib.vh_last_error().decode(errors="replace")
        super().__init__(f"{where} failed with status {code}: {msg}")
        self.code = code


def check(rc: int, where: str):
    if rc != VH_OK:
        raise VhError(rc, where)


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def default_config() -> VhConfig:
    c = VhConfig()
    check(lib.vh_config_default(C.byref(c)), "vh_config_default")
    return c


# ------------------------------------------------------------------ workloads
def synthetic_eos_table(nrows: int = 2000, T_lo: float = 0.05, e_max: float = 60.0,
                        a: float = 15.6269, dip: float = 0.2, Tc: float = 0.16, w: float = 0.04) -> np.ndarray:
    """Crossover EoS, cs^2(T) = 1/3 - dip exp(-((T-Tc)/w)^2) integrated from T_lo,
    as rows (e [GeV/fm^3], P [GeV/fm^3], s [fm^-3], T [GeV]) uniform in e."""
    rows = np.zeros((nrows, 4))
    check(lib.vh_eos_synthetic_table(nrows, T_lo, e_max, a, dip, Tc, w, rows), "vh_eos_synthetic_table")
    return rows


def hotspot_config(n=101) -> VhConfig:
    """2+1D lumpy event of the batched workload: n x n cells, dx = 0.1 fm,
    tau0 = 0.6 fm/c, dtau = 0.01 fm/c, table EoS, eta/s = 0.08, Gaussian
    zeta/s (bulk evolved), as the 3+1D Glauber event."""
    c = glauber_config(n, n, 1)
    c.dx = c.dy = c.dz = 0.1
    c.t0, c.dt = 0.6, 0.01
    return c


def gubser_config(nx=101, ny=101) -> VhConfig:
    c = default_config()
    c.nx, c.ny, c.nz = nx, ny, 1
    c.dx = c.dy = 0.1
    c.dz = 0.1
    c.t0, c.dt = 1.0, 0.01
    c.etabar = 0.2
    c.T_freezeout_GeV = 0.15
    c.theta = 1.8
    c.eos_kind, c.eos_factor = VH_EOS_CONFORMAL, 15.6269
    c.bulk = 0
    return c


def glauber_config(nx=131, ny=131, nz=61) -> VhConfig:
    c = default_config()
    c.nx, c.ny, c.nz = nx, ny, nz
    c.dx = c.dy = 0.15
    c.dz = 0.2
    c.t0, c.dt = 0.6, 0.015
    c.etabar = 0.08
    c.T_freezeout_GeV = 0.15
    c.theta = 1.8
    c.eos_kind, c.eos_factor = VH_EOS_TABLE, 15.6269
    c.bulk = 1
    c.zeta_law, c.zeta_norm, c.zeta_T0_GeV, c.zeta_width_GeV = VH_ZETA_GAUSSIAN, 0.05, 0.17, 0.02
    return c


@dataclass
class InitialState:
    e: np.ndarray
    p: np.ndarray
    u: np.ndarray          # (4, N)
    pi: np.ndarray | None  # (10, N)
    Pi: np.ndarray | None  # (N,)


def gubser_ic(cfg: VhConfig, q: float = 1.0, T0_GeV: float = 0.3) -> InitialState:
    N = cfg.nx * cfg.ny * cfg.nz
    e, p, u, pi = np.zeros(N), np.zeros(N), np.zeros(4 * N), np.zeros(10 * N)
    check(lib.vh_ic_gubser(C.byref(cfg), q, T0_GeV, e, p, u, _ptr(pi)), "vh_ic_gubser")
    return InitialState(e, p, u.reshape(4, N), pi.reshape(10, N), None)


def glauber_ic(cfg: VhConfig, rows: np.ndarray, R=6.38, a=0.535, sigma_nn=4.2, b=7.0, e0=30.0,
               eta_flat=3.0, eta_sigma=1.3) -> InitialState:
    N = cfg.nx * cfg.ny * cfg.nz
    e, p, u = np.zeros(N), np.zeros(N), np.zeros(4 * N)
    rr = np.ascontiguousarray(rows, dtype=np.float64)
    check(lib.vh_ic_glauber(C.byref(cfg), _ptr(rr), len(rr), R, a, sigma_nn, b, e0, eta_flat, eta_sigma, e, p, u),
          "vh_ic_glauber")
    return InitialState(e, p, u.reshape(4, N), None, np.zeros(N) if cfg.bulk else None)


def hotspot_ic(cfg: VhConfig, rows: np.ndarray | None, seed: int, mean_spots=200.0, w=0.4, k_gamma=1.6,
               amp=20.0, R=6.38, a=0.535) -> InitialState:
    N = cfg.nx * cfg.ny * cfg.nz
    e, p, u = np.zeros(N), np.zeros(N), np.zeros(4 * N)
    rr = None if rows is None else np.ascontiguousarray(rows, dtype=np.float64)
    check(lib.vh_ic_hotspots(C.byref(cfg), _ptr(rr), 0 if rr is None else len(rr), seed, mean_spots, w, k_gamma,
                             amp, R, a, e, p, u), "vh_ic_hotspots")
    return InitialState(e, p, u.reshape(4, N), None, np.zeros(N) if cfg.bulk else None)


def eos_eval(cfg: VhConfig, rows, what: int, x: float) -> float:
    rr = None if rows is None else np.ascontiguousarray(rows, dtype=np.float64)
    return lib.vh_eos_eval(C.byref(cfg), _ptr(rr), 0 if rr is None else len(rr), what, x)


# ---------------------------------------------------------------------- event
class Event:
    """One hydro event resident on the current CUDA device."""

    def __init__(self, cfg: VhConfig, eos_rows: np.ndarray | None = None):
        self.cfg = cfg
        self._rows = None if eos_rows is None else np.ascontiguousarray(eos_rows, dtype=np.float64)
        h = C.c_void_p()
        check(lib.vh_event_create(C.byref(cfg), _ptr(self._rows), 0 if self._rows is None else len(self._rows),
                                  C.byref(h)), "vh_event_create")
        self.h = h
        self.nq = cfg.nq()

    def close(self):
        if getattr(self, "h", None) and lib is not None:
            lib.vh_event_destroy(self.h)
        self.h = None

    def __del__(self):
        self.close()

    def set_initial(self, st: InitialState):
        pi = None if st.pi is None else np.ascontiguousarray(st.pi, dtype=np.float64)
        Pi = None if st.Pi is None else np.ascontiguousarray(st.Pi, dtype=np.float64)
        check(lib.vh_event_set_initial(self.h, np.ascontiguousarray(st.e), np.ascontiguousarray(st.p),
                                       np.ascontiguousarray(st.u).reshape(-1), _ptr(pi), _ptr(Pi)),
              "vh_event_set_initial")
        self._keep = (pi, Pi)

    def step(self, n: int = 1):
        check(lib.vh_event_step(self.h, n), "vh_event_step")

    def status(self):
        s, c = C.c_int(), C.c_longlong()
        rc = lib.vh_event_status(self.h, C.byref(s), C.byref(c))
        return rc, s.value, c.value

    def sync(self):
        rc, s, c = self.status()
        check(rc, "vh_event_status")

    def progress(self):
        n, t = C.c_int(), C.c_double()
        check(lib.vh_event_progress(self.h, C.byref(n), C.byref(t)), "vh_event_progress")
        return n.value, t.value

    def field(self, fid: int) -> np.ndarray:
        ncx, ncy, ncz = self.cfg.padded()
        out = np.zeros(ncx * ncy * ncz)
        check(lib.vh_event_get_field(self.h, fid, out), "vh_event_get_field")
        return out

    def freezeout(self):
        ne, na = C.c_int(), C.c_int()
        check(lib.vh_event_freezeout(self.h, C.byref(ne), C.byref(na)), "vh_event_freezeout")
        return ne.value, na.value

    def surface(self) -> np.ndarray:
        n = C.c_int()
        lib.vh_event_fetch_surface(self.h, None, 0, C.byref(n))
        out = np.zeros((n.value, VH_FO_COLUMNS))
        if n.value:
            check(lib.vh_event_fetch_surface(self.h, _ptr(out), n.value, C.byref(n)), "vh_event_fetch_surface")
        return out

    def launches_per_step(self) -> int:
        n = C.c_int()
        check(lib.vh_event_kernel_launches(self.h, C.byref(n)), "vh_event_kernel_launches")
        return n.value

    def phase_timing(self, enable: bool = True) -> None:
        check(lib.vh_event_phase_timing(self.h, 1 if enable else 0), "vh_event_phase_timing")

    def init_glauber(self, R=6.38, a=0.535, sigma_nn=4.2, b=7.0, e0=30.0, eta_flat=3.0, eta_sigma=1.3):
        """optical-Glauber initial state generated on the device (see glauber_ic)"""
        check(lib.vh_event_init_glauber(self.h, R, a, sigma_nn, b, e0, eta_flat, eta_sigma), "vh_event_init_glauber")

    def init_hotspots(self, seed: int, mean_spots=200.0, w=0.4, k_gamma=1.6, amp=20.0, R=6.38, a=0.535):
        """hotspot initial state generated on the device (see hotspot_ic)"""
        check(lib.vh_event_init_hotspots(self.h, seed, mean_spots, w, k_gamma, amp, R, a), "vh_event_init_hotspots")

    def set_sources(self, src) -> None:
        """dynamical sources: (4, N) interior array (t, x, y, eta components) or None"""
        if src is None:
            check(lib.vh_event_set_sources(self.h, None, None, None, None), "vh_event_set_sources")
            return
        self._src = np.ascontiguousarray(src, dtype=np.float64)
        check(lib.vh_event_set_sources(self.h, *[_ptr(self._src[c]) for c in range(4)]), "vh_event_set_sources")

    def keep_regulation(self, enable: bool = True) -> None:
        """keep the regulation factors of the last stage (fields VH_F_REGFAC, +1)"""
        check(lib.vh_event_keep_regulation(self.h, 1 if enable else 0), "vh_event_keep_regulation")

    def vorticity(self, enable: bool = True) -> None:
        """thermal vorticity now and after every step (fields VH_F_W.., VH_F_BETA..)"""
        check(lib.vh_event_vorticity(self.h, 1 if enable else 0), "vh_event_vorticity")

    def phase_times(self) -> dict:
        """{phase name: (total ms, launches)} since phase_timing(True) or the last call."""
        ms = (C.c_double * 6)()
        n = (C.c_longlong * 6)()
        check(lib.vh_event_phase_times(self.h, ms, n), "vh_event_phase_times")
        return {name: (ms[i], n[i]) for i, name in enumerate(PHASES) if n[i]}

    def stream(self) -> int:
        s = C.c_void_p()
        check(lib.vh_event_stream(self.h, C.byref(s)), "vh_event_stream")
        return s.value or 0

    def powf_misses(self) -> int:
        m = C.c_ulonglong()
        check(lib.vh_event_powf_misses(self.h, C.byref(m)), "vh_event_powf_misses")
        return m.value

    def energy_of_T(self, T: float) -> float:
        e = C.c_double()
        check(lib.vh_event_energy_of_T(self.h, T, C.byref(e)), "vh_event_energy_of_T")
        return e.value


class BatchTuning(C.Structure):
    """vh_batch_tuning: launch configuration of a batch (per phase, indexed as PHASES)."""
    _fields_ = [("fused", C.c_int), ("tile_x", C.c_int * 6), ("tile_y", C.c_int * 6),
                ("persistent", C.c_int * 6), ("stage_ms", C.c_double)]

    def describe(self) -> dict:
        phases = ["fused"] if self.fused else ["source", "flux_x", "flux_y", "flux_eta", "final"]
        return {"fused": bool(self.fused), "stage_ms": self.stage_ms,
                "phases": {p: f"{self.tile_x[PHASES.index(p)]}x{self.tile_y[PHASES.index(p)]}"
                              f"{' persistent' if self.persistent[PHASES.index(p)] else ''}" for p in phases}}


_sig("vh_batch_autotune", C.c_int, [_btp, C.POINTER(BatchTuning)])
_sig("vh_batch_get_tuning", C.c_int, [_btp, C.POINTER(BatchTuning)])
_sig("vh_batch_set_tuning", C.c_int, [_btp, C.POINTER(BatchTuning)])


class Batch:
    """Events advanced together (vh_batch_*): one launch per RK phase for all
    members; the members stay ordinary Events (fields, freezeout, status)."""

    def __init__(self, events):
        self.events = list(events)
        arr = (C.c_void_p * len(self.events))(*[e.h.value if isinstance(e.h, C.c_void_p) else e.h
                                                for e in self.events])
        h = C.c_void_p()
        check(lib.vh_batch_create(arr, len(self.events), C.byref(h)), "vh_batch_create")
        self.h = h

    def close(self):
        if getattr(self, "h", None) and lib is not None:
            lib.vh_batch_destroy(self.h)
        self.h = None

    def __del__(self):
        self.close()

    def step(self, n: int = 1):
        check(lib.vh_batch_step(self.h, n), "vh_batch_step")

    def set_active(self, i: int, active: bool):
        check(lib.vh_batch_set_active(self.h, i, 1 if active else 0), "vh_batch_set_active")

    def autotune(self) -> BatchTuning:
        t = BatchTuning()
        check(lib.vh_batch_autotune(self.h, C.byref(t)), "vh_batch_autotune")
        return t

    def tuning(self) -> BatchTuning:
        t = BatchTuning()
        check(lib.vh_batch_get_tuning(self.h, C.byref(t)), "vh_batch_get_tuning")
        return t

    def set_tuning(self, t: BatchTuning):
        check(lib.vh_batch_set_tuning(self.h, C.byref(t)), "vh_batch_set_tuning")

    def launches_per_step(self) -> int:
        n = C.c_int()
        check(lib.vh_batch_kernel_launches(self.h, C.byref(n)), "vh_batch_kernel_launches")
        return n.value

    def phase_timing(self, enable: bool = True) -> None:
        check(lib.vh_batch_phase_timing(self.h, 1 if enable else 0), "vh_batch_phase_timing")

    def phase_times(self) -> dict:
        ms = (C.c_double * 6)()
        n = (C.c_longlong * 6)()
        check(lib.vh_batch_phase_times(self.h, ms, n), "vh_batch_phase_times")
        return {name: (ms[i], n[i]) for i, name in enumerate(PHASES) if n[i]}

    def stream(self) -> int:
        s = C.c_void_p()
        check(lib.vh_batch_stream(self.h, C.byref(s)), "vh_batch_stream")
        return s.value or 0


class ServerConfig(C.Structure):
    _fields_ = [("hbm_fraction", C.c_double), ("max_events", C.c_int), ("max_steps", C.c_int),
                ("solo_cells", C.c_int)]


class ServerDone(C.Structure):
    _fields_ = [("tag", C.c_ulonglong), ("status", C.c_int), ("steps", C.c_int), ("n_elements", C.c_longlong),
                ("t_submit", C.c_double), ("t_admit", C.c_double), ("t_done", C.c_double)]


class ServerStats(C.Structure):
    _fields_ = [("submitted", C.c_longlong), ("queued", C.c_longlong), ("active", C.c_longlong),
                ("done", C.c_longlong), ("steps", C.c_longlong), ("fo_blocks", C.c_longlong),
                ("batch_builds", C.c_longlong), ("bytes_in_use", C.c_ulonglong), ("budget_bytes", C.c_ulonglong),
                ("t_admit_s", C.c_double), ("t_build_s", C.c_double), ("t_step_s", C.c_double), ("t_fo_s", C.c_double),
                ("t_fo_copy_s", C.c_double), ("fo_elements", C.c_longlong), ("t_retire_s", C.c_double),
                ("t_wait_s", C.c_double)]


_sig("vh_server_config_default", None, [C.POINTER(ServerConfig)])
_sig("vh_server_create", C.c_int, [C.POINTER(ServerConfig), C.c_void_p, C.c_int, C.POINTER(C.c_void_p)])
_sig("vh_server_submit", C.c_int, [C.c_void_p, _cfgp, _dp, _dp, _dp, C.c_void_p, C.c_void_p, C.c_ulonglong])
_sig("vh_server_submit_glauber", C.c_int, [C.c_void_p, _cfgp] + [C.c_double] * 7 + [C.c_ulonglong])
_sig("vh_server_submit_hotspots", C.c_int, [C.c_void_p, _cfgp, C.c_ulonglong] + [C.c_double] * 6 + [C.c_ulonglong])
_sig("vh_server_poll", C.c_int, [C.c_void_p, C.POINTER(ServerDone), C.c_int, C.POINTER(C.c_int)])
_sig("vh_server_take_surface", C.c_int, [C.c_void_p, C.c_ulonglong, C.c_void_p, C.c_longlong,
                                         C.POINTER(C.c_longlong)])
_sig("vh_server_wait", C.c_int, [C.c_void_p, C.c_double])
_sig("vh_server_stats_get", C.c_int, [C.c_void_p, C.POINTER(ServerStats)])
_sig("vh_server_destroy", C.c_int, [C.c_void_p])


class Server:
    """vh_server_*: submit events at any time; a worker thread admits them by
    free device memory, advances them concurrently (small events in one batch
    per kind, events of at least solo_cells cells alone; None: the library's
    default), streams their freezeout surfaces to host memory and retires
    them."""

    def __init__(self, eos_rows=None, hbm_fraction=0.8, max_events=4096, max_steps=0, solo_cells=None):
        c = ServerConfig()
        lib.vh_server_config_default(C.byref(c))
        c.hbm_fraction, c.max_events, c.max_steps = hbm_fraction, max_events, max_steps
        if solo_cells is not None:
            c.solo_cells = solo_cells
        self.solo_cells = c.solo_cells
        self._rows = None if eos_rows is None else np.ascontiguousarray(eos_rows, dtype=np.float64)
        h = C.c_void_p()
        check(lib.vh_server_create(C.byref(c), _ptr(self._rows), 0 if self._rows is None else len(self._rows),
                                   C.byref(h)), "vh_server_create")
        self.h = h

    def submit(self, cfg: VhConfig, st: InitialState, tag: int):
        pi = None if st.pi is None else np.ascontiguousarray(st.pi, dtype=np.float64)
        Pi = None if st.Pi is None else np.ascontiguousarray(st.Pi, dtype=np.float64)
        check(lib.vh_server_submit(self.h, C.byref(cfg), np.ascontiguousarray(st.e), np.ascontiguousarray(st.p),
                                   np.ascontiguousarray(st.u).reshape(-1), _ptr(pi), _ptr(Pi), tag),
              "vh_server_submit")

    def submit_glauber(self, cfg: VhConfig, tag: int, R=6.38, a=0.535, sigma_nn=4.2, b=7.0, e0=30.0,
                       eta_flat=3.0, eta_sigma=1.3):
        """an optical-Glauber event whose initial state is generated on the device at admission"""
        check(lib.vh_server_submit_glauber(self.h, C.byref(cfg), R, a, sigma_nn, b, e0, eta_flat, eta_sigma, tag),
              "vh_server_submit_glauber")

    def submit_hotspots(self, cfg: VhConfig, tag: int, seed: int, mean_spots=200.0, w=0.4, k_gamma=1.6, amp=20.0,
                        R=6.38, a=0.535):
        """a hotspot event whose initial state is generated on the device at admission"""
        check(lib.vh_server_submit_hotspots(self.h, C.byref(cfg), seed, mean_spots, w, k_gamma, amp, R, a, tag),
              "vh_server_submit_hotspots")

    def poll(self, max_n: int = 1024) -> list:
        out = (ServerDone * max_n)()
        n = C.c_int()
        check(lib.vh_server_poll(self.h, out, max_n, C.byref(n)), "vh_server_poll")
        return [out[i] for i in range(n.value)]

    def take_surface(self, tag: int) -> np.ndarray:
        n = C.c_longlong()
        lib.vh_server_take_surface(self.h, tag, None, 0, C.byref(n))
        out = np.zeros((n.value, VH_FO_COLUMNS))
        check(lib.vh_server_take_surface(self.h, tag, _ptr(out), n.value, C.byref(n)), "vh_server_take_surface")
        return out

    def wait(self, timeout_s: float = 600.0):
        check(lib.vh_server_wait(self.h, timeout_s), "vh_server_wait")

    def stats(self) -> dict:
        st = ServerStats()
        check(lib.vh_server_stats_get(self.h, C.byref(st)), "vh_server_stats_get")
        return {k: getattr(st, k) for k, _ in ServerStats._fields_}

    def close(self):
        if getattr(self, "h", None) and lib is not None:
            lib.vh_server_destroy(self.h)
        self.h = None

    def __del__(self):
        self.close()


def run_like_server(cfg: VhConfig, rows, st, max_steps: int = 0):
    """One event alone with the server's cadence: freezeout blocks before loop
    index n when n % fo_factor == 0, retired after three blocks with no cell
    above e_F, at max_steps, or when the device reports an error.  st is an
    InitialState or a callable that initialises the Event (a device generator).
    Returns (steps, surface, status)."""
    ev = Event(cfg, rows)
    if callable(st):
        st(ev)
    else:
        ev.set_initial(st)
    fac = max(1, cfg.fo_factor)
    steps, last, zero, parts, status = 0, -1, 0, [], VH_OK

    def to_block():
        k = 1 if last == steps else 0
        while (steps + k + 1) % fac:
            k += 1
        return k

    while True:
        k = to_block()
        if max_steps:
            k = min(k, max(0, max_steps - steps))
        if k:
            ev.step(k)
            steps += k
        if to_block() == 0:
            last = steps
            n, na = ev.freezeout()
            if n:
                parts.append(ev.surface())
            status = ev.status()[0]
            if status != VH_OK:
                break
            zero += na == 0
        if zero >= 3 or (max_steps and steps >= max_steps):
            break
    if status == VH_OK:
        status = ev.status()[0]        # errors of the steps after the last block
    ev.close()
    return steps, (np.concatenate(parts) if parts else np.zeros((0, VH_FO_COLUMNS))), status


def make_tuning(fused: bool, tx: int, persistent: bool) -> BatchTuning:
    t = BatchTuning()
    t.fused = 1 if fused else 0
    for i in range(6):
        t.tile_x[i], t.tile_y[i], t.persistent[i] = tx, 128 // tx, 1 if persistent else 0
    return t


def cornelius_surfaces(dim: int, cubes: np.ndarray, value0: float, dx) -> tuple[np.ndarray, np.ndarray]:
    """Cornelius elements (centroid, normal) of each cube on the device."""
    cubes = np.ascontiguousarray(cubes, dtype=np.float64).reshape(len(cubes), -1)
    dxa = np.ascontiguousarray(dx, dtype=np.float64)
    counts = np.zeros(len(cubes), dtype=np.int32)
    n = C.c_int()
    cap = 10 * len(cubes)
    out = np.zeros((cap, 2 * dim))
    check(lib.vh_cornelius_surfaces(dim, _ptr(cubes), len(cubes), value0, _ptr(dxa), _ptr(out), cap, _ptr(counts),
                                    C.byref(n)), "vh_cornelius_surfaces")
    return out[:n.value], counts


def device_math(which: int, a: np.ndarray, b: np.ndarray | None = None) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.float64)
    bb = None if b is None else np.ascontiguousarray(b, dtype=np.float64)
    out = np.zeros_like(a)
    check(lib.vh_device_math_check(which, _ptr(a), _ptr(bb), len(a), _ptr(out)), "vh_device_math_check")
    return out


def interior(cfg: VhConfig, a: np.ndarray) -> np.ndarray:
    ncx, ncy, ncz = cfg.padded()
    return a.reshape(ncz, ncy, ncx)[2:-2, 2:-2, 2:-2]


def face_cells(cfg: VhConfig, a: np.ndarray) -> np.ndarray:
    """Interior plus the face ghost cells (the cells the stencils read)."""
    ncx, ncy, ncz = cfg.padded()
    A = a.reshape(ncz, ncy, ncx)
    parts = [A[2:-2, 2:-2, :], A[2:-2, :, 2:-2].transpose(0, 2, 1), A[:, 2:-2, 2:-2].transpose(1, 2, 0)]
    return np.concatenate([p.reshape(-1) for p in parts])
