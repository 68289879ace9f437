#!/usr/bin/env python
"""Benchmark of the B200 KT RK2 step (cell-updates/s).

Workload (default): the 3+1D optical-Glauber event, 131x131x61 cells,
dx=dy=0.15 fm, deta=0.2, tau0=0.6 fm/c, dtau=0.015 fm/c, 2000-row synthetic
crossover EoS table, eta/s=0.08, Gaussian zeta/s (bulk evolved, 15 conserved
components), FP64 in the reference's operation order.  One "step" is one RK2
step over the whole lattice.  Synthetic seeded inputs stand in for physics
event generators (none are public for this path).

  value  cell-updates/s with the state resident in HBM, CUDA events on the
         event's stream around K steps (the state, ~580 MB, is larger than
         the 126 MB L2, so no flush is needed between steps)
  e2e    the same metric through the C ABI with pinned host buffers: upload of
         the initial condition, K steps, download of the energy density, timed
         on the host clock
  roofline  dominant kernel = the one with the largest share of the timed
         device time (on large lattices the x/y/eta flux kernel, else the
         fused stage kernel); its launches are timed with CUDA events that the
         library records between the stage kernels on the event's stream
         during the timed steps.  Algorithmic bytes per launch = per-cell
         compulsory words of that phase x interior cells (PHASE_WORDS);
         peak = measured HBM copy bandwidth; traffic = DRAM bytes per launch
         from an ncu capture of the same workload (NCU_TRAFFIC)
  cpu_baseline  the reference's own sources (oracle/_ref, OpenMP over all host
         cores) on a bounded sample of the same workload

`--impl reference` times the reference CPU implementation instead (rank 0).
Multi-GPU: independent replicas (events share nothing), max time over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "cpu-vh_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

BYTES_PER_CELL_STEP = 856          # (5*Nq + 32) * 8 with Nq = 15


def phase_words(nq):
    """Compulsory FP64 words per interior cell of one launch of each phase."""
    return {
        # q, u, up, e, p read; q* written
        "source": 2 * nq + 10,
        # q stencil (each value once), e, u^tau, u^dir, q* read; q* written
        "flux": 3 * nq + 3,
        # q* and e read (+ q^n in stage 2), q, e, p, u written: mean of stages
        "final": 2.5 * nq + 7,
        # the whole stage in one kernel: (46 + 61) / 2 words at Nq = 15
        "fused": 2.5 * nq + 16,
    }


# DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum) from the
# ncu captures kept in profiles/kt_flux_lines_kernel_glauber_131x131x61.md
# (FP64: mean of the x, y, eta launches) and
# profiles/kt_flux_face_kernel_glauber_131x131x61_mixed.md (mixed)
NCU_TRAFFIC = {("glauber_3p1d", "fp64", "flux"): 381.57e6, ("glauber_3p1d", "fp64", "source"): 336.57e6,
               ("glauber_3p1d", "mixed", "flux"): 388.30e6, ("glauber_3p1d", "mixed", "source"): 322.01e6}


# FP64 pipe use of the dominant kernel from the same captures: mean over the
# x, y, eta launches of sm__pipe_fp64_cycles_active (% of peak sustained),
# the launch's duration under ncu (ms) and its FP64-pipe warp instructions.
# The fraction of the FP64 pipe's peak at live speed is that percentage
# scaled by the ratio of the durations.
NCU_FP64 = {("glauber_3p1d", "fp64", "flux"): (27.01, 0.3473, 51.47e6)}


# batched flux launches: DRAM bytes per cell from ncu captures of the same
# batch cut to its first 64 events (1 312 264 cells), scaled by the cell count
# (the traffic of a launch is per cell: each member's stencil once), from
# profiles/kt_batch_kernel_hotspots_64ev_fp64.md and
# profiles/kt_batch_face_kernel_hotspots_64ev_mixed.md
NCU_TRAFFIC_PER_CELL = {("fp64", "flux"): 371.7, ("mixed", "flux"): 371.6}


# steps of the mixed-precision error report: the Gubser event's 300 steps
# (tau = 4 fm/c); the Glauber event to tau = 12.6 fm/c (800 steps) -- at step
# 909 its FP64 evolution, bit-identical to the reference's, trips the
# reference's NaN guard (EnergyMomentumTensor.cpp:197-203) in the dilute
# edge.  No cell is above e_F after about step 150 (Gubser) and 400
# (Glauber): the reference's stop rule would end the events there.
PRECISION_STEPS = {"gubser_2p1d": 300, "glauber_3p1d": 800}


KERNEL_NAMES = {"source": "kt_source_kernel", "flux": "kt_flux_lines_kernel (x, y, eta)",
                "final": "kt_final_kernel", "fused": "kt_stage_kernel"}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="glauber_3p1d",
                    choices=["glauber_3p1d", "gubser_2p1d", "batch_hotspots_2p1d", "serve_mix"])
    ap.add_argument("--rate", type=float, default=6.0, help="serve_mix: Poisson arrival rate (events/s)")
    ap.add_argument("--max-steps", type=int, default=100, help="serve_mix: RK2 steps after which an event retires")
    ap.add_argument("--events", type=int, default=256, help="batch_hotspots_2p1d: events in the batch")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"],
                    help="mixed: FP32 limiter/flux/source arithmetic, FP64 accumulation and root solve")
    ap.add_argument("--no-baseline", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end leg")
    ap.add_argument("--precision-steps", type=int, default=0,
                    help="--precision mixed: steps of the error report (0: the workload's whole event)")
    ap.add_argument("--fo-blocks", type=int, default=4,
                    help="freezeout blocks timed after the steps (0: none), one per fo_factor steps")
    ap.add_argument("--no-extras", action="store_true",
                    help="glauber_3p1d FP64 line without its batch / precision / serve records")
    ap.add_argument("--serve-events", type=int, default=24,
                    help="events of the serve record of the default line (each run to the stop rule)")
    return ap.parse_args()


DESC_GUBSER = ("gubser_2p1d: 101x101x1, dx=0.1 fm, tau0=1.0, dtau=0.01, conformal a=15.6269, eta/s=0.2, "
               "theta=1.8, T0=0.3 GeV, pi at Navier-Stokes")
DESC_GLAUBER = ("glauber_3p1d: 131x131x61, dx=dy=0.15 fm, deta=0.2, tau0=0.6, dtau=0.015, Au+Au optical Glauber "
                "b=7 fm, peak 30 GeV/fm^3, 2000-row synthetic crossover EoS, eta/s=0.08, Gaussian zeta/s (bulk on), "
                "FP64")


def desc_batch(n_events):
    return (f"batch_hotspots_2p1d: {n_events} events, n x n x 1 with n uniform in {{81..201 step 20}} (seed 2024), "
            "dx=0.1 fm, tau0=0.6, dtau=0.01, Poisson(200) hotspots of width 0.4 fm, Gamma(1.6) amplitudes, "
            "mean peak 20 GeV/fm^3, centres in the b=0 Woods-Saxon overlap, 2000-row synthetic EoS, eta/s=0.08, "
            "Gaussian zeta/s (bulk on), FP64")


def single_config(desc, nx, ny, nz, nq, world):
    """the config record of a single-event line (both arms print the same)"""
    state_mb = (3 * nq + 16) * (nx + 4) * (ny + 4) * (nz + 4) * 8 / 1e6   # q x3, e/p x2, u x3 planes
    l2 = (f"state {state_mb:.0f} MB > 126 MB L2, no flush" if state_mb > 126 else
          f"state {state_mb:.0f} MB fits in the 126 MB L2 (not flushed; latency-bound small lattice)")
    return {"workload": desc, "cells": nx * ny * nz, "parallelism": f"replicas x{world}", "l2": l2}


def workload(name):
    import vh
    if name == "gubser_2p1d":
        cfg = vh.gubser_config()
        return cfg, None, vh.gubser_ic(cfg), "conf", DESC_GUBSER
    cfg = vh.glauber_config()
    rows = vh.synthetic_eos_table()
    return cfg, rows, vh.glauber_ic(cfg, rows), "table", DESC_GLAUBER


BATCH_SIZES = (81, 101, 121, 141, 161, 181, 201)
EVENT_STEPS = 300      # RK2 steps of one event for events/s (the Gubser event's step count)


def batch_sizes(n_events):
    """n of each n x n event of the batched workload, drawn uniformly from
    BATCH_SIZES (seed 2024)"""
    import numpy as np
    rng = np.random.default_rng(2024)
    return [int(x) for x in rng.choice(BATCH_SIZES, size=n_events)]


def batch_workload(n_events):
    """Lumpy 2+1D events, n x n with n drawn uniformly from BATCH_SIZES
    (seed 2024), hotspot initial conditions seeded with the event index."""
    import vh
    rows = vh.synthetic_eos_table()
    cfgs = [vh.hotspot_config(n) for n in batch_sizes(n_events)]
    ics = [vh.hotspot_ic(c, rows, seed=i) for i, c in enumerate(cfgs)]
    return cfgs, rows, ics, desc_batch(n_events)


def precision_report(cfg, rows, st, steps, ev_mixed=None):
    """Error of a mixed-precision event after `steps` steps against the FP64
    path (bit-identical to the oracle), next to the FP64 path's own
    sensitivity: the same FP64 run from an initial energy density scaled by
    (1 + 2^-50).  Relative L-infinity = max|a - b| / max|b|, relative L2 =
    |a - b|_2 / |b|_2, over the interior cells; then the freezeout over the
    same steps (element count, sums of d sigma_mu) of single events.  ev_mixed:
    the mixed event to judge (a batch member), else a single mixed event is
    run."""
    import numpy as np
    import vh
    fields = [("e", vh.VH_F_E), ("ut", vh.VH_F_UT), ("ux", vh.VH_F_UT + 1), ("uy", vh.VH_F_UT + 2),
              ("un", vh.VH_F_UT + 3), ("pixx", 8), ("pixy", 9), ("piyy", 11), ("pinn", 13)]
    if cfg.bulk:
        fields.append(("Pi", 14))

    def run(ic, prec=vh.VH_PREC_FP64):
        e = vh.Event(cfg.copy(precision=prec), rows)
        e.set_initial(ic)
        e.step(steps)
        e.sync()
        return e

    e_F = vh.eos_eval(cfg, rows, 3, cfg.T_freezeout_GeV / 0.197326938)

    def errs(a_ev, b_ev):
        """relative L-inf / L2 over the interior, and over the cells above e_F
        (the fluid that has not frozen out yet) of the FP64 run b_ev"""
        out = {}
        hot = vh.interior(cfg, b_ev.field(vh.VH_F_E)).ravel() > e_F
        for name, fid in fields:
            a = vh.interior(cfg, a_ev.field(fid)).ravel()
            b = vh.interior(cfg, b_ev.field(fid)).ravel()
            d = a - b
            out[name] = {"linf": float(np.max(np.abs(d)) / max(np.max(np.abs(b)), 1e-300)),
                         "l2": float(np.linalg.norm(d) / max(np.linalg.norm(b), 1e-300))}
            if hot.any():
                out[name]["linf_above_eF"] = float(np.max(np.abs(d[hot])) / max(np.max(np.abs(b[hot])), 1e-300))
                out[name]["l2_above_eF"] = float(np.linalg.norm(d[hot]) / max(np.linalg.norm(b[hot]), 1e-300))
        out["cells_above_eF"] = int(hot.sum())
        return out

    bumped = vh.InitialState(st.e * (1 + 2.0 ** -50), st.p, st.u, st.pi, st.Pi)
    own = ev_mixed is None
    if own:
        # the three runs side by side, compared at eight points of the event:
        # while fluid is above e_F, the error there is the one that reaches
        # the freezeout surface
        def make(ic, prec=vh.VH_PREC_FP64):
            e = vh.Event(cfg.copy(precision=prec), rows)
            e.set_initial(ic)
            return e
        ref, floor, ev_mixed = make(st), make(bumped), make(st, vh.VH_PREC_MIXED)
        marks, done = [], 0
        for k in range(1, 9):
            n = steps * k // 8 - done
            for e in (ref, floor, ev_mixed):
                e.step(n)
                e.sync()
            done += n
            marks.append({"step": done, "mixed_vs_fp64": errs(ev_mixed, ref), "fp64_sensitivity": errs(floor, ref)})
        rep = {"steps": steps, "tau_fm": cfg.t0 + steps * cfg.dt, "mixed_vs_fp64": marks[-1]["mixed_vs_fp64"],
               "fp64_sensitivity": marks[-1]["fp64_sensitivity"]}
        for key in ("mixed_vs_fp64", "fp64_sensitivity"):
            hot = [m[key]["e"].get("linf_above_eF") for m in marks if "linf_above_eF" in m[key]["e"]]
            rep[key]["e_linf_above_eF_max_over_event"] = max(hot) if hot else None
        rep["checkpoints"] = [{"step": m["step"], "cells_above_eF": m["mixed_vs_fp64"]["cells_above_eF"],
                               "e_linf_mixed": m["mixed_vs_fp64"]["e"]["linf"],
                               "e_linf_above_eF_mixed": m["mixed_vs_fp64"]["e"].get("linf_above_eF"),
                               "e_linf_fp64_sensitivity": m["fp64_sensitivity"]["e"]["linf"],
                               "e_linf_above_eF_fp64_sensitivity": m["fp64_sensitivity"]["e"].get("linf_above_eF")}
                              for m in marks]
        for e in (ref, floor, ev_mixed):
            e.close()
    else:
        ref, floor = run(st), run(bumped)
        rep = {"steps": steps, "tau_fm": cfg.t0 + steps * cfg.dt, "mixed_vs_fp64": errs(ev_mixed, ref),
               "fp64_sensitivity": errs(floor, ref)}
        for e in (ref, floor):
            e.close()

    # freezeout over the same steps, a block every fo_factor steps as run()
    # does: element count and the sums of d sigma_mu over all elements
    def surf(ic, prec):
        e = vh.Event(cfg.copy(precision=prec), rows)
        e.set_initial(ic)
        fac = max(1, cfg.fo_factor)
        n, ds = 0, np.zeros(4)
        for _ in range(max(1, steps // fac)):
            e.step(fac)
            ne, _ = e.freezeout()
            if ne:
                n += ne
                ds += e.surface()[:, 4:8].sum(axis=0)
        e.close()
        return n, ds

    n64, s64 = surf(st, vh.VH_PREC_FP64)
    fo = {"blocks": max(1, steps // max(1, cfg.fo_factor)), "elements_fp64": n64}
    for key, (ic, prec) in (("mixed_vs_fp64", (st, vh.VH_PREC_MIXED)), ("fp64_sensitivity", (bumped, vh.VH_PREC_FP64))):
        n, sm = surf(ic, prec)
        fo[key] = {"elements": n, "count_rel": abs(n - n64) / max(n64, 1),
                   "dsigma_sum_rel_linf": float(np.max(np.abs(sm - s64)) / max(np.max(np.abs(s64)), 1e-300))}
    rep["freezeout"] = fo
    return rep


def serve_stream(n_events, rate, seed=2025):
    """The served mix: 70 % 2+1D lumpy events (n x n, n uniform in 61..201
    step 20, hotspot initial conditions) and 30 % 3+1D smooth events (n x n x
    n_eta, n uniform in 101..201 step 20, n_eta in 21..81 step 20, optical
    Glauber with b uniform in 0-12 fm); Poisson arrivals at `rate`.  Each
    event is (arrival time, config, generator kind, generator argument): the
    initial states are made on the device when the event is admitted."""
    import numpy as np
    import vh
    rng = np.random.default_rng(seed)
    rows = vh.synthetic_eos_table()
    t, out = 0.0, []
    for i in range(n_events):
        t += rng.exponential(1.0 / rate)
        if rng.random() < 0.7:
            c = vh.hotspot_config(int(rng.choice(np.arange(61, 202, 20))))
            c.fo_factor = 10
            out.append((t, c, "hotspots", 10_000 + i))
        else:
            n = int(rng.choice(np.arange(101, 202, 20)))
            c = vh.glauber_config(n, n, int(rng.choice([21, 41, 61, 81])))
            c.fo_factor = 10
            out.append((t, c, "glauber", float(rng.uniform(0.0, 12.0))))
    desc = (f"serve_mix: {n_events} events, Poisson arrivals at {rate:g}/s (seed {seed}); 70% 2+1D hotspot events "
            "n x n, n in 61..201 step 20; 30% 3+1D optical-Glauber events n x n x n_eta, n in 101..201 step 20, "
            "n_eta in 21..81 step 20, b uniform 0-12 fm; initial states generated on the device; freezeout every "
            "10 steps, surfaces to host")
    return out, rows, desc


def _init_of(kind, arg):
    if kind == "hotspots":
        return lambda ev: ev.init_hotspots(seed=arg)
    return lambda ev: ev.init_glauber(b=arg)


def pct(xs, q):
    import numpy as np
    return float(np.percentile(np.asarray(xs), q)) if len(xs) else None


def run_serve(args, rank):
    line = serve_record(args.events, args.rate, args.max_steps, args.precision)
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def serve_record(n_events, rate, max_steps, precision):
    """The event server under a Poisson stream, next to the same stream served
    one event at a time by the plain FP64 path (FCFS queue over the measured
    per-event service times).  max_steps 0: every event runs to the
    reference's stop rule (three freezeout blocks with no cell above e_F,
    HydroPlugin.cpp:267-281) or to a device error."""
    import numpy as np
    import vh
    from types import SimpleNamespace
    args = SimpleNamespace(events=n_events, rate=rate, max_steps=max_steps, precision=precision)
    stream, rows, desc = serve_stream(args.events, args.rate)
    mixed = args.precision == "mixed"
    prec = vh.VH_PREC_MIXED if mixed else vh.VH_PREC_FP64
    srv = vh.Server(rows, hbm_fraction=0.8, max_steps=args.max_steps)
    solo_cells = srv.solo_cells
    # warm the server (tuning, modules) on one small event outside the timed stream
    wc = vh.hotspot_config(61).copy(precision=prec)
    srv.submit(wc, vh.hotspot_ic(wc, rows, seed=1), 1 << 40)
    srv.wait(600)
    srv.poll()
    srv.take_surface(1 << 40)
    t_start = time.perf_counter()
    base = None
    for i, (t_arr, c, kind, arg) in enumerate(stream):
        dt = t_arr - (time.perf_counter() - t_start)
        if dt > 0:
            time.sleep(dt)
        if kind == "hotspots":
            srv.submit_hotspots(c.copy(precision=prec), i, seed=arg)
        else:
            srv.submit_glauber(c.copy(precision=prec), i, b=arg)
    srv.wait(3600)
    done = srv.poll(len(stream) + 16)
    stats = srv.stats()
    lat = [d.t_done - d.t_submit for d in done]
    first = min(d.t_submit for d in done)
    span = max(d.t_done for d in done) - first
    cells = sum(d.steps * c.nx * c.ny * c.nz for d, (_, c, _, _) in zip(sorted(done, key=lambda d: d.tag), stream))
    bad = [d.tag for d in done if d.status != 0]
    srv.close()

    # the plain path: each event alone, FP64, same cadence and cap, FCFS
    service, serial_bad = [], []
    for i, (_, c, kind, arg) in enumerate(stream):
        t0 = time.perf_counter()
        _, _, status = vh.run_like_server(c.copy(precision=vh.VH_PREC_FP64), rows, _init_of(kind, arg),
                                          max_steps=args.max_steps)
        service.append(time.perf_counter() - t0)
        if status:
            serial_bad.append(i)
    free_at, slat = 0.0, []
    for (t_arr, _, _, _), sv in zip(stream, service):
        start = max(t_arr, free_at)
        free_at = start + sv
        slat.append(free_at - t_arr)
    serial_span = free_at - stream[0][0]

    line = {"metric": "events/s", "value": len(done) / span, "unit": "events/s", "n_gpus": 1,
            "steps": None, "warmup": 1, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32/f64 mixed" if mixed else "f64", "data": "synthetic",
            "config": {"workload": desc, "events": len(stream), "max_steps": args.max_steps,
                       "admission": "80% of free HBM", "precision": args.precision,
                       "solo_cells": solo_cells},
            "latency_s": {"p50": pct(lat, 50), "p95": pct(lat, 95), "p99": pct(lat, 99), "max": max(lat)},
            "cell_updates_per_s": cells / span,
            "server": {k: stats[k] for k in ("steps", "fo_blocks", "batch_builds", "t_admit_s", "t_build_s",
                                             "t_step_s", "t_fo_s", "t_fo_copy_s", "fo_elements", "t_retire_s", "t_wait_s")} | {"events_with_device_error": bad},
            "serial_plain_fp64": {"events_per_s": len(stream) / serial_span,
                                  "latency_s": {"p50": pct(slat, 50), "p95": pct(slat, 95), "p99": pct(slat, 99)},
                                  "events_with_device_error": serial_bad,
                                  "how": "each event alone through vh_event_step/freezeout (FP64), same cadence "
                                         "and step cap; FCFS queue over the measured service times"}}
    line["server_vs_serial_events_per_s"] = line["value"] / line["serial_plain_fp64"]["events_per_s"]
    line["steps_per_event"] = {"mean": float(np.mean([d.steps for d in done])), "max": int(max(d.steps for d in done))}
    return line


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_baseline(cfg, rows, st, variant, steps=2):
    """The reference's own code (oracle/_ref) on all host cores, `steps` RK2 steps."""
    import oracle as O
    threads = os.cpu_count() or 1
    N = cfg.nx * cfg.ny * cfg.nz
    if O.ref_available(variant):
        ref = O.RefEvent(variant, cfg, rows, threads=threads)
        kind = "reference"
    else:
        ref = O.OracleEvent(cfg, rows)
        threads = 1
        kind = "port"
    ref.set_initial(st)
    if kind == "reference":
        ref.time_steps(1)                      # warm-up step
        secs = ref.time_steps(steps)
    else:
        ref.step(1)
        t0 = time.perf_counter()
        ref.step(steps)
        secs = time.perf_counter() - t0
    return {"value": N * steps / secs, "unit": "cell-updates/s", "cores": threads, "kind": kind,
            "sample": f"{steps} RK2 steps of the same {cfg.nx}x{cfg.ny}x{cfg.nz} event after 1 warm-up step, "
                      f"{threads} OpenMP threads" + (" (reference sources, -O3 -ffp-contract=off)" if kind == "reference"
                                                      else " (C restatement, 1 thread)"),
            "seconds": secs}


def reference_freezeout(cfg, rows, variant):
    """One freezeout block of the reference's own code (serial Cornelius scan
    that writes its surface.dat lines, FreezeOut.cpp:200-361), timed on the
    host clock after the first block and fo_factor more steps.  Its cost is
    ~90 us per cell (~100 s for a 10^6-cell lattice), so it runs on a bounded
    sample: the same event on a lattice of about 6e4 cells covering the same
    volume, scaled to the full lattice by the cell count."""
    import tempfile
    import oracle as O
    import vh
    if variant != "table" or not O.ref_available(variant):
        return None
    N = cfg.nx * cfg.ny * cfg.nz
    f = max(1.0, (N / 6e4) ** (1.0 / (3 if cfg.nz > 1 else 2)))
    sc = cfg.copy(nx=max(8, int(round(cfg.nx / f))), ny=max(8, int(round(cfg.ny / f))),
                  nz=max(1, int(round(cfg.nz / f))) if cfg.nz > 1 else 1)
    sc.dx, sc.dy = cfg.dx * cfg.nx / sc.nx, cfg.dy * cfg.ny / sc.ny
    sc.dz = cfg.dz * cfg.nz / sc.nz
    ref = O.RefEvent(variant, sc, rows, threads=os.cpu_count() or 1)
    ref.set_initial(vh.glauber_ic(sc, rows))
    ref.step(2)
    path = os.path.join(tempfile.gettempdir(), f"vh_ref_surface_{os.getpid()}.dat")
    ref.freezeout(path)
    ref.step(max(1, cfg.fo_factor))
    t0 = time.perf_counter()
    ref.freezeout(path)
    secs = time.perf_counter() - t0
    os.remove(path)
    Ns = sc.nx * sc.ny * sc.nz
    return {"ms_per_block": secs * 1e3 * N / Ns, "cores": 1, "kind": "reference",
            "sample": f"one block on the same event at {sc.nx}x{sc.ny}x{sc.nz} ({secs:.2f} s), scaled by the "
                      f"cell count to {cfg.nx}x{cfg.ny}x{cfg.nz}; serial, writes its surface.dat lines"}


def _ref_steps_timed(refs, args, budget_s):
    """warm-up then K timed steps of every reference event, K bounded so the
    timed part stays within about budget_s seconds"""
    def step_all(k):
        for r in refs:
            r.step(k)
    t0 = time.perf_counter()
    step_all(1)
    est = time.perf_counter() - t0
    warm = max(0, min(args.warmup, int(budget_s / 5 / max(est, 1e-3))) - 1)
    if warm:
        step_all(warm)
    k = max(1, min(args.steps, int(budget_s / max(est, 1e-3))))
    t0 = time.perf_counter()
    step_all(k)
    return k, time.perf_counter() - t0


def run_reference(args):
    """The reference's own CPU implementation (its sources compiled in place
    by oracle/ref.mk into oracle/_ref) on the same workload and config.  The
    inputs come from the copy of the workload generators linked into those
    libraries (oracle/workload_gen.c) and the reference's own EoS, so this
    process loads no library of this repository but oracle/_ref."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import oracle as O
    threads = os.cpu_count() or 1
    batch = args.workload == "batch_hotspots_2p1d"
    if batch:
        variant = "table"
        sizes = batch_sizes(args.events)[:8]
        cfgs = [O.hotspot_workload(n) for n in sizes]
        desc, sample = desc_batch(args.events), "the first 8 events of the batch, one after another"
    elif args.workload == "gubser_2p1d":
        variant, cfgs, desc, sample = "conf", [O.gubser_workload()], DESC_GUBSER, "the event"
    else:
        variant, cfgs, desc, sample = "table", [O.glauber_workload()], DESC_GLAUBER, "the event"
    if not O.ref_available(variant):
        print(json.dumps({"impl": "reference", "unavailable": "the reference's sources were not compiled "
                          "(oracle/_ref missing: build() needs the reference tree)"}), flush=True)
        return 0
    lib = O.ref_lib_path(variant)
    rows = O.synthetic_eos_rows(O.load_gen_lib(lib)) if variant == "table" else None

    def make_refs(var, nthreads):
        out = []
        for i, c in enumerate(cfgs):
            r = O.RefEvent(var, c, rows, threads=nthreads)
            gl = O.load_gen_lib(O.ref_lib_path(var))
            if batch:
                st = O.hotspot_state(c, r.pressure, seed=i, lib=gl)
            elif var.startswith("conf"):
                st = O.gubser_state(c, lib=gl)
            else:
                st = O.glauber_state(c, r.pressure, lib=gl)
            r.set_initial(st)
            out.append(r)
        return out

    N = sum(c.nx * c.ny * c.nz for c in cfgs)
    # the reference keeps its state in process globals: one event per library
    # at a time, so a batch sample runs its events one after another
    if batch:
        cells, secs = 0, 0.0
        gl = O.load_gen_lib(lib)
        for i, c in enumerate(cfgs):
            ev = O.RefEvent(variant, c, rows, threads=threads)
            ev.set_initial(O.hotspot_state(c, ev.pressure, seed=i, lib=gl))
            k, sc = _ref_steps_timed([ev], args, 150.0 / len(cfgs))
            cells += k * c.nx * c.ny
            secs += sc
        v, k, ms_step = cells / secs, None, None
    else:
        refs = make_refs(variant, threads)
        k, secs = _ref_steps_timed(refs, args, 120.0)
        v = N * k / secs
        ms_step = secs / k * 1e3
    line = {"metric": "cell-updates/s", "value": v, "unit": "cell-updates/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "impl": "reference",
            "config": ({"workload": desc, "events": args.events, "parallelism": f"replicas x{args.gpus}"} if batch
                       else single_config(desc, cfgs[0].nx, cfgs[0].ny, cfgs[0].nz, 15 if cfgs[0].bulk else 14,
                                          args.gpus)),
            "timed_steps": k,
            "ghost_cells": "race-fixed restatement of setGhostCells (private loop indices; the shipped loops "
                           "share them across OpenMP threads, DynamicalVariables.cpp:290-291, :324-325, :358-359)",
            "build": "the reference's sources, g++ -O3 -fopenmp -std=c++11 -march=x86-64-v3 -ffp-contract=off",
            "cpu_baseline": {"value": v, "unit": "cell-updates/s", "cores": threads, "kind": "reference",
                             "sample": (f"{k} RK2 steps of {sample}" if k else f"RK2 steps of {sample}") +
                                       f", of {args.steps} requested (bounded to ~150 s), {threads} OpenMP threads"},
            "e2e": {"value": v, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if not batch:
        # the same code on one thread, and as the shipped CMake flags build it
        # (-march=native, the compiler's own multiply-add contraction), on a
        # bounded sample of the same event
        del refs
        one = make_refs(variant, 1)
        k1, s1 = _ref_steps_timed(one, argparse.Namespace(steps=2, warmup=1), 25.0)
        line["one_thread"] = {"value": N * k1 / s1, "unit": "cell-updates/s", "cores": 1,
                              "sample": f"{k1} RK2 steps of the event after 1 warm-up step"}
        del one
        shipped = variant + "_shipped"
        if O.ref_available(shipped) and O.shipped_runs_here():
            sh = make_refs(shipped, threads)
            k2, s2 = _ref_steps_timed(sh, args, 30.0)
            line["shipped_flags"] = {"value": N * k2 / s2, "unit": "cell-updates/s", "cores": threads,
                                     "build": O.shipped_build_flags(),
                                     "sample": f"{k2} RK2 steps of the event, {threads} OpenMP threads"}
    print(json.dumps(line), flush=True)
    return 0


def batch_record(torch, n_events=256, steps=10, warmup=3, error_steps=EVENT_STEPS):
    """The batched workload in FP64 and in mixed precision against the plain
    single-event FP64 path, and the error of every member over its whole
    event (error_steps RK2 steps) against the FP64 path, next to the FP64
    path's own sensitivity (initial e scaled by 1 + 2^-50)."""
    import numpy as np
    import vh
    cfgs, rows, ics, desc = batch_workload(n_events)
    Ntot = sum(c.nx * c.ny * c.nz for c in cfgs)
    rec = {"workload": desc, "events": n_events, "cells": Ntot, "steps": steps, "warmup": warmup,
           "event_steps": EVENT_STEPS}

    def make(prec, states):
        out = []
        for c, st in zip(cfgs, states):
            e = vh.Event(c.copy(precision=prec), rows)
            e.set_initial(st)
            out.append(e)
        return out

    def close(evs, b):
        b.close()
        for e in evs:
            e.close()

    def timed(prec):
        evs = make(prec, ics)
        b = vh.Batch(evs)
        tune = b.autotune()
        stream = torch.cuda.ExternalStream(b.stream())
        b.step(warmup)
        for e in evs:
            e.sync()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        b.step(steps)
        e1.record(stream)
        e1.synchronize()
        for e in evs:
            vh.check(e.status()[0], "batched steps")
        ms = e0.elapsed_time(e1) / steps
        launches = b.launches_per_step()
        close(evs, b)
        return {"ms_per_step": ms, "cell_updates_per_s": Ntot / (ms / 1e3),
                "events_per_s": n_events / (ms / 1e3 * EVENT_STEPS), "gpu_launches_per_step": launches,
                "tuning": tune.describe()}

    t_mark = [time.perf_counter()]

    def mark(what):
        now = time.perf_counter()
        print(f"[bench] batch record: {what} {now - t_mark[0]:.1f} s", file=sys.stderr, flush=True)
        t_mark[0] = now

    mark("workload")
    rec["fp64"] = timed(vh.VH_PREC_FP64)
    mark("fp64 batch")
    rec["mixed"] = timed(vh.VH_PREC_MIXED)
    mark("mixed batch")
    # the plain single-event FP64 path, one event at a time
    t_solo, s0, s1 = 0.0, torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for c, st in zip(cfgs, ics):
        e = vh.Event(c, rows)
        e.set_initial(st)
        es = torch.cuda.ExternalStream(e.stream())
        e.step(1)
        s0.record(es)
        e.step(steps)
        s1.record(es)
        s1.synchronize()
        t_solo += s0.elapsed_time(s1)
        e.close()
    solo_ms = t_solo / steps
    rec["plain_single_event_fp64"] = {"ms_per_step_all_events": solo_ms, "cell_updates_per_s": Ntot / (solo_ms / 1e3),
                                      "events_per_s": n_events / (solo_ms / 1e3 * EVENT_STEPS),
                                      "how": f"vh_event_step, one event at a time, {steps} steps each after 1, "
                                             "CUDA events per event"}
    mark("plain path")
    rec["fp64_batch_vs_plain"] = solo_ms / rec["fp64"]["ms_per_step"]
    rec["mixed_batch_vs_plain"] = solo_ms / rec["mixed"]["ms_per_step"]

    # every member over its whole event: mixed vs FP64 and FP64 vs itself perturbed
    def run_all(prec, states):
        """error_steps steps; a member whose device flags an error (the
        reference's NaN guard) is no longer computed by the batch"""
        evs = make(prec, states)
        b = vh.Batch(evs)
        b.step(error_steps)
        for e in evs:
            e.status()
        return evs, b

    e_F = vh.eos_eval(cfgs[0], rows, 3, cfgs[0].T_freezeout_GeV / 0.197326938)
    ref_evs, rb = run_all(vh.VH_PREC_FP64, ics)
    mix_evs, mb = run_all(vh.VH_PREC_MIXED, ics)
    bumped = [vh.InitialState(st.e * (1 + 2.0 ** -50), st.p, st.u, st.pi, st.Pi) for st in ics]
    bmp_evs, bb = run_all(vh.VH_PREC_FP64, bumped)
    per = {"mixed_vs_fp64": {"linf": [], "linf_above_eF": []}, "fp64_sensitivity": {"linf": [], "linf_above_eF": []}}
    errored = {"fp64": 0, "mixed": 0, "fp64_perturbed": 0}
    for c, r, m, q in zip(cfgs, ref_evs, mix_evs, bmp_evs):
        st = {"fp64": r.status()[0], "mixed": m.status()[0], "fp64_perturbed": q.status()[0]}
        for k, v in st.items():
            errored[k] += v != 0
        if any(st.values()):
            continue            # a device error (the reference's NaN guard) before the last step
        b = vh.interior(c, r.field(vh.VH_F_E)).ravel()
        hot = b > e_F
        for key, ev in (("mixed_vs_fp64", m), ("fp64_sensitivity", q)):
            d = vh.interior(c, ev.field(vh.VH_F_E)).ravel() - b
            per[key]["linf"].append(float(np.max(np.abs(d)) / np.max(np.abs(b))))
            per[key]["linf_above_eF"].append(float(np.max(np.abs(d[hot])) / np.max(np.abs(b[hot]))) if hot.any()
                                             else 0.0)
    close(ref_evs, rb)
    close(mix_evs, mb)
    close(bmp_evs, bb)
    mark("whole-event errors")
    compared = len(per["mixed_vs_fp64"]["linf"])
    err = {"steps": error_steps, "field": "e", "members_compared": compared,
           "members_with_device_error": errored,
           "note": "members whose run in any of the three modes flagged a device error (the reference's NaN "
                   "guard, EnergyMomentumTensor.cpp:197-203, reached in the dilute edge of lumpy events) "
                   "within the steps are not compared"}
    for key, v in per.items():
        err[key] = {k: {"max": float(np.max(x)), "median": float(np.median(x)),
                        "members_within_1e-4": int(np.sum(np.asarray(x) <= 1e-4))} for k, x in v.items()}
    rec["precision_error"] = err
    return rec


def run_batch(args, torch, world, rank, barrier, max_over_ranks):
    """All events of the batched workload advanced by one vh_batch: one launch
    per RK phase for every event, CUDA-graph replay, autotuned launch shapes."""
    import numpy as np
    import vh
    cfgs, rows, ics, desc = batch_workload(args.events)
    mixed = args.precision == "mixed"
    if mixed:
        cfgs = [c.copy(precision=vh.VH_PREC_MIXED) for c in cfgs]
        desc = desc.replace("FP64", "mixed precision")
    Ns = [c.nx * c.ny * c.nz for c in cfgs]
    Ntot = sum(Ns)
    evs = []
    for c, st in zip(cfgs, ics):
        e = vh.Event(c, rows)
        e.set_initial(st)
        evs.append(e)
    b = vh.Batch(evs)
    tune = b.autotune()
    stream = torch.cuda.ExternalStream(b.stream())
    b.step(args.warmup)
    for e in evs:
        e.sync()
    clocks = ClockSampler(int(os.environ.get("LOCAL_RANK", "0")))
    clocks.start()
    time.sleep(0.3)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    torch.cuda.synchronize()
    e0.record(stream)
    b.step(args.steps)
    e1.record(stream)
    e1.synchronize()
    barrier()
    torch.cuda.synchronize()
    clk = clocks.stop()
    for e in evs:
        vh.check(e.status()[0], "batched steps")
    ms = max_over_ranks(e0.elapsed_time(e1))
    ms_step = ms / args.steps
    value = Ntot * args.steps * world / (ms / 1e3)
    b.phase_timing(True)
    b.step(args.steps)
    phases = b.phase_times()
    b.phase_timing(False)
    kern = {}
    for name, (t, n) in phases.items():
        k = "flux" if name.startswith("flux") else name
        kt, kn = kern.get(k, (0.0, 0))
        kern[k] = (kt + t, kn + n)
    dom = max(kern, key=lambda k: kern[k][0])
    dom_ms, dom_n = kern[dom]
    launch_s = dom_ms / 1e3 / dom_n
    peak, peak_kind = measured_peaks()
    alg_bytes = phase_words(cfgs[0].nq())[dom] * 8 * Ntot
    achieved = alg_bytes / launch_s / 1e9

    prec = None
    if mixed and rank == 0:
        reps = [precision_report(c.copy(precision=vh.VH_PREC_FP64), rows, st, e.progress()[0], e)
                for c, st, e in list(zip(cfgs, ics, evs))[:4]]
        prec = {"members": "the first 4 events of the batch, worst case over them", "steps": reps[0]["steps"]}
        for key in ("mixed_vs_fp64", "fp64_sensitivity"):
            prec[key] = {f: {m: max(r[key][f][m] for r in reps) for m in ("linf", "l2")} for f in reps[0][key]
                         if isinstance(reps[0][key][f], dict)}

    # the plain single-event FP64 path on the same events, one event at a time
    solo_steps = max(1, min(args.steps, 10))
    solo = []
    for c, st in zip(cfgs, ics):
        e = vh.Event(c.copy(precision=vh.VH_PREC_FP64), rows)
        e.set_initial(st)
        solo.append(e)
    t_solo = 0.0
    s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for e in solo:
        es = torch.cuda.ExternalStream(e.stream())
        e.step(1)
        s0.record(es)
        e.step(solo_steps)
        s1.record(es)
        s1.synchronize()
        t_solo += s0.elapsed_time(s1)
    solo_value = Ntot * solo_steps / (t_solo / 1e3)
    for e in solo:
        e.close()

    e2e = None
    if not args.no_e2e:
        pins = []
        for st in ics:
            N = st.e.shape[0]
            pin = torch.empty((17, N), dtype=torch.float64, pin_memory=True)
            h = pin.numpy()
            h[0], h[1], h[2:6], h[6:16], h[16] = st.e, st.p, st.u, 0.0, 0.0 if st.Pi is None else st.Pi
            pins.append((pin, vh.InitialState(h[0], h[1], h[2:6], None, h[16])))
        outs = [torch.empty(int(np.prod(c.padded())), dtype=torch.float64, pin_memory=True).numpy() for c in cfgs]
        torch.cuda.synchronize()
        barrier()
        t0 = time.perf_counter()
        for e, (_, init) in zip(evs, pins):
            e.set_initial(init)
        b.step(args.steps)
        for e, o in zip(evs, outs):
            vh.check(vh.lib.vh_event_get_field(e.h, vh.VH_F_E, o), "vh_event_get_field")
        t1 = time.perf_counter()
        barrier()
        secs = max_over_ranks(t1 - t0)
        h2d = sum((6 * N + (N if c.bulk else 0)) * 8 for c, N in zip(cfgs, Ns))
        d2h = sum(o.nbytes for o in outs)
        e2e = {"value": Ntot * args.steps * world / secs, "unit": "cell-updates/s",
               "h2d_bytes_per_step": h2d / args.steps, "d2h_bytes_per_step": d2h / args.steps,
               "timer": "host wall clock, pinned buffers, IC upload of every event + K batched steps + e download"}

    base = None
    if rank == 0 and world == 1 and not args.no_baseline:
        # the reference on a bounded sample: the first 4 events, 2 steps each
        tot_cells, tot_s = 0, 0.0
        for c, st in list(zip(cfgs, ics))[:4]:
            r = cpu_baseline(c, rows, st, "table", steps=2)
            tot_cells += c.nx * c.ny * c.nz * 2
            tot_s += r["seconds"]
        base = dict(r)
        base["value"] = tot_cells / tot_s
        base["sample"] = ("2 RK2 steps of each of the first 4 events of the batch after 1 warm-up step, "
                          f"{r['cores']} OpenMP threads (reference sources, one event at a time)")

    if rank == 0:
        line = {"metric": "cell-updates/s", "value": value, "unit": "cell-updates/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32/f64 mixed" if mixed else "f64", "data": "synthetic",
                "config": {"workload": desc, "events": len(cfgs), "cells": Ntot, "parallelism": f"replicas x{world}",
                           "l2": "batch state > 126 MB L2, no flush", "tuning": tune.describe()},
                "events_per_s": value / Ntot / EVENT_STEPS * len(cfgs),
                "events_per_s_note": f"events of {EVENT_STEPS} RK2 steps, from the batched step time",
                "plain_single_event": {"value": solo_value, "unit": "cell-updates/s",
                                       "events_per_s": solo_value / Ntot / EVENT_STEPS * len(cfgs),
                                       "speedup_of_batch": value / solo_value,
                                       "how": f"FP64 vh_event_step, one event at a time, {solo_steps} steps each, "
                                              "CUDA events per event"},
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                             "frac": achieved / peak,
                             "traffic": (NCU_TRAFFIC_PER_CELL[(args.precision, dom)] * Ntot
                                         if (args.precision, dom) in NCU_TRAFFIC_PER_CELL else None),
                             "kernel": ("kt_batch_face_kernel " if mixed and dom == "flux" else "kt_batch_kernel ") + dom,
                             "launches": dom_n,
                             "launch_us": launch_s * 1e6, "algorithmic_bytes": alg_bytes,
                             "share": dom_ms / sum(t for t, _ in kern.values()),
                             "note": f"peak: {peak_kind} HBM copy bandwidth; FP64-issue bound"},
                "phases_ms_per_step": {k: t / args.steps for k, (t, _) in phases.items()},
                "clocks": clk, "gpu_launches": b.launches_per_step() * args.steps}
        if prec:
            line["precision_error"] = prec
        if e2e:
            line["e2e"] = e2e
        if base:
            line["cpu_baseline"] = {k: base[k] for k in ("value", "unit", "cores", "kind", "sample")}
        print(json.dumps(line), flush=True)
    b.close()
    for e in evs:
        e.close()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    import numpy as np
    import torch
    import vh
    from replicas import Replicas

    R = Replicas("nccl")
    world, rank, local = R.world, R.rank, R.local
    barrier, max_over_ranks = R.barrier, R.max

    if args.workload == "batch_hotspots_2p1d":
        rc = run_batch(args, torch, world, rank, barrier, max_over_ranks)
        R.close()
        return rc
    if args.workload == "serve_mix":
        rc = run_serve(args, rank)
        R.close()
        return rc
    cfg, rows, st, variant, desc = workload(args.workload)
    mixed = args.precision == "mixed"
    if mixed:
        cfg = cfg.copy(precision=vh.VH_PREC_MIXED)
        desc = desc.replace("FP64", "mixed precision") if "FP64" in desc else desc + ", mixed precision"
    N = cfg.nx * cfg.ny * cfg.nz
    px, py, pz = cfg.padded()
    state_mb = (3 * cfg.nq() + 16) * px * py * pz * 8 / 1e6   # q x3, e/p x2, u x3 planes
    l2_note = (f"state {state_mb:.0f} MB > 126 MB L2, no flush" if state_mb > 126 else
               f"state {state_mb:.0f} MB fits in the 126 MB L2 (not flushed; latency-bound small lattice)")
    ev = vh.Event(cfg, rows)
    ev.set_initial(st)
    stream = torch.cuda.ExternalStream(ev.stream())
    ev.step(args.warmup)
    ev.sync()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    torch.cuda.synchronize()
    e0.record(stream)
    ev.step(args.steps)
    e1.record(stream)
    e1.synchronize()
    rc, _, _ = ev.status()
    barrier()
    torch.cuda.synchronize()
    clk = clocks.stop()
    vh.check(rc, "timed steps")
    ms = max_over_ranks(e0.elapsed_time(e1))
    ms_step = ms / args.steps
    value = N * args.steps * world / (ms / 1e3)
    # the same K steps again with CUDA events recorded between the stage
    # kernels on the event's stream: per-kernel launch durations
    ev.phase_timing(True)
    ev.step(args.steps)
    phases = ev.phase_times()
    ev.phase_timing(False)
    # dominant kernel: group the three flux directions (one kernel template)
    kern = {}
    for name, (t, n) in phases.items():
        k = "flux" if name.startswith("flux") else name
        kt, kn = kern.get(k, (0.0, 0))
        kern[k] = (kt + t, kn + n)
    dom = max(kern, key=lambda k: kern[k][0])
    dom_ms, dom_n = kern[dom]
    launch_s = dom_ms / 1e3 / dom_n
    peak, peak_kind = measured_peaks()
    alg_bytes = phase_words(ev.nq)[dom] * 8 * N
    achieved = alg_bytes / launch_s / 1e9
    traffic = NCU_TRAFFIC.get((args.workload, args.precision, dom))

    # freezeout at the event's cadence (run() calls it every fo_factor steps,
    # HydroPlugin.cpp:249-266): device time of a block -- slab gather, the
    # Cornelius cube scan, compaction, element emission and the count read
    # back -- reported beside the step and combined with it
    fo = None
    if args.fo_blocks > 0:
        fac = max(1, cfg.fo_factor)
        ev.freezeout()                           # the first block compares against a zero slab: untimed
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        fo_ms, fo_el = [], []
        for _ in range(args.fo_blocks):
            ev.step(fac)
            ev.sync()
            f0.record(stream)
            ne, _ = ev.freezeout()
            f1.record(stream)
            f1.synchronize()
            fo_ms.append(f0.elapsed_time(f1))
            fo_el.append(ne)
        ms_fo = max_over_ranks(sum(fo_ms) / len(fo_ms))
        fo = {"ms_per_block": ms_fo, "elements_per_block": sum(fo_el) / len(fo_el), "blocks": len(fo_ms),
              "fo_factor": fac, "cells_scanned_per_s": N * world / (ms_fo / 1e3),
              "combined_cell_updates_per_s": N * fac * world / ((fac * ms_step + ms_fo) / 1e3),
              "timer": "CUDA events around vh_event_freezeout on the event's stream (kernels and the "
                       "element-count read-back); combined = one block per fo_factor steps"}

    e2e = None
    if not args.no_e2e:
        # pinned host buffers; one event = upload IC, K steps, download e
        nq_in = 17
        pin = torch.empty((nq_in, N), dtype=torch.float64, pin_memory=True)
        h = pin.numpy()
        h[0], h[1], h[2:6] = st.e, st.p, st.u
        h[6:16] = 0.0 if st.pi is None else st.pi
        h[16] = 0.0 if st.Pi is None else st.Pi
        outp = torch.empty(ev.cfg.padded()[0] * ev.cfg.padded()[1] * ev.cfg.padded()[2], dtype=torch.float64,
                           pin_memory=True).numpy()
        init = vh.InitialState(h[0], h[1], h[2:6], h[6:16], h[16] if cfg.bulk else None)
        ev.set_initial(init)
        ev.step(1)
        ev.sync()
        barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ev.set_initial(init)
        ev.step(args.steps)
        vh.check(vh.lib.vh_event_get_field(ev.h, vh.VH_F_E, outp), "vh_event_get_field")
        rc, _, _ = ev.status()
        t1 = time.perf_counter()
        barrier()
        vh.check(rc, "e2e steps")
        secs = max_over_ranks(t1 - t0)
        h2d = (6 * N + 10 * N + (N if cfg.bulk else 0)) * 8
        e2e = {"value": N * args.steps * world / secs, "unit": "cell-updates/s",
               "h2d_bytes_per_step": h2d / args.steps, "d2h_bytes_per_step": outp.nbytes / args.steps,
               "timer": "host wall clock, pinned buffers, IC upload + K steps + e download"}

    prec = None
    if mixed and rank == 0:
        psteps = args.precision_steps or PRECISION_STEPS.get(args.workload, args.steps)
        prec = precision_report(cfg, rows, st, psteps)

    base = None
    if rank == 0 and world == 1 and not args.no_baseline:
        base = cpu_baseline(cfg, rows, st, variant)
        if fo is not None:
            fo["reference"] = reference_freezeout(cfg, rows, variant)

    if rank == 0:
        line = {"metric": "cell-updates/s", "value": value, "unit": "cell-updates/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32/f64 mixed" if mixed else "f64", "data": "synthetic",
                "config": {"workload": desc, "cells": N, "parallelism": f"replicas x{world}",
                           "l2": l2_note},
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                             "frac": achieved / peak, "traffic": traffic,
                             "kernel": ("kt_flux_face_kernel (x, y, eta)" if mixed and dom == "flux" and
                                        ev.launches_per_step() > 2 else KERNEL_NAMES[dom]), "launches": dom_n,
                             "launch_us": launch_s * 1e6, "algorithmic_bytes": alg_bytes,
                             "share": dom_ms / sum(t for t, _ in kern.values()),
                             "note": f"peak: {peak_kind} HBM copy bandwidth; the step is bound by "
                                     "FP64/FP32 issue latency (memory and barrier stalls), not HBM"},
                "phases_ms_per_step": {k: t / args.steps for k, (t, _) in phases.items()},
                "clocks": clk, "gpu_launches": ev.launches_per_step() * args.steps}
        fp = NCU_FP64.get((args.workload, args.precision, dom))
        if fp:
            pct, t_ncu_ms, inst = fp
            line["roofline_fp64_pipe"] = {
                "kernel": line["roofline"]["kernel"], "frac": pct / 100.0 * t_ncu_ms / (launch_s * 1e3),
                "fp64_warp_instructions_per_launch": inst,
                "achieved_warp_instructions_per_s": inst / launch_s,
                "how": f"ncu sm__pipe_fp64_cycles_active {pct:.1f} % of peak over the captured launch "
                       f"({t_ncu_ms:.3f} ms under ncu), scaled to the live launch duration"}
        if prec:
            line["precision_error"] = prec
        if fo:
            line["freezeout"] = fo
        if e2e:
            line["e2e"] = e2e
        if base:
            line["cpu_baseline"] = {k: base[k] for k in ("value", "unit", "cores", "kind", "sample")}
    ev.close()
    if rank == 0 and world == 1 and args.workload == "glauber_3p1d" and not mixed and not args.no_extras:
        # the other targets of the benchmark's configurations, each a record
        # of its own: batched events (FP64, mixed) against the plain path; the
        # mixed-precision error of whole events; the event server on a sample
        # of the served mix with every event run to the stop rule
        secs = {}
        t0 = time.perf_counter()
        line["batch"] = batch_record(torch)
        secs["batch"] = time.perf_counter() - t0
        print(f"[bench] batch record {secs['batch']:.1f} s", file=sys.stderr, flush=True)
        t0 = time.perf_counter()
        gc = vh.gubser_config()
        line["precision"] = {
            "gubser_2p1d": precision_report(gc, None, vh.gubser_ic(gc), PRECISION_STEPS["gubser_2p1d"]),
            "glauber_3p1d": precision_report(cfg, rows, st, PRECISION_STEPS["glauber_3p1d"])}
        secs["precision"] = time.perf_counter() - t0
        print(f"[bench] precision record {secs['precision']:.1f} s", file=sys.stderr, flush=True)
        if args.serve_events > 0:
            t0 = time.perf_counter()
            line["serve"] = serve_record(args.serve_events, 30.0, 0, "mixed")
            line["serve"]["note"] = (f"a sample of {args.serve_events} events of the served mix (the "
                                     "configuration names 10,000), arrivals at 30/s (saturating), every event "
                                     "to the stop rule")
            secs["serve"] = time.perf_counter() - t0
        line["extras_seconds"] = secs
    if rank == 0:
        print(json.dumps(line), flush=True)
    R.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
