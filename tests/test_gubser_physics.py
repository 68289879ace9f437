"""The semi-analytic viscous Gubser solution (the reference's own physics
check, mathematica/gubserFlowTest.nb) against the evolution started from it.

Agreement is limited by the KT discretisation and by the second-order terms
the code carries beyond the ODE, so it is checked at the percent level near
the centre and shown to improve when the lattice is refined."""
import numpy as np
import pytest

import vh
import gubser
from oracle import OracleEvent

T0 = 0.3 / 0.197326938      # T(tau = 1/q, r = 0) of the Gubser event [fm^-1]


def _errors(cfg, sol, ev, steps):
    tau = cfg.t0 + steps * cfg.dt
    X, Y = gubser.lattice_xy(cfg)
    R = np.hypot(X, Y)
    e = vh.interior(cfg, ev.field(vh.VH_F_E)).ravel()
    ux = vh.interior(cfg, ev.field(vh.VH_F_UT + 1)).ravel()
    pinn = vh.interior(cfg, ev.field(13)).ravel()
    ea, ua, pa = gubser.milne_fields(sol, tau, X, Y, 1.0, cfg.eos_factor)
    out = {}
    for rmax in (1.0, 2.0):
        m = R <= rmax
        out[rmax] = {"T": float(np.max(np.abs((e[m] / ea[m]) ** 0.25 - 1))),
                     "ux": float(np.max(np.abs(ux[m] - ua[1][m]))),
                     "pinn": float(np.max(np.abs(pinn[m] - pa[9][m])) / np.max(np.abs(pa[9][m])))}
    return out


def _grid(n, dx):
    cfg = vh.gubser_config(n, n)
    cfg.dx = cfg.dy = cfg.dz = dx
    cfg.dt = dx / 10
    return cfg


def test_semianalytic_solution_is_consistent():
    """the rho-space solution reproduces the ideal Gubser temperature for
    small eta/s (forward in rho: backward, the relaxation equation amplifies
    errors like exp(int T / (5 eta/s)), harmless at eta/s = 0.2 only) and
    starts at T0 with pi = 0 at rho = 0"""
    sol = gubser.Solution(T0, 1e-3, rho_max=3.0, rho_min=0.0)
    rho = np.linspace(0.0, 2.5, 11)
    T, _ = sol.at(rho)
    assert np.allclose(T, T0 * np.cosh(rho) ** (-2.0 / 3.0), rtol=2e-3)
    sol = gubser.Solution(T0, 0.2)
    assert sol.at(0.0)[0] == pytest.approx(T0) and sol.at(0.0)[1] == 0.0


def test_oracle_follows_gubser():
    """the reference's algorithm (its C restatement) on the Gubser grid, 50 steps"""
    cfg = _grid(101, 0.1)
    sol = gubser.Solution(T0, cfg.etabar)
    o = OracleEvent(cfg)
    o.set_initial(gubser.initial_state(cfg, sol))
    assert o.step(50) == 0
    err = _errors(cfg, sol, o, 50)
    assert err[1.0]["T"] < 1e-2 and err[1.0]["ux"] < 2e-2, err
    assert err[2.0]["T"] < 4e-2, err


@pytest.mark.gpu
def test_device_follows_gubser_and_converges():
    sol = gubser.Solution(T0, 0.2)
    res = {}
    for n, dx in ((101, 0.1), (201, 0.05)):
        cfg = _grid(n, dx)
        ev = vh.Event(cfg)
        ev.set_initial(gubser.initial_state(cfg, sol))
        steps = int(round(1.0 / cfg.dt))            # to tau = 2
        ev.step(steps)
        ev.sync()
        res[n] = _errors(cfg, sol, ev, steps)
    coarse, fine = res[101], res[201]
    assert coarse[1.0]["T"] < 1e-2 and coarse[1.0]["ux"] < 2e-2 and coarse[1.0]["pinn"] < 0.15, res
    assert coarse[2.0]["T"] < 5e-2, res
    # halving the spacing reduces the central deviation (to tau = 2 the
    # remainder is mostly the code's second-order terms beyond the ODE)
    assert fine[1.0]["T"] < 0.8 * coarse[1.0]["T"], res
    assert fine[1.0]["ux"] < coarse[1.0]["ux"] and fine[1.0]["pinn"] < coarse[1.0]["pinn"], res
