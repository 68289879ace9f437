"""Semi-analytic viscous Gubser flow, the reference's physics check for the
2+1D conformal evolution (mathematica/gubserFlowTest.nb).

In de Sitter time rho, with sinh(rho) = -(1 - q^2 tau^2 + q^2 r^2) / (2 q tau),
the notebook integrates (from rho = 0, T(0) given, pi(0) = 0)

    T'(rho)  = -(2/3) T tanh(rho) - (1/3) T pi tanh(rho)
    pi'(rho) = -T pi / (5 eta/s) + (4/3) pi^2 tanh(rho) - (4/15) tanh(rho)

and maps back to Milne coordinates with T(tau, r) = T(rho) / tau (q = 1/fm:
T in fm^-1 when tau is in fm) and the Gubser velocity.  pi here is minus the
de Sitter shear component pi^eta_eta / (e + P); in the fluid's local rest
frame the Milne shear tensor has the eigenvalue P = -(4/3) e pi along eta and
-P/2 along the two transverse directions (the azimuth and the rest-frame
radial direction), which gives every component below.

Everything here is host-side validation tooling for the tests.
"""
from __future__ import annotations

import numpy as np

import vh


def _rhs(rho, T, p, etas):
    th = np.tanh(rho)
    return (-(2.0 / 3.0) * T * th - (1.0 / 3.0) * T * p * th,
            -T * p / (5.0 * etas) + (4.0 / 3.0) * p * p * th - (4.0 / 15.0) * th)


class Solution:
    """T(rho), pi(rho) on a uniform rho grid by classical RK4 from rho = 0,
    forward to rho_max and backward to rho_min (default -rho_max)."""

    def __init__(self, T0: float, etas: float, rho_max: float = 10.0, h: float = 1e-3, rho_min: float | None = None):
        n_hi = int(round(rho_max / h))
        n_lo = int(round(-(-rho_max if rho_min is None else rho_min) / h))
        self.rho = np.arange(-n_lo, n_hi + 1) * h
        T = np.empty(n_lo + n_hi + 1)
        P = np.empty(n_lo + n_hi + 1)
        T[n_lo], P[n_lo] = T0, 0.0
        for sgn, n in ((1, n_hi), (-1, n_lo)):
            t, p = T0, 0.0
            for k in range(n):
                r = sgn * k * h
                hh = sgn * h
                k1 = _rhs(r, t, p, etas)
                k2 = _rhs(r + hh / 2, t + hh / 2 * k1[0], p + hh / 2 * k1[1], etas)
                k3 = _rhs(r + hh / 2, t + hh / 2 * k2[0], p + hh / 2 * k2[1], etas)
                k4 = _rhs(r + hh, t + hh * k3[0], p + hh * k3[1], etas)
                t += hh / 6 * (k1[0] + 2 * k2[0] + 2 * k3[0] + k4[0])
                p += hh / 6 * (k1[1] + 2 * k2[1] + 2 * k3[1] + k4[1])
                T[n_lo + sgn * (k + 1)], P[n_lo + sgn * (k + 1)] = t, p
        self.T, self.pi = T, P

    def at(self, rho):
        return np.interp(rho, self.rho, self.T), np.interp(rho, self.rho, self.pi)


def milne_fields(sol: Solution, tau: float, x, y, q: float, a: float):
    """e, u (ut, ux, uy) and pi (tt, tx, ty, tn, xx, xy, xn, yy, yn, nn) at (tau, x, y)."""
    x = np.asarray(x, dtype=np.float64)
    y = np.asarray(y, dtype=np.float64)
    r = np.hypot(x, y)
    rho = np.arcsinh(-(1 - q * q * tau * tau + q * q * r * r) / (2 * q * tau))
    That, pib = sol.at(rho)
    T = That / tau
    e = a * T ** 4
    vr = 2 * q * q * tau * r / (1 + q * q * tau * tau + q * q * r * r)
    ut = 1 / np.sqrt(1 - vr * vr)
    ur = ut * vr
    c = np.where(r > 0, x / np.where(r > 0, r, 1), 1.0)
    s = np.where(r > 0, y / np.where(r > 0, r, 1), 0.0)
    ux, uy = ur * c, ur * s
    P = -(4.0 / 3.0) * e * pib          # rest-frame eigenvalue along eta
    h = -P / 2                          # along azimuth and rest-frame radius
    pi = np.zeros((10,) + np.shape(x))
    pi[0] = h * ur * ur                 # tt
    pi[1] = h * ur * ut * c             # tx
    pi[2] = h * ur * ut * s             # ty
    pi[4] = h * (ut * ut * c * c + s * s)          # xx
    pi[5] = h * (ut * ut - 1) * c * s               # xy
    pi[7] = h * (ut * ut * s * s + c * c)          # yy
    pi[9] = P / (tau * tau)                         # nn
    return e, np.stack([ut, ux, uy]), pi


def lattice_xy(cfg):
    """Cell centres of the interior lattice, the layout vh_ic_gubser uses."""
    xs = (np.arange(cfg.nx) - (cfg.nx - 1) / 2.0) * cfg.dx
    ys = (np.arange(cfg.ny) - (cfg.ny - 1) / 2.0) * cfg.dy
    X, Y = np.meshgrid(xs, ys)          # (ny, nx): index i + nx * j
    return X.ravel(), Y.ravel()


def initial_state(cfg, sol: Solution, q: float = 1.0) -> vh.InitialState:
    """The semi-analytic solution at tau = cfg.t0 as an initial condition."""
    X, Y = lattice_xy(cfg)
    e, u3, pi = milne_fields(sol, cfg.t0, X, Y, q, cfg.eos_factor)
    N = X.size
    u = np.zeros((4, N))
    u[:3] = u3
    return vh.InitialState(e, e / 3.0, u, pi, None)
