"""Exact solution of the Riemann problem of the 1D Euler equations for an
ideal gas -- test infrastructure (the exact answer for the Sod configuration).

The reference claims agreement with the exact solution for its Sod run
(README.md:30-37) but ships no solver (pypkg/plot_sod.py only overlays
frames).  This restates the published method of E. F. Toro, "Riemann
Solvers and Numerical Methods for Fluid Dynamics", 3rd ed., Springer 2009,
chapter 4: the pressure functions f_K (eqs. 4.6-4.8), the Newton iteration
for the star pressure started from the primitive-variable guess (4.46), the
star velocity (4.9) and the sampling of the self-similar solution at
S = (x - x0)/t (section 4.5).  The reference's HLLC (hllc.cpp:13-19) cites the
same book.
"""
from __future__ import annotations

from typing import Tuple

import numpy as np


def _f_and_df(p, rho_k, p_k, c_k, g):
    """Toro's f_K(p) and its derivative: shock branch for p > p_K (4.6, 4.37),
    rarefaction branch otherwise (4.7, 4.37)."""
    if p > p_k:
        a = 2.0 / ((g + 1.0) * rho_k)
        b = (g - 1.0) / (g + 1.0) * p_k
        q = np.sqrt(a / (p + b))
        return (p - p_k) * q, q * (1.0 - 0.5 * (p - p_k) / (b + p))
    r = (p / p_k) ** ((g - 1.0) / (2.0 * g))
    return 2.0 * c_k / (g - 1.0) * (r - 1.0), 1.0 / (rho_k * c_k) * (p / p_k) ** (-(g + 1.0) / (2.0 * g))


def star_state(left: Tuple[float, float, float], right: Tuple[float, float, float],
               gamma: float = 1.4, tol: float = 1e-14) -> Tuple[float, float]:
    """(p*, u*) of the Riemann problem with primitive states (rho, u, p)."""
    rl, ul, pl = left
    rr, ur, pr = right
    g = gamma
    cl, cr = np.sqrt(g * pl / rl), np.sqrt(g * pr / rr)
    if 2.0 * (cl + cr) / (g - 1.0) <= ur - ul:
        raise ValueError("the data generate a vacuum")
    # primitive-variable guess (4.46), kept positive
    p = max(tol, 0.5 * (pl + pr) - 0.125 * (ur - ul) * (rl + rr) * (cl + cr))
    for _ in range(100):
        fl, dfl = _f_and_df(p, rl, pl, cl, g)
        fr, dfr = _f_and_df(p, rr, pr, cr, g)
        p_new = max(tol, p - (fl + fr + ur - ul) / (dfl + dfr))
        change = 2.0 * abs(p_new - p) / (p_new + p)
        p = p_new
        if change < tol:
            break
    fl, _ = _f_and_df(p, rl, pl, cl, g)
    fr, _ = _f_and_df(p, rr, pr, cr, g)
    return p, 0.5 * (ul + ur) + 0.5 * (fr - fl)


def star_densities(left, right, gamma: float = 1.4) -> Tuple[float, float]:
    """rho*L, rho*R: the shock (4.50, 4.57) or isentropic (4.53, 4.60) relations."""
    p, _ = star_state(left, right, gamma)
    g = gamma
    gg = (g - 1.0) / (g + 1.0)
    out = []
    for rho_k, p_k in ((left[0], left[2]), (right[0], right[2])):
        if p > p_k:
            out.append(rho_k * (p / p_k + gg) / (gg * p / p_k + 1.0))
        else:
            out.append(rho_k * (p / p_k) ** (1.0 / g))
    return out[0], out[1]


def sample(x: np.ndarray, t: float, x0: float, left, right,
           gamma: float = 1.4) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
    """rho, u, p of the exact solution at positions x and time t > 0, the
    discontinuity initially at x0 (Toro section 4.5, figure 4.14)."""
    rl, ul, pl = left
    rr, ur, pr = right
    g = gamma
    ps, us = star_state(left, right, gamma)
    cl, cr = np.sqrt(g * pl / rl), np.sqrt(g * pr / rr)
    gg = (g - 1.0) / (g + 1.0)
    s = (np.asarray(x, dtype=np.float64) - x0) / t
    rho, u, p = np.empty_like(s), np.empty_like(s), np.empty_like(s)
    for n, si in enumerate(s):
        if si <= us:  # left of the contact
            if ps > pl:  # left shock (4.52)
                sl = ul - cl * np.sqrt((g + 1.0) / (2.0 * g) * ps / pl + (g - 1.0) / (2.0 * g))
                if si <= sl:
                    rho[n], u[n], p[n] = rl, ul, pl
                else:
                    rho[n], u[n], p[n] = rl * (ps / pl + gg) / (gg * ps / pl + 1.0), us, ps
            else:  # left rarefaction (4.54-4.56)
                shl = ul - cl
                csl = cl * (ps / pl) ** ((g - 1.0) / (2.0 * g))
                stl = us - csl
                if si <= shl:
                    rho[n], u[n], p[n] = rl, ul, pl
                elif si > stl:
                    rho[n], u[n], p[n] = rl * (ps / pl) ** (1.0 / g), us, ps
                else:
                    c = 2.0 / (g + 1.0) * (cl + 0.5 * (g - 1.0) * (ul - si))
                    u[n] = 2.0 / (g + 1.0) * (cl + 0.5 * (g - 1.0) * ul + si)
                    rho[n] = rl * (c / cl) ** (2.0 / (g - 1.0))
                    p[n] = pl * (c / cl) ** (2.0 * g / (g - 1.0))
        else:  # right of the contact
            if ps > pr:  # right shock (4.59)
                sr = ur + cr * np.sqrt((g + 1.0) / (2.0 * g) * ps / pr + (g - 1.0) / (2.0 * g))
                if si >= sr:
                    rho[n], u[n], p[n] = rr, ur, pr
                else:
                    rho[n], u[n], p[n] = rr * (ps / pr + gg) / (gg * ps / pr + 1.0), us, ps
            else:  # right rarefaction (4.61-4.63)
                shr = ur + cr
                csr = cr * (ps / pr) ** ((g - 1.0) / (2.0 * g))
                str_ = us + csr
                if si >= shr:
                    rho[n], u[n], p[n] = rr, ur, pr
                elif si < str_:
                    rho[n], u[n], p[n] = rr * (ps / pr) ** (1.0 / g), us, ps
                else:
                    c = 2.0 / (g + 1.0) * (cr - 0.5 * (g - 1.0) * (ur - si))
                    u[n] = 2.0 / (g + 1.0) * (-cr + 0.5 * (g - 1.0) * ur + si)
                    rho[n] = rr * (c / cr) ** (2.0 / (g - 1.0))
                    p[n] = pr * (c / cr) ** (2.0 * g / (g - 1.0))
    return rho, u, p


def cell_average(xl: np.ndarray, xr: np.ndarray, t: float, x0: float, left, right,
                 gamma: float = 1.4, sub: int = 64) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
    """Cell averages of rho, rho u and E of the exact solution over [xl, xr],
    by the midpoint rule on `sub` points per cell (the discontinuities make
    point values at cell centres a poor stand-in for cell averages)."""
    n = len(xl)
    f = (np.arange(sub) + 0.5) / sub
    xs = (xl[:, None] + (xr - xl)[:, None] * f[None, :]).ravel()
    rho, u, p = sample(xs, t, x0, left, right, gamma)
    e = p / (gamma - 1.0) + 0.5 * rho * u * u
    return tuple(v.reshape(n, sub).mean(axis=1) for v in (rho, rho * u, e))
