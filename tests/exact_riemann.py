"""Exact solution of the 1-D Riemann problem of the Euler equations for an
ideal gas (Toro, "Riemann Solvers and Numerical Methods for Fluid
Dynamics", ch. 4: pressure function, Newton iteration for p*, sampling).
Used to pin the CPU oracle's solvers on the Sod problem."""
from __future__ import annotations

import numpy as np


def _fk(p, rk, pk, ck, g):
    if p > pk:  # shock
        A = 2.0 / ((g + 1) * rk)
        B = (g - 1) / (g + 1) * pk
        q = np.sqrt(A / (p + B))
        return (p - pk) * q, q * (1 - 0.5 * (p - pk) / (B + p))
    pr = p / pk  # rarefaction
    f = 2 * ck / (g - 1) * (pr ** ((g - 1) / (2 * g)) - 1)
    return f, 1.0 / (rk * ck) * pr ** (-(g + 1) / (2 * g))


def star_state(rl, ul, pl, rr, ur, pr, g):
    cl, cr = np.sqrt(g * pl / rl), np.sqrt(g * pr / rr)
    p = max(1e-12, 0.5 * (pl + pr))
    for _ in range(200):
        fl, dl = _fk(p, rl, pl, cl, g)
        fr, dr = _fk(p, rr, pr, cr, g)
        dp = (fl + fr + ur - ul) / (dl + dr)
        pn = max(1e-12, p - dp)
        if abs(pn - p) < 1e-14 * 0.5 * (pn + p):
            p = pn
            break
        p = pn
    fl, _ = _fk(p, rl, pl, cl, g)
    fr, _ = _fk(p, rr, pr, cr, g)
    return p, 0.5 * (ul + ur) + 0.5 * (fr - fl)


def sample(x, t, x0, rl, ul, pl, rr, ur, pr, g):
    """Density, velocity, pressure at positions x and time t."""
    ps, us = star_state(rl, ul, pl, rr, ur, pr, g)
    cl, cr = np.sqrt(g * pl / rl), np.sqrt(g * pr / rr)
    out = np.zeros((3, len(x)))
    for n, xx in enumerate(x):
        s = (xx - x0) / t
        if s <= us:  # left of contact
            if ps > pl:
                sl = ul - cl * np.sqrt((g + 1) / (2 * g) * ps / pl + (g - 1) / (2 * g))
                if s <= sl:
                    out[:, n] = rl, ul, pl
                else:
                    r = rl * (ps / pl + (g - 1) / (g + 1)) / ((g - 1) / (g + 1) * ps / pl + 1)
                    out[:, n] = r, us, ps
            else:
                shl = ul - cl
                csl = cl * (ps / pl) ** ((g - 1) / (2 * g))
                stl = us - csl
                if s <= shl:
                    out[:, n] = rl, ul, pl
                elif s >= stl:
                    out[:, n] = rl * (ps / pl) ** (1 / g), us, ps
                else:
                    c = 2 / (g + 1) * (cl + (g - 1) / 2 * (ul - s))
                    u = 2 / (g + 1) * (cl + (g - 1) / 2 * ul + s)
                    r = rl * (c / cl) ** (2 / (g - 1))
                    out[:, n] = r, u, pl * (c / cl) ** (2 * g / (g - 1))
        else:
            if ps > pr:
                sr = ur + cr * np.sqrt((g + 1) / (2 * g) * ps / pr + (g - 1) / (2 * g))
                if s >= sr:
                    out[:, n] = rr, ur, pr
                else:
                    r = rr * (ps / pr + (g - 1) / (g + 1)) / ((g - 1) / (g + 1) * ps / pr + 1)
                    out[:, n] = r, us, ps
            else:
                shr = ur + cr
                csr = cr * (ps / pr) ** ((g - 1) / (2 * g))
                str_ = us + csr
                if s >= shr:
                    out[:, n] = rr, ur, pr
                elif s <= str_:
                    out[:, n] = rr * (ps / pr) ** (1 / g), us, ps
                else:
                    c = 2 / (g + 1) * (cr - (g - 1) / 2 * (ur - s))
                    u = 2 / (g + 1) * (-cr + (g - 1) / 2 * ur + s)
                    r = rr * (c / cr) ** (2 / (g - 1))
                    out[:, n] = r, u, pr * (c / cr) ** (2 * g / (g - 1))
    return out
