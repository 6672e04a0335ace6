"""Exact Riemann solver for the 1D Euler equations of an ideal gas (Toro,
"Riemann Solvers and Numerical Methods for Fluid Dynamics", ch. 4: pressure
function with Newton iteration, then sampling). Test-side known answers."""
import math

import numpy as np


def _f(p, rho, pk, ck, g):
    if p > pk:  # shock
        A = 2.0 / ((g + 1) * rho)
        B = (g - 1) / (g + 1) * pk
        s = math.sqrt(A / (p + B))
        return (p - pk) * s, s * (1 - 0.5 * (p - pk) / (B + p))
    r = p / pk  # rarefaction
    return 2 * ck / (g - 1) * (r ** ((g - 1) / (2 * g)) - 1), 1.0 / (rho * ck) * r ** (-(g + 1) / (2 * g))


def star_state(rl, ul, pl, rr, ur, pr, g):
    cl, cr = math.sqrt(g * pl / rl), math.sqrt(g * pr / rr)
    p = max(1e-12, 0.5 * (pl + pr) - 0.125 * (ur - ul) * (rl + rr) * (cl + cr))
    for _ in range(100):
        fl, dl = _f(p, rl, pl, cl, g)
        fr, dr = _f(p, rr, pr, cr, g)
        pn = max(1e-12, p - (fl + fr + ur - ul) / (dl + dr))
        if abs(pn - p) < 1e-14 * (pn + p):
            p = pn
            break
        p = pn
    fl, _ = _f(p, rl, pl, cl, g)
    fr, _ = _f(p, rr, pr, cr, g)
    return p, 0.5 * (ul + ur) + 0.5 * (fr - fl)


def sample(x, t, x0, rl, ul, pl, rr, ur, pr, g=1.4):
    """(rho, u, p) at positions x and time t for an interface at x0."""
    ps, us = star_state(rl, ul, pl, rr, ur, pr, g)
    cl, cr = math.sqrt(g * pl / rl), math.sqrt(g * pr / rr)
    out = np.zeros((3, len(x)))
    for i, xi in enumerate(np.asarray(x, dtype=float)):
        s = (xi - x0) / t
        if s <= us:  # left of contact
            if ps > pl:
                sl = ul - cl * math.sqrt((g + 1) / (2 * g) * ps / pl + (g - 1) / (2 * g))
                if s <= sl:
                    out[:, i] = (rl, ul, pl)
                else:
                    r = rl * ((ps / pl + (g - 1) / (g + 1)) / ((g - 1) / (g + 1) * ps / pl + 1))
                    out[:, i] = (r, us, ps)
            else:
                shl = ul - cl
                csl = cl * (ps / pl) ** ((g - 1) / (2 * g))
                stl = us - csl
                if s <= shl:
                    out[:, i] = (rl, ul, pl)
                elif s >= stl:
                    out[:, i] = (rl * (ps / pl) ** (1 / g), us, ps)
                else:
                    u = 2 / (g + 1) * (cl + (g - 1) / 2 * ul + s)
                    c = 2 / (g + 1) * (cl + (g - 1) / 2 * (ul - s))
                    r = rl * (c / cl) ** (2 / (g - 1))
                    out[:, i] = (r, u, pl * (c / cl) ** (2 * g / (g - 1)))
        else:
            if ps > pr:
                sr = ur + cr * math.sqrt((g + 1) / (2 * g) * ps / pr + (g - 1) / (2 * g))
                if s >= sr:
                    out[:, i] = (rr, ur, pr)
                else:
                    r = rr * ((ps / pr + (g - 1) / (g + 1)) / ((g - 1) / (g + 1) * ps / pr + 1))
                    out[:, i] = (r, us, ps)
            else:
                shr = ur + cr
                csr = cr * (ps / pr) ** ((g - 1) / (2 * g))
                str_ = us + csr
                if s >= shr:
                    out[:, i] = (rr, ur, pr)
                elif s <= str_:
                    out[:, i] = (rr * (ps / pr) ** (1 / g), us, ps)
                else:
                    u = 2 / (g + 1) * (-cr + (g - 1) / 2 * ur + s)
                    c = 2 / (g + 1) * (cr - (g - 1) / 2 * (ur - s))
                    r = rr * (c / cr) ** (2 / (g - 1))
                    out[:, i] = (r, u, pr * (c / cr) ** (2 * g / (g - 1)))
    return out
