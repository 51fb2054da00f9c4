"""Exact solution of the 1D Riemann problem for an ideal gas (test
infrastructure): the star-region pressure by Newton iteration on the
pressure function, then the self-similar solution sampled at x/t
(Toro, Riemann Solvers and Numerical Methods for Fluid Dynamics, ch. 4)."""
import math

import numpy as np


def _f(p, rho, pk, ck, g):
    """pressure function of one side and its derivative"""
    if p > pk:   # shock
        A, B = 2.0 / ((g + 1.0) * rho), (g - 1.0) / (g + 1.0) * pk
        s = math.sqrt(A / (p + B))
        return (p - pk) * s, s * (1.0 - 0.5 * (p - pk) / (B + p))
    r = p / pk   # rarefaction
    return 2.0 * ck / (g - 1.0) * (r ** ((g - 1.0) / (2.0 * g)) - 1.0), 1.0 / (rho * ck) * r ** (-(g + 1.0) / (2.0 * g))


def star(rl, ul, pl, rr, ur, pr, g):
    cl, cr = math.sqrt(g * pl / rl), math.sqrt(g * pr / rr)
    p = max(1e-12, 0.5 * (pl + pr))
    for _ in range(100):
        fl, dl = _f(p, rl, pl, cl, g)
        fr, dr = _f(p, rr, pr, cr, g)
        dp = (fl + fr + ur - ul) / (dl + dr)
        p = max(1e-12, p - dp)
        if abs(dp) < 1e-14 * p:
            break
    fl, _ = _f(p, rl, pl, cl, g)
    fr, _ = _f(p, rr, pr, cr, g)
    return p, 0.5 * (ul + ur) + 0.5 * (fr - fl)


def sample(rl, ul, pl, rr, ur, pr, g, xi):
    """density, velocity, pressure at the similarity coordinates xi = (x - x0) / t"""
    ps, us = star(rl, ul, pl, rr, ur, pr, g)
    cl, cr = math.sqrt(g * pl / rl), math.sqrt(g * pr / rr)
    out = np.zeros((3, len(xi)))
    for n, s in enumerate(xi):
        if s <= us:   # left of the contact
            if ps > pl:   # left shock
                sl = ul - cl * math.sqrt((g + 1) / (2 * g) * ps / pl + (g - 1) / (2 * g))
                if s <= sl:
                    w = (rl, ul, pl)
                else:
                    w = (rl * ((ps / pl + (g - 1) / (g + 1)) / ((g - 1) / (g + 1) * ps / pl + 1)), us, ps)
            else:         # left rarefaction
                shl, csl = ul - cl, cl * (ps / pl) ** ((g - 1) / (2 * g))
                stl = us - csl
                if s <= shl:
                    w = (rl, ul, pl)
                elif s >= stl:
                    w = (rl * (ps / pl) ** (1 / g), us, ps)
                else:
                    c = 2 / (g + 1) * (cl + (g - 1) / 2 * (ul - s))
                    u = 2 / (g + 1) * (cl + (g - 1) / 2 * ul + s)
                    w = (rl * (c / cl) ** (2 / (g - 1)), u, pl * (c / cl) ** (2 * g / (g - 1)))
        else:             # right of the contact
            if ps > pr:   # right shock
                sr = ur + cr * math.sqrt((g + 1) / (2 * g) * ps / pr + (g - 1) / (2 * g))
                if s >= sr:
                    w = (rr, ur, pr)
                else:
                    w = (rr * ((ps / pr + (g - 1) / (g + 1)) / ((g - 1) / (g + 1) * ps / pr + 1)), us, ps)
            else:         # right rarefaction
                shr, csr = ur + cr, cr * (ps / pr) ** ((g - 1) / (2 * g))
                str_ = us + csr
                if s >= shr:
                    w = (rr, ur, pr)
                elif s <= str_:
                    w = (rr * (ps / pr) ** (1 / g), us, ps)
                else:
                    c = 2 / (g + 1) * (cr - (g - 1) / 2 * (ur - s))
                    u = 2 / (g + 1) * (-cr + (g - 1) / 2 * ur + s)
                    w = (rr * (c / cr) ** (2 / (g - 1)), u, pr * (c / cr) ** (2 * g / (g - 1)))
        out[:, n] = w
    return out
