"""Exact solution of the Riemann problem for one ideal or stiffened gas
(test support).

Written from the standard relations of gas dynamics (e.g. E. F. Toro,
"Riemann Solvers and Numerical Methods for Fluid Dynamics", ch. 4): the star
pressure solves f_L(p) + f_R(p) + u_R - u_L = 0, with f_K the shock
(Rankine-Hugoniot) or rarefaction (isentropic) branch; the solution is then
sampled on x/t.  A stiffened gas (p = (g-1) rho e - g pinf) has the
Rankine-Hugoniot relations and isentropes of an ideal gas in the shifted
pressure p + pinf (the pinf terms of the Hugoniot energy jump cancel), and
sound speed sqrt(g (p + pinf) / rho): its solution is the ideal-gas one in
p + pinf."""
import math


def _f(p, rho, pk, c, g):
    if p > pk:
        a = 2.0 / ((g + 1.0) * rho)
        b = (g - 1.0) / (g + 1.0) * pk
        q = math.sqrt(a / (p + b))
        return (p - pk) * q, q * (1.0 - 0.5 * (p - pk) / (b + p))
    r = p / pk
    return 2.0 * c / (g - 1.0) * (r ** ((g - 1.0) / (2.0 * g)) - 1.0), 1.0 / (rho * c) * r ** (-(g + 1.0) / (2.0 * g))


def star_state(left, right, g, pinf=0.0):
    if pinf:
        ps, us = star_state(_shift(left, pinf), _shift(right, pinf), g)
        return ps - pinf, us
    (rl, ul, pl), (rr, ur, pr) = left, right
    cl, cr = math.sqrt(g * pl / rl), math.sqrt(g * pr / rr)
    p = max(1e-12, 0.5 * (pl + pr))
    for _ in range(100):
        fl, dl = _f(p, rl, pl, cl, g)
        fr, dr = _f(p, rr, pr, cr, g)
        dp = (fl + fr + ur - ul) / (dl + dr)
        pn = max(1e-12, p - dp)
        if abs(pn - p) < 1e-14 * (pn + p):
            p = pn
            break
        p = pn
    fl, _ = _f(p, rl, pl, cl, g)
    fr, _ = _f(p, rr, pr, cr, g)
    return p, 0.5 * (ul + ur) + 0.5 * (fr - fl)


def _shift(state, pinf):
    return state[0], state[1], state[2] + pinf


def sample(left, right, g, xi, pinf=0.0):
    """(rho, u, p) at x/t = xi."""
    if pinf:
        r, u, p = sample(_shift(left, pinf), _shift(right, pinf), g, xi)
        return r, u, p - pinf
    (rl, ul, pl), (rr, ur, pr) = left, right
    cl, cr = math.sqrt(g * pl / rl), math.sqrt(g * pr / rr)
    ps, us = star_state(left, right, g)
    gm = (g - 1.0) / (g + 1.0)
    if xi <= us:
        if ps > pl:   # left shock
            s = ul - cl * math.sqrt((g + 1.0) / (2.0 * g) * ps / pl + (g - 1.0) / (2.0 * g))
            if xi < s:
                return rl, ul, pl
            return rl * (ps / pl + gm) / (gm * ps / pl + 1.0), us, ps
        csl = cl * (ps / pl) ** ((g - 1.0) / (2.0 * g))
        if xi < ul - cl:
            return rl, ul, pl
        if xi > us - csl:
            return rl * (ps / pl) ** (1.0 / g), us, ps
        u = 2.0 / (g + 1.0) * (cl + (g - 1.0) / 2.0 * ul + xi)
        c = 2.0 / (g + 1.0) * (cl + (g - 1.0) / 2.0 * (ul - xi))
        return rl * (c / cl) ** (2.0 / (g - 1.0)), u, pl * (c / cl) ** (2.0 * g / (g - 1.0))
    if ps > pr:       # right shock
        s = ur + cr * math.sqrt((g + 1.0) / (2.0 * g) * ps / pr + (g - 1.0) / (2.0 * g))
        if xi > s:
            return rr, ur, pr
        return rr * (ps / pr + gm) / (gm * ps / pr + 1.0), us, ps
    csr = cr * (ps / pr) ** ((g - 1.0) / (2.0 * g))
    if xi > ur + cr:
        return rr, ur, pr
    if xi < us + csr:
        return rr * (ps / pr) ** (1.0 / g), us, ps
    u = 2.0 / (g + 1.0) * (-cr + (g - 1.0) / 2.0 * ur + xi)
    c = 2.0 / (g + 1.0) * (cr - (g - 1.0) / 2.0 * (ur - xi))
    return rr * (c / cr) ** (2.0 / (g - 1.0)), u, pr * (c / cr) ** (2.0 * g / (g - 1.0))
