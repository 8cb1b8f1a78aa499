"""Analytic reference solutions and profile metrics used by the validation
cases (the same quantities test/references.jl and test/cases.jl measure):
the exact Riemann solution of the Euler equations (Toro, "Riemann Solvers
and Numerical Methods for Fluid Dynamics", ch. 4: Newton iteration on the
pressure function, then sampling of the self-similar fan), Noh's implosion,
front positions and L1 means."""
import math

import numpy as np


def riemann_star(rl, ul, pl, rr, ur, pr, g):
    """Star-region pressure and velocity (Toro ch. 4.2-4.3)."""
    cl = math.sqrt(g * pl / rl)
    cr = math.sqrt(g * pr / rr)

    def fk(p, rk, pk, ck):
        if p > pk:  # shock branch
            A = 2.0 / ((g + 1) * rk)
            B = (g - 1) / (g + 1) * pk
            s = math.sqrt(A / (p + B))
            return (p - pk) * s, s * (1 - (p - pk) / (2 * (p + B)))
        # rarefaction branch
        e = (g - 1) / (2 * g)
        return 2 * ck / (g - 1) * ((p / pk) ** e - 1), (p / pk) ** (-(g + 1) / (2 * g)) / (rk * ck)

    p = max(0.5 * (pl + pr), 1e-8)
    for _ in range(200):
        f1, d1 = fk(p, rl, pl, cl)
        f2, d2 = fk(p, rr, pr, cr)
        F = f1 + f2 + (ur - ul)
        dp = F / (d1 + d2)
        pn = max(p - dp, 1e-12)
        if abs(pn - p) <= 1e-14 * 0.5 * (pn + p):
            p = pn
            break
        p = pn
    f1, _ = fk(p, rl, pl, cl)
    f2, _ = fk(p, rr, pr, cr)
    u = 0.5 * (ul + ur) + 0.5 * (f2 - f1)
    return p, u, cl, cr


def riemann_sample(S, rl, ul, pl, rr, ur, pr, g, ps, us, cl, cr):
    """Solution at similarity coordinate S = (x - x0)/t (Toro ch. 4.5)."""
    g1 = (g - 1) / (2 * g)
    g6 = (g - 1) / (g + 1)
    if S <= us:
        if ps > pl:
            sl = ul - cl * math.sqrt((g + 1) / (2 * g) * ps / pl + g1)
            if S <= sl:
                return rl, ul, pl
            return rl * ((ps / pl + g6) / (g6 * ps / pl + 1)), us, ps
        shl = ul - cl
        stl = us - cl * (ps / pl) ** g1
        if S <= shl:
            return rl, ul, pl
        if S >= stl:
            return rl * (ps / pl) ** (1 / g), us, ps
        u = 2 / (g + 1) * (cl + (g - 1) / 2 * ul + S)
        c = 2 / (g + 1) * (cl + (g - 1) / 2 * (ul - S))
        r = rl * (c / cl) ** (2 / (g - 1))
        return r, u, pl * (c / cl) ** (2 * g / (g - 1))
    if ps > pr:
        sr = ur + cr * math.sqrt((g + 1) / (2 * g) * ps / pr + g1)
        if S >= sr:
            return rr, ur, pr
        return rr * ((ps / pr + g6) / (g6 * ps / pr + 1)), us, ps
    shr = ur + cr
    str_ = us + cr * (ps / pr) ** g1
    if S >= shr:
        return rr, ur, pr
    if S <= str_:
        return rr * (ps / pr) ** (1 / g), us, ps
    u = 2 / (g + 1) * (-cr + (g - 1) / 2 * ur + S)
    c = 2 / (g + 1) * (cr - (g - 1) / 2 * (ur - S))
    r = rr * (c / cr) ** (2 / (g - 1))
    return r, u, pr * (c / cr) ** (2 * g / (g - 1))


def riemann_profile(xs, t, x0, left, right, g):
    ps, us, cl, cr = riemann_star(*left, *right, g)
    out = np.array([riemann_sample((x - x0) / t, *left, *right, g, ps, us, cl, cr) for x in xs])
    return out[:, 0], out[:, 1], out[:, 2]


def noh_exact(r, t, nu, g, rho0=1.0):
    S = (g - 1) / 2
    if r <= S * t:
        rho = rho0 * ((g + 1) / (g - 1)) ** nu
        return rho, 0.0, (g - 1) * rho * 0.5
    return rho0 * (1 + t / r) ** (nu - 1), -1.0, 0.0


def front_position(xs, f, level):
    """Outermost crossing of `level`, scanning from the high end."""
    for i in range(len(f) - 1, 0, -1):
        lo, hi = f[i - 1], f[i]
        if (lo - level) * (hi - level) <= 0 and lo != hi:
            return xs[i - 1] + (xs[i] - xs[i - 1]) * (level - lo) / (hi - lo)
    return float("nan")


def l1(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.sum(np.abs(a - b)) / len(a))


def interp1(xs, ys, xq):
    xs = np.asarray(xs)
    ys = np.asarray(ys)
    return np.interp(xq, xs, ys)


def read_profile(path):
    """Read a stored (x, rho, u, p) CSV profile ('#' comment lines)."""
    rows = [list(map(float, ln.split(","))) for ln in open(path) if ln.strip() and not ln.startswith("#")]
    a = np.array(rows)
    return a[:, 0], a[:, 1], a[:, 2], a[:, 3]
