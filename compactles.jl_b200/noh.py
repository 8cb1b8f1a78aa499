"""The Noh implosion in three geometries (test/cases.jl:186-236,
test/references.jl:100-114, test/validation.jl:217-233).

Cold gas at u = -1 stagnates on a symmetry point: planar (slip wall at
x = 0), cylindrical (AxisBC fold, theta collapsed) and spherical (OriginBC
fold, theta and phi collapsed, warm-started from the exact solution at
t0 = 0.3).  The outer face carries the exact inflow as a DirichletBC(fun)
evaluated at the stage times, which for nu > 1 compresses as it converges.
Every feature of the answer is a fixed number: the post-shock plateau 4^nu,
the shock radius (gamma - 1)/2 t, the pre-shock density (1 + t/r)^(nu-1).

`noh_case(cl, nu, schemes, make_solver)` builds and runs one case with the
given solver class (device or oracle); `noh_metrics` measures it as the
reference's validation battery does.
"""
import math

import numpy as np

NOH_G = 5 / 3
NOH_T = 0.6
NOH_P0 = 1e-4
NOH_CFL = 0.15
NOH_N = {1: 400, 2: 256, 3: 256}
NOH_T0 = {1: 0.0, 2: 0.0, 3: 0.3}
NMAX = 2_000_000
# validation tolerances on the plateau (test/validation.jl:219)
NOH_PTOL = {1: 0.01, 2: 0.10, 3: 0.15}


def noh_exact(r, t, nu, g, rho0=1.0):
    """noh_exact(r, t, nu, gamma) -> (rho, u, p), vectorised over r."""
    r = np.asarray(r, dtype=np.float64)
    S = (g - 1) / 2
    shocked = r <= S * t
    with np.errstate(divide="ignore", invalid="ignore"):
        free = rho0 * (1 + t / r) ** (nu - 1)
    rho = np.where(shocked, rho0 * ((g + 1) / (g - 1)) ** nu, free)
    u = np.where(shocked, 0.0, -1.0)
    p = np.where(shocked, (g - 1) * rho * 0.5, 0.0)
    return rho, u, p


def noh_desc(cl, nu, schemes, N=None, t0=None, cfl=NOH_CFL, R=1.0, precision="fp64"):
    N = N or NOH_N[nu]
    t0 = NOH_T0[nu] if t0 is None else t0
    metric = {1: cl.CartesianMetric(), 2: cl.CylindricalMetric(), 3: cl.SphericalMetric()}[nu]
    lobc = {1: cl.SlipWallBC(), 2: cl.AxisBC(), 3: cl.OriginBC()}[nu]
    dom2 = (0.0, R / N) if nu == 1 else (0.0, 1.0) if nu == 2 else (math.pi / 2, math.pi / 2 + 1)
    dom3 = (0.0, R / N) if nu == 1 else (0.0, 1.0)

    def inflow(x, y, z, t):
        # a run that has lost positivity drives t to NaN: freeze the state at t0
        tt = t + t0 if math.isfinite(t) else t0
        rho, uu, _ = noh_exact(x, tt, nu, NOH_G)
        return cl.Prim(rho=rho, u=(uu, 0.0 * x, 0.0 * x), p=NOH_P0 + 0.0 * x)

    w = 4 * R / N

    def ic(x, y, z):
        if t0 <= 0:
            return cl.Prim(rho=1.0 + 0 * x, u=(-1.0 + 0 * x, 0.0, 0.0), p=NOH_P0 + 0 * x)
        rin, _, pin = noh_exact(0.0, t0, nu, NOH_G)
        rout, _, _ = noh_exact(x, t0, nu, NOH_G)
        th = cl.tanh_blend(x, (NOH_G - 1) / 2 * t0, w)
        return cl.Prim(rho=(1 - th) * rin + th * rout, u=(-th, 0.0 * x, 0.0 * x),
                       p=(1 - th) * pin + th * NOH_P0)

    bcs = ((lobc, cl.DirichletBC(inflow)), cl.PER3[1], cl.PER3[2])
    d = cl.solver_desc((N, 1, 1), (R, dom2[1] - dom2[0], dom3[1] - dom3[0]), bcs, *schemes,
                       eos=cl.single_species(gamma=NOH_G, R=1.0), transport=cl.Transport(mu0=0.0),
                       art=cl.ArtParams(enabled=True), origin=(0.0, dom2[0], dom3[0]), cfl=cfl,
                       filter_interval=1, metric=metric, precision=precision)
    return d, ic, NOH_T - t0


def front_position(xs, f, level):
    """Outermost crossing of `level` (test/references.jl:160-168)."""
    for i in range(len(f) - 1, 0, -1):
        lo, hi = f[i - 1], f[i]
        if (lo - level) * (hi - level) <= 0 and lo != hi:
            return xs[i - 1] + (xs[i] - xs[i - 1]) * (level - lo) / (hi - lo)
    return float("nan")


def noh_metrics(xs, rho, nu):
    """(plateau, wall deficit, shock radius, pre-shock L1) (test/cases.jl:298-310)."""
    exact = 4.0 ** nu
    Rs = (NOH_G - 1) / 2 * NOH_T
    core = (xs >= 0.3 * Rs) & (xs <= 0.7 * Rs)
    plat = float(rho[core].sum() / core.sum())
    pre = xs > Rs + 0.05
    epre = float(np.abs(rho[pre] - noh_exact(xs[pre], NOH_T, nu, NOH_G)[0]).sum() / pre.sum())
    return plat, 1 - rho[0] / exact, front_position(xs, rho, 0.5 * exact), epre


def check_noh(xs, rho, nu):
    """The validation battery's assertions (test/validation.jl:220-232); returns the metrics."""
    plat, deficit, Rnum, epre = noh_metrics(xs, rho, nu)
    exact = 4.0 ** nu
    assert abs(plat / exact - 1) < NOH_PTOL[nu], (nu, plat)
    assert 0 < deficit < 0.7, (nu, deficit)
    assert abs(Rnum - (NOH_G - 1) / 2 * NOH_T) < 0.025, (nu, Rnum)
    assert epre < 5e-2, (nu, epre)
    return plat, deficit, Rnum, epre
