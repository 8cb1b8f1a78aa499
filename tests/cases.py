"""Case builders shared by the oracle pins and the GPU parity tests.

Each builder returns (desc, Q0, tfinal): a cles_solver_desc and the initial
conserved state in the padded layout, evaluated once so that the oracle and
the GPU start from identical bits.  The 1-D cases restate test/cases.jl and
the Sod test of test/runtests.jl:1903-1950; the Taylor-Green box is the
README quick-start (README.md:31-39)."""
import numpy as np

import compactles_b200 as cl
from compactles_b200 import abi


def _tube_desc(N, L, xlo, left_bc, right_bc, cfl, schemes, gamma=1.4):
    h = L / (N - 1)
    deriv, filt = schemes
    return cl.solver_desc((N, 1, 1), (L, h, h), ((left_bc, right_bc), cl.PER3[1], cl.PER3[2]),
                          deriv, filt, eos=cl.single_species(gamma=gamma, R=1.0),
                          transport=cl.Transport(mu0=0.0), art=cl.ArtParams(enabled=True),
                          origin=(xlo, 0.0, 0.0), cfl=cfl, filter_interval=1)


def _tube_ic(left, right, x0, delta, rhofun=None):
    rL, uL, pL = left
    rR, uR, pR = right

    def ic(x, y, z):
        th = cl.tanh_blend(x, x0, delta)
        rr = rR if rhofun is None else rhofun(x)
        return cl.Prim(rho=(1 - th) * rL + th * rr, u=((1 - th) * uL + th * uR, 0.0 * x, 0.0 * x),
                       p=(1 - th) * pL + th * pR)
    return ic


def tube(left, right, N, tfin, schemes, L=1.0, xlo=0.0, x0=0.5, cfl=0.4, rhofun=None, delta=None):
    """tube(left, right; N, L, x0, tfin, ...) with Dirichlet ends (test/cases.jl:78-100)."""
    h = L / (N - 1)
    d = 2 * h if delta is None else delta
    rL, uL, pL = left
    rR, uR, pR = right
    x_hi = xlo + (N - 1) * h
    rr_hi = rR if rhofun is None else float(rhofun(np.float64(x_hi)))
    lbc = cl.DirichletBC(cl.Prim(rho=rL, u=(uL, 0.0, 0.0), p=pL))
    rbc = cl.DirichletBC(cl.Prim(rho=rr_hi, u=(uR, 0.0, 0.0), p=pR))
    desc = _tube_desc(N, L, xlo, lbc, rbc, cfl, schemes)
    Q0 = cl.initialize(desc, _tube_ic(left, right, x0, d, rhofun))
    return desc, Q0, tfin


LAX_L = (0.445, 0.698, 3.528)
LAX_R = (0.5, 0.0, 0.571)


def lax(schemes, N=400):
    return tube(LAX_L, LAX_R, N, 0.14, schemes)


SO_L = (3.857143, 2.629369, 10.333333333333333)


def shu_osher(schemes, N=800):
    return tube(SO_L, (1.0, 0.0, 1.0), N, 1.8, schemes, L=10.0, xlo=-5.0, x0=-4.0,
                rhofun=lambda x: 1 + 0.2 * np.sin(5 * x))


def sod(schemes, N=400):
    """Sod with slip walls (test/runtests.jl:1903-1950)."""
    h = 1.0 / (N - 1)
    desc = _tube_desc(N, 1.0, 0.0, cl.SlipWallBC(), cl.SlipWallBC(), 0.4, schemes)
    Q0 = cl.initialize(desc, _tube_ic((1.0, 0.0, 1.0), (0.125, 0.0, 0.1), 0.5, 2 * h))
    return desc, Q0, 0.2


def woodward(schemes, N=800):
    """Woodward-Colella blast waves between slip walls (test/cases.jl:140-160)."""
    h = 1.0 / (N - 1)
    d = 2 * h
    desc = _tube_desc(N, 1.0, 0.0, cl.SlipWallBC(), cl.SlipWallBC(), 0.3, schemes)

    def ic(x, y, z):
        a = cl.tanh_blend(x, 0.1, d)
        b = cl.tanh_blend(x, 0.9, d)
        return cl.Prim(rho=1.0 + 0 * x, u=(0 * x, 0 * x, 0 * x), p=1000 * (1 - a) + 0.01 * (a - b) + 100 * b)
    return desc, cl.initialize(desc, ic), 0.038


NOH_G = 5.0 / 3.0
NOH_P0 = 1e-4


def noh_planar(schemes, N=400, cfl=0.15, control=None):
    """Planar Noh (nu = 1): slip wall at x = 0, exact (constant) inflow at x = 1
    (test/cases.jl:224-262 with nu = 1; test/runtests.jl:712-763)."""
    deriv, filt = schemes
    inflow = cl.DirichletBC(cl.Prim(rho=1.0, u=(-1.0, 0.0, 0.0), p=NOH_P0))
    desc = cl.solver_desc((N, 1, 1), (1.0, 1.0 / N, 1.0 / N), ((cl.SlipWallBC(), inflow), cl.PER3[1], cl.PER3[2]),
                          deriv, filt, eos=cl.single_species(gamma=NOH_G, R=1.0),
                          transport=cl.Transport(mu0=0.0), art=cl.ArtParams(enabled=True),
                          cfl=cfl, filter_interval=1, control=control)
    Q0 = cl.initialize(desc, lambda x, y, z: cl.Prim(rho=1.0 + 0 * x, u=(-1.0 + 0 * x, 0 * x, 0 * x), p=NOH_P0 + 0 * x))
    return desc, Q0, 0.6


def taylor_green(schemes, n=64, art=None, transport=None, cfl=0.5, precision="fp64", p0=71.43):
    deriv, filt = schemes
    prob = cl.taylor_green_problem(p0=p0)
    two_pi = 2 * np.pi
    desc = cl.solver_desc((n, n, n), (two_pi, two_pi, two_pi), prob.bcs, deriv, filt,
                          art=art or cl.ArtParams(), transport=transport or cl.Transport(),
                          cfl=cfl, precision=precision)
    return desc, cl.initialize(desc, prob.ic), 1.0


def random_smooth_state(desc, seed=3, amp=0.05):
    """A smooth, positive, non-trivial state for RHS parity checks: a few
    seeded Fourier modes on top of a uniform gas (periodic dims only vary
    smoothly; closed dims get polynomial-free smooth profiles)."""
    rng = np.random.default_rng(seed)
    x, y, z = cl.coords(desc)
    X, Y, Z = x[None, None, :], y[None, :, None], z[:, None, None]
    L = [desc.L[k] if desc.n_global[k] > 1 else 1.0 for k in range(3)]

    def mode():
        k = rng.integers(1, 3, size=3)
        ph = rng.uniform(0, 2 * np.pi, size=3)
        return (np.sin(2 * np.pi * k[0] * X / L[0] + ph[0]) * np.cos(2 * np.pi * k[1] * Y / L[1] + ph[1])
                * np.cos(2 * np.pi * k[2] * Z / L[2] + ph[2]))

    ns = desc.n_species
    Ys = [np.full(1, 1.0)] if ns == 1 else None
    if ns > 1:
        w = [1.0 + 0.3 * mode() for _ in range(ns)]
        tot = sum(w)
        Ys = [wi / tot for wi in w]
    pr = cl.Prim(rho=1.0 + amp * mode(), u=(amp * mode(), amp * mode(), amp * mode()),
                 p=1.0 + amp * mode(), Y=tuple(Ys))
    eos = cl.IdealMixture([cl.IdealSpecies(f"s{k}", desc.R[k], desc.gamma[k]) for k in range(ns)])
    return cl.initialize(desc, lambda *_: pr, eos=eos)
