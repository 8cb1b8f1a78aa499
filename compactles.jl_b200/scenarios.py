"""Scenario builders for the ensemble and serving workloads.

Each builder returns (desc, Q0, tfinal): a cles_solver_desc, the padded
initial state and the end time.  Schemes are passed in so that the same
builders serve the CUDA library and the CPU oracle.

* two_species_tube: a 1-D two-species shock tube between slip walls, the
  pattern of test/runtests.jl:1903-1950 with a second species
  (R2 = (1 - A)/(1 + A) for Atwood number A, gamma 1.4 for both), a pressure
  ratio across the diaphragm at x = 0.5, equal temperatures, tanh smearing
  of two cells, run to t = 0.2.
* shock_interface_2d: a planar shock in helium hitting a perturbed He/CO2
  interface (the geometry of examples/shock_tube.jl): IdealMixture of He
  (gamma 5/3, W 4.0026e-3) and CO2 (gamma 1.289, W 44.01e-3), pre-shock He at
  1 atm and 300 K, post-shock state from the normal-shock relations of the
  given Mach number at x = 0.2 Lx, interface at 0.4 Lx plus an 8-mode seeded
  perturbation, tanh thickness 3 cells, slip walls in x, periodic in y, run
  to 0.5 Lx / c_He.  Mode m has weight U[0.2, 1] / m^2 ("red", the default):
  with equal weights ("flat") about a third of the cases end in
  SolverFailure(:nonfinite) a little after the shock reaches the interface,
  on the CPU oracle and on the device at the same step, because the upper
  modes are only 8-16 cells long.
* taylor_green_box: the README Taylor-Green vortex on an n^3 periodic box.
* slip_wall_box: the same velocity field on [0, pi]^3 closed by slip walls on
  all six faces (the field's normal velocity vanishes on each of them): every
  line is closed, so the x pass runs the closed-line x kernel with its
  subtract store and the z pass the closed-line RK-fused store.
* he_co2_shock_tube: examples/shock_tube.jl -- a 4 m closed tube of a NASA-9
  He/CO2 mixture at 300 K, 10 atm He driver against 1 atm He, diaphragm at
  2 m, sinusoidally perturbed He/CO2 contact at 3 m (amplitude 10% of the
  0.2 m span, one wavelength), diffuse widths 3 h_x, slip walls in x,
  periodic y, artificial properties on, cfl 0.5 with four rollback retries,
  run to 2.5 ms.  The NASA-9 mixture is passed in (read_nasa9 on a CEA
  thermo.inp, He then CO2).
"""
import math

import numpy as np

from .problem import (ArtParams, IdealMixture, IdealSpecies, PER3, Prim, SlipWallBC, StepControl, Transport,
                      initialize, single_species, solver_desc, tanh_blend, taylor_green_problem)

R_UNIVERSAL = 8.31446261815324  # J/(mol K), src/nasa9_data.jl:19


def two_species_tube(schemes, N, pressure_ratio, atwood, cfl=0.4, tfinal=0.2, precision="fp64"):
    deriv, filt = schemes
    R1, R2 = 1.0, (1.0 - atwood) / (1.0 + atwood)
    eos = IdealMixture([IdealSpecies("light", R1, 1.4), IdealSpecies("heavy", R2, 1.4)])
    h = 1.0 / (N - 1)
    desc = solver_desc((N, 1, 1), (1.0, h, h), ((SlipWallBC(), SlipWallBC()), PER3[1], PER3[2]), deriv, filt,
                       eos=eos, transport=Transport(mu0=0.0), art=ArtParams(enabled=True), cfl=cfl,
                       filter_interval=1, precision=precision)

    def ic(x, y, z):
        th = tanh_blend(x, 0.5, 2 * h)
        return Prim(p=(1 - th) * pressure_ratio + th * 1.0, T_ion=1.0 + 0 * x, u=(0 * x, 0 * x, 0 * x),
                    Y=(1 - th, th))
    return desc, initialize(desc, ic, eos=eos), tfinal


def normal_shock(M, gamma, rho1, p1):
    """Post-shock (rho2, u2, p2) behind a shock of Mach M moving into gas at rest."""
    c1 = math.sqrt(gamma * p1 / rho1)
    p2 = p1 * (1 + 2 * gamma / (gamma + 1) * (M * M - 1))
    rho2 = rho1 * (gamma + 1) * M * M / ((gamma - 1) * M * M + 2)
    u2 = c1 * 2 / (gamma + 1) * (M - 1 / M)
    return rho2, u2, p2


def shock_interface_2d(schemes, nx, ny, mach, seed, cfl=0.5, precision="fp64", spectrum="red"):
    deriv, filt = schemes
    rng = np.random.default_rng(seed)
    g_he, g_co2 = 5.0 / 3.0, 1.289
    R_he, R_co2 = R_UNIVERSAL / 4.0026e-3, R_UNIVERSAL / 44.01e-3
    eos = IdealMixture([IdealSpecies("He", R_he, g_he), IdealSpecies("CO2", R_co2, g_co2)])
    Ly = 1.0
    h = Ly / ny
    Lx = h * (nx - 1)
    p1, T1 = 101325.0, 300.0
    rho1 = p1 / (R_he * T1)
    c_he = math.sqrt(g_he * p1 / rho1)
    rho2, u2, p2 = normal_shock(mach, g_he, rho1, p1)
    amp_total = rng.uniform(0.05, 0.15) * Ly
    w = rng.uniform(0.2, 1.0, size=8)
    if spectrum == "red":
        w = w / np.arange(1, 9) ** 2
    A = amp_total * w / w.sum() * rng.choice([-1, 1], size=8)
    phi = rng.uniform(0, 2 * math.pi, size=8)
    xs, xi0 = 0.2 * Lx, 0.4 * Lx
    desc = solver_desc((nx, ny, 1), (Lx, Ly, h), ((SlipWallBC(), SlipWallBC()), PER3[1], PER3[2]), deriv, filt,
                       eos=eos, transport=Transport(mu0=0.0), art=ArtParams(enabled=True), cfl=cfl,
                       filter_interval=1, precision=precision)

    def ic(x, y, z):
        xi = xi0 + sum(A[m] * np.cos(2 * math.pi * (m + 1) * y / Ly + phi[m]) for m in range(8))
        ths = tanh_blend(x, xs, 3 * h)          # 0 behind the shock, 1 ahead of it
        thi = tanh_blend(x, xi, 3 * h)          # 0 helium, 1 carbon dioxide
        Yco2 = thi + 0 * x + 0 * y
        Yhe = 1 - Yco2
        p = (1 - ths) * p2 + ths * p1 + 0 * y
        rho_pre = 1.0 / (Yhe / rho1 + Yco2 / (p1 / (R_co2 * T1)))   # same p and T on both sides
        rho = (1 - ths) * rho2 + ths * rho_pre
        u = (1 - ths) * u2 + 0 * y
        return Prim(rho=rho, p=p, u=(u, 0 * u, 0 * u), Y=(Yhe, Yco2))
    return desc, initialize(desc, ic, eos=eos), 0.5 * Lx / c_he


def taylor_green_box(schemes, n, tfinal=1.0, precision="fp64"):
    deriv, filt = schemes
    prob = taylor_green_problem()
    tp = 2 * math.pi
    desc = solver_desc((n, n, n), (tp, tp, tp), prob.bcs, deriv, filt, precision=precision)
    return desc, initialize(desc, prob.ic), tfinal


def slip_wall_box(schemes, n, tfinal=1.0, precision="fp64"):
    deriv, filt = schemes
    wall = (SlipWallBC(), SlipWallBC())
    desc = solver_desc((n, n, n), (math.pi,) * 3, (wall, wall, wall), deriv, filt, precision=precision)

    def ic(x, y, z):
        return Prim(u=(np.sin(x) * np.cos(y), -np.cos(x) * np.sin(y), 0.0 * z), p=71.43 + 0.0 * x, rho=1.0 + 0.0 * x)
    return desc, initialize(desc, ic), tfinal


def he_co2_shock_tube(schemes, eos, nx=768, ny=48, tfinal=2.5e-3, precision="fp64", retries=4):
    deriv, filt = schemes
    Lx, Lyz = 4.0, 0.2
    atm = 101325.0
    p_driver, p_driven, T0 = 10 * atm, 1 * atm, 300.0
    hx = Lx / (nx - 1)
    delta = 3 * hx
    desc = solver_desc((nx, ny, 1), (Lx, Lyz, Lyz), ((SlipWallBC(), SlipWallBC()), PER3[1], PER3[2]), deriv, filt,
                       eos=eos, transport=Transport(mu0=0.0), art=ArtParams(enabled=True), cfl=0.5,
                       control=StepControl(retries=retries), filter_interval=1, precision=precision)

    def ic(x, y, z):
        xi = 3.0 + 0.1 * Lyz * np.cos(2 * math.pi * y / Lyz)
        th = tanh_blend(x, xi, delta)
        p = p_driven + (p_driver - p_driven) * (1 - tanh_blend(x, 2.0, delta))
        return Prim(Y=(1 - th, th), p=p + 0 * y, T_ion=T0 + 0 * x + 0 * y)
    return desc, initialize(desc, ic, eos=eos), tfinal
