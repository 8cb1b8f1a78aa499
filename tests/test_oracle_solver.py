"""Pins the CPU oracle's RHS, integrator and run loop against the reference's
known-answer tests and its measured/stored validation results
(test/runtests.jl, test/validation.jl, test/cases.jl, test/refs/*.csv)."""
import pathlib

import numpy as np
import pytest

import cases
import compactles_b200 as cl
import refsolutions as ref
from compactles_b200 import abi

GOLDEN = pathlib.Path(__file__).resolve().parent / "golden"


@pytest.fixture(scope="module")
def schemes(orc):
    return orc.lele_d1_6(), orc.compact_filter(0.45)


def _interior_max(orc, S, A):
    return float(np.abs(orc.interior(S.g, A)).max())


def test_freestream_preservation(orc, schemes):
    # test/runtests.jl:305-340 (Cartesian periodic case)
    d = cl.solver_desc((24, 12, 12), (1.0, 1.0, 1.0), cl.PER3, *schemes, art=cl.ArtParams(enabled=False))
    S = orc.Solver(d)
    S.set_state(cl.initialize(d, lambda x, y, z: cl.Prim(u=(0.0, 0.0, 0.0), p=1.0 + 0 * x, rho=1.0 + 0 * x)))
    S.apply_bcs()
    dQ = S.compute_rhs()
    assert _interior_max(orc, S, dQ) < 1e-8


def test_freestream_walls_and_art(orc, schemes):
    # uniform state between slip walls with artificial properties on
    d = cl.solver_desc((24, 16, 12), (1.0, 1.0, 1.0), ((cl.SlipWallBC(), cl.SlipWallBC()),) * 2 + (cl.PER3[2],),
                       *schemes)
    S = orc.Solver(d)
    S.set_state(cl.initialize(d, lambda x, y, z: cl.Prim(u=(0.0, 0.0, 0.0), p=1.0 + 0 * x, rho=1.0 + 0 * x)))
    S.apply_bcs()
    assert _interior_max(orc, S, S.compute_rhs()) < 1e-8


def test_eos_round_trip_two_species(orc, schemes):
    # test/runtests.jl:342-356
    eos = cl.IdealMixture([cl.IdealSpecies("a", 1.0, 1.4), cl.IdealSpecies("b", 0.2, 1.09)])
    d = cl.solver_desc((12, 12, 12), (2 * np.pi,) * 3, cl.PER3, *schemes, eos=eos, art=cl.ArtParams(enabled=False))
    S = orc.Solver(d)
    S.set_state(cl.initialize(d, lambda x, y, z: cl.Prim(u=(0.3, -0.1, 0.2), p=0.8 + 0 * x, T_ion=1.7 + 0 * x,
                                                        Y=(0.35, 0.65)), eos=eos))
    S.max_rate()  # exchange_state! + primitives!
    I = (4 + 4, 4 + 3, 4 + 2)  # gidx(solver, 3, 4, 5) in (z, y, x) order
    assert abs(S.field(abi.CLES_FIELD_P)[I] - 0.8) < 1e-12
    assert abs(S.field(abi.CLES_FIELD_T)[I] - 1.7) < 1e-12
    assert abs(S.field(abi.CLES_FIELD_U)[I] - 0.3) < 1e-12
    assert abs(S.field(abi.CLES_FIELD_Y0 + 1)[I] - 0.65) < 1e-12


def test_periodic_conservation(orc, schemes):
    # test/runtests.jl:409-421
    d = cl.solver_desc((16, 16, 16), (2 * np.pi,) * 3, cl.PER3, *schemes, transport=cl.Transport(mu0=1e-3),
                       art=cl.ArtParams(enabled=False))
    S = orc.Solver(d)
    S.set_state(cl.initialize(d, lambda x, y, z: cl.Prim(
        u=(0.1 * np.sin(x) * np.cos(y), -0.1 * np.cos(x) * np.sin(y), 0.05 * np.sin(z)),
        p=1 + 0.05 * np.cos(x) * np.cos(z), rho=1 + 0.1 * np.sin(y) + 0 * x)))
    dQ = orc.interior(S.g, S.compute_rhs())
    for c in range(5):
        assert abs(dQ[c].sum()) < 1e-8 * 16 ** 3


def test_conservation_with_artificial_two_species(orc, schemes):
    # Sum_k J_k = 0 and periodic divergence: every component integrates to 0
    eos = cl.IdealMixture([cl.IdealSpecies("a", 1.0, 1.4), cl.IdealSpecies("b", 0.2, 1.09)])
    d = cl.solver_desc((16, 12, 10), (2 * np.pi,) * 3, cl.PER3, *schemes, eos=eos, transport=cl.Transport(mu0=1e-3))
    S = orc.Solver(d)
    S.set_state(cases.random_smooth_state(d, seed=4, amp=0.2))
    dQ = orc.interior(S.g, S.compute_rhs())
    for c in range(6):
        assert abs(dQ[c].sum()) < 1e-9 * np.abs(dQ[c]).sum()


def test_step_control_floors(orc):
    # test/runtests.jl:667-691 (pure check_step)
    c = abi.step_control_default()
    ok = lambda dt, rho, seen=1.0, ctl=c: orc.check_step(ctl, dt, rho, seen)
    assert ok(1e-3, 1.0) is None
    assert ok(float("nan"), 1.0) == "nonfinite"
    assert ok(float("inf"), 1.0) == "nonfinite"
    assert ok(1e-3, -1e-9) == "negative_density"
    assert ok(1e-3, 0.0) == "negative_density"
    assert ok(1e-50, 1.0) == "planck"
    assert ok(1e-40, 1.0) == "dt_collapse"
    bare = cl.StepControl(dt_min=0.0, dt_min_ratio=0.0).to_c()
    assert ok(1e-50, 1.0, ctl=bare) == "planck"
    assert ok(1e-40, 1.0, ctl=bare) is None
    assert ok(1e-9, 1.0, ctl=cl.StepControl(dt_min=1e-6).to_c()) == "dt_min"
    assert ok(float("nan"), -1.0) == "nonfinite"


def test_max_rate_uniform_flow(orc, schemes):
    # test/runtests.jl:692-699: rho_min and the CFL rate of a quiet state
    d = cl.solver_desc((16, 16, 16), (2 * np.pi,) * 3, cl.PER3, *schemes)
    S = orc.Solver(d)
    S.set_state(cl.initialize(d, lambda x, y, z: cl.Prim(u=(0.2 * np.sin(x), 0 * x, 0 * x), p=1.0 + 0 * x, rho=1.0 + 0 * x)))
    rate, rmin = S.max_rate()
    assert abs(rmin - 1.0) < 1e-12
    h = 2 * np.pi / 16
    c = np.sqrt(1.4)
    assert abs(rate - (0.2 + 3 * c) / h) < 1e-9 * rate


@pytest.mark.parametrize("which", ["c6", "c10"])
def test_smoke_three_steps(orc, which):
    # test/runtests.jl:1880-1901 (Cartesian configurations)
    deriv = orc.lele_d1_6() if which == "c6" else orc.lele_d1_10()
    d = cl.solver_desc((16, 16, 16), (2 * np.pi,) * 3, cl.PER3, deriv, orc.compact_filter(0.45))
    S = orc.Solver(d)
    S.set_state(cl.initialize(d, lambda x, y, z: cl.Prim(u=(0.1 * np.sin(x), 0 * x, 0 * x), p=1.0 + 0 * x, rho=1.0 + 0 * x)))
    rc, res = S.run(1e9, 3)
    assert rc == 0 and res.steps == 3
    assert np.all(np.isfinite(orc.interior(S.g, S.get_state())))


def _profile(orc, S):
    S.max_rate()  # exchange_state! + primitives!
    sl = (S.field_shape[0] // 2, S.field_shape[1] // 2)
    rho = S.field(abi.CLES_FIELD_RHO)[sl][4:-4]
    u = S.field(abi.CLES_FIELD_U)[sl][4:-4]
    p = S.field(abi.CLES_FIELD_P)[sl][4:-4]
    return rho, u, p


def _xs(desc):
    return cl.coords(desc)[0]


def test_sod_matches_exact_riemann(orc, schemes):
    # test/runtests.jl:1903-1950: measured L1 rho 2.9e-3, u 4.6e-3, p 2.5e-3
    desc, Q0, tfin = cases.sod(schemes)
    S = orc.Solver(desc)
    S.set_state(Q0)
    rc, res = S.run(tfin, 100_000)
    assert rc == 0 and abs(res.t - tfin) < 1e-12
    rho, u, p = _profile(orc, S)
    xs = _xs(desc)
    er, eu, ep = ref.riemann_profile(xs, tfin, 0.5, (1.0, 0.0, 1.0), (0.125, 0.0, 0.1), 1.4)
    ps, us, _, _ = ref.riemann_star(1.0, 0.0, 1.0, 0.125, 0.0, 0.1, 1.4)
    assert abs(ps - 0.30313) < 1e-4 and abs(us - 0.92745) < 1e-4
    e_rho, e_u, e_p = ref.l1(rho, er), ref.l1(u, eu), ref.l1(p, ep)
    assert e_rho < 2e-2 and e_u < 2e-2 and e_p < 1e-2
    assert round(e_rho, 4) == 0.0029 and round(e_u, 4) == 0.0046 and round(e_p, 4) == 0.0025


@pytest.mark.slow
def test_lax_measured_l1(orc, schemes):
    # test/validation.jl:136-150; measured L1 rho 5.01e-3, u 7.53e-3, p 7.57e-3
    desc, Q0, tfin = cases.lax(schemes)
    S = orc.Solver(desc)
    S.set_state(Q0)
    rc, res = S.run(tfin, 2_000_000)
    assert rc == 0
    rho, u, p = _profile(orc, S)
    er, eu, ep = ref.riemann_profile(_xs(desc), tfin, 0.5, cases.LAX_L, cases.LAX_R, 1.4)
    e = (ref.l1(rho, er), ref.l1(u, eu), ref.l1(p, ep))
    assert e[0] < 1e-2 and e[1] < 1.5e-2 and e[2] < 1.5e-2
    assert abs(e[0] - 5.01e-3) < 0.02e-3 and abs(e[1] - 7.53e-3) < 0.02e-3 and abs(e[2] - 7.57e-3) < 0.02e-3


@pytest.mark.slow
def test_shu_osher_against_stored_reference(orc, schemes):
    # test/validation.jl:155-170 against test/refs/shu_osher.csv;
    # measured L1 rho 6.84e-3, wave train 2.08e-2, train peak 4.682
    desc, Q0, tfin = cases.shu_osher(schemes)
    S = orc.Solver(desc)
    S.set_state(Q0)
    rc, res = S.run(tfin, 2_000_000)
    assert rc == 0
    rho, _, _ = _profile(orc, S)
    xs = _xs(desc)
    xr, rr, _, _ = ref.read_profile(GOLDEN / "shu_osher.csv")
    rf = ref.interp1(xr, rr, xs)
    band = (xs >= 0.5) & (xs <= 2.2)
    l1_all, l1_band, peak = ref.l1(rho, rf), ref.l1(rho[band], rf[band]), float(rho[band].max())
    assert l1_all < 1.5e-2 and l1_band < 4e-2 and peak > 4.3
    assert abs(l1_all - 6.84e-3) < 0.02e-3
    assert abs(l1_band - 2.08e-2) < 0.02e-2
    assert abs(peak - 4.682) < 0.002


@pytest.mark.slow
def test_woodward_colella_against_stored_reference(orc, schemes):
    # test/validation.jl:180-193; measured L1 rho 3.15e-2, peak rho 6.595 at x = 0.7785
    desc, Q0, tfin = cases.woodward(schemes)
    S = orc.Solver(desc)
    S.set_state(Q0)
    rc, res = S.run(tfin, 2_000_000)
    assert rc == 0
    rho, _, _ = _profile(orc, S)
    xs = _xs(desc)
    xr, rr, _, _ = ref.read_profile(GOLDEN / "woodward_colella.csv")
    e = ref.l1(rho, ref.interp1(xr, rr, xs))
    imax = int(np.argmax(rho))
    assert np.all(np.isfinite(rho)) and rho.min() > 0 and e < 6e-2 and 0.75 < xs[imax] < 0.80
    assert abs(e - 3.15e-2) < 0.02e-2
    assert abs(rho[imax] - 6.595) < 0.005 and abs(xs[imax] - 0.7785) < 0.0005


@pytest.mark.slow
def test_noh_planar_measured(orc, schemes):
    # test/validation.jl:210-225 for nu = 1: plateau 3.9968/4, shock 0.2043/0.2, wall deficit 58%
    desc, Q0, tfin = cases.noh_planar(schemes)
    S = orc.Solver(desc)
    S.set_state(Q0)
    rc, res = S.run(tfin, 2_000_000)
    assert rc == 0
    rho, _, _ = _profile(orc, S)
    xs = _xs(desc)
    Rs = (cases.NOH_G - 1) / 2 * 0.6
    core = (xs >= 0.3 * Rs) & (xs <= 0.7 * Rs)
    plat = float(rho[core].mean())
    deficit = 1 - rho[0] / 4.0
    shock = ref.front_position(xs, rho, 2.0)
    assert abs(plat / 4 - 1) < 0.01 and 0 < deficit < 0.7 and abs(shock - 0.2) < 0.025
    assert abs(plat - 3.9968) < 0.001 and abs(shock - 0.2043) < 0.0005 and round(100 * deficit) == 58


@pytest.mark.slow
def test_run_failure_and_retry(orc, schemes):
    # test/runtests.jl:712-763: cfl 0.3 fails loudly; cfl 0.9 with retries recovers
    desc, Q0, tfin = cases.noh_planar(schemes, cfl=0.3)
    S = orc.Solver(desc)
    S.set_state(Q0)
    rc, res = S.run(tfin, 20_000)
    assert rc == abi.CLES_EFAILURE
    assert abi.FAIL_NAMES[res.failure] in ("negative_density", "dt_collapse")
    assert res.steps < 20_000
    desc, Q0, tfin = cases.noh_planar(schemes, cfl=0.9, control=cl.StepControl(retries=5, savepoint_interval=20))
    S = orc.Solver(desc)
    S.set_state(Q0)
    rc, res = S.run(tfin, 20_000)
    assert rc == 0
    assert abs(res.t - tfin) < 1e-9 * tfin
    assert res.cfl < 0.9 and res.cfl <= 0.9 * 0.5 + 1e-12
    rho, _, _ = _profile(orc, S)
    xs = _xs(desc)
    core = (xs >= 0.06) & (xs <= 0.14)
    assert abs(rho[core].mean() / 4.0 - 1) < 0.05
