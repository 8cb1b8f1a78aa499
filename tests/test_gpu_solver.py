"""GPU parity of the solver path (cles_compute_rhs / cles_step / cles_run
through the C ABI) against the CPU oracle on identical initial states.

Bounds (the FP64 drop-in's contract):
* per RHS, every conserved component c: max_points |dQ_gpu - dQ_oracle| is at
  most 1e-12 of that component's RHS scale, max(max|dQ_c|, max_d max|F_dc|/h_d).
  The second term is the size of the directional flux-divergence terms that
  are summed into dQ_c; it matters where they cancel (the energy equation of
  the Taylor-Green box sums terms of size ~250/h into an O(1) result, so an
  error of a few ulp of the terms is 1e-12 of the result);
* after 100 steps, the relative L2 difference of the state is at most 1e-10.
"""
import numpy as np
import pytest

import cases
import compactles_b200 as cl
import refsolutions as ref
from compactles_b200 import abi

pytestmark = pytest.mark.gpu


def rhs_errors(a, b, interior, scales=None):
    a = interior(a)
    b = interior(b)
    errs = []
    for c in range(b.shape[0]):
        sc = max(np.abs(b[c]).max(), scales[c] if scales else 0.0)
        errs.append(np.abs(a[c] - b[c]).max() / sc if sc > 0 else np.abs(a[c] - b[c]).max())
    return errs


def both(orc, desc_pair, Q0):
    dg, do = desc_pair
    S = cl.Solver(dg)
    S.set_state(Q0)
    O = orc.Solver(do)
    O.set_state(Q0)
    return S, O


def descs(orc, build, **kw):
    dg, Q0, tfin = build((cl.lele_d1_6(), cl.compact_filter(0.45)), **kw)
    do, _, _ = build((orc.lele_d1_6(), orc.compact_filter(0.45)), **kw)
    return (dg, do), Q0, tfin


def _interior(desc):
    sl = cl.interior_slices(desc)
    return lambda A: A[(slice(None),) + sl]


@pytest.mark.parametrize("n", [16, 64])
def test_tgv_rhs_parity(orc, n):
    pair, Q0, _ = descs(orc, cases.taylor_green, n=n)
    S, O = both(orc, pair, Q0)
    dQo = O.compute_rhs()
    errs = rhs_errors(S.compute_rhs(), dQo, _interior(pair[0]), O.rhs_scales(cl.grid_spacing(pair[0])))
    assert max(errs) < 1e-12, errs


@pytest.mark.parametrize("variant", ["walls_two_species", "c10", "gated", "dilatation", "viscous"])
def test_rhs_parity_variants(orc, variant):
    eos = cl.single_species()
    bcs = cl.PER3
    art = cl.ArtParams()
    tr = cl.Transport()
    mk_d = lambda m: m.lele_d1_6()
    ng = (24, 20, 16)
    if variant == "walls_two_species":
        eos = cl.IdealMixture([cl.IdealSpecies("a", 1.0, 1.4), cl.IdealSpecies("b", 0.2, 1.09)])
        bcs = (cl.PER3[0], (cl.SlipWallBC(), cl.SlipWallBC()), cl.PER3[2])
        tr = cl.Transport(mu0=1e-3)
    elif variant == "c10":
        mk_d = lambda m: m.lele_d1_10()
        bcs = ((cl.SlipWallBC(), cl.SlipWallBC()), cl.PER3[1], (cl.SlipWallBC(), cl.SlipWallBC()))
    elif variant == "gated":
        art = cl.ArtParams(beta_sensor="gated_strain")
    elif variant == "dilatation":
        art = cl.ArtParams(beta_sensor="dilatation")
        bcs = (cl.PER3[0], cl.PER3[1], (cl.SlipWallBC(), cl.SlipWallBC()))
    elif variant == "viscous":
        tr = cl.Transport(mu0=2e-3, Pr=0.72, Sc=0.9)
    L = (1.0, 1.3, 0.9)
    dg = cl.solver_desc(ng, L, bcs, mk_d(cl), cl.compact_filter(0.45), eos=eos, transport=tr, art=art)
    do = cl.solver_desc(ng, L, bcs, mk_d(orc), orc.compact_filter(0.45), eos=eos, transport=tr, art=art)
    Q0 = cases.random_smooth_state(dg, seed=11, amp=0.2)
    S, O = both(orc, (dg, do), Q0)
    S.apply_bcs()
    O.apply_bcs()
    dQo = O.compute_rhs()
    errs = rhs_errors(S.compute_rhs(), dQo, _interior(dg), O.rhs_scales(cl.grid_spacing(dg)))
    assert max(errs) < 1e-12, errs
    # the artificial coefficients themselves
    for which in (abi.CLES_FIELD_MU_ART, abi.CLES_FIELD_BETA_ART, abi.CLES_FIELD_KAPPA_ART):
        a = _interior(dg)(S.field(which)[None])
        b = _interior(dg)(O.field(which)[None])
        scale = max(np.abs(b).max(), 1e-300)
        assert np.abs(a - b).max() / scale < 1e-11


def test_max_rate_and_primitives_parity(orc):
    pair, Q0, _ = descs(orc, cases.taylor_green, n=32)
    S, O = both(orc, pair, Q0)
    S.compute_rhs()
    O.compute_rhs()
    rg, mg = S.max_rate()
    ro, mo = O.max_rate()
    assert abs(rg - ro) <= 1e-13 * ro and mg == mo
    for w in (abi.CLES_FIELD_RHO, abi.CLES_FIELD_P, abi.CLES_FIELD_T, abi.CLES_FIELD_C):
        a, b = S.field(w), O.field(w)
        sl = cl.interior_slices(pair[0])
        assert np.abs(a[sl] - b[sl]).max() <= 1e-14 * np.abs(b[sl]).max()


@pytest.mark.parametrize("deriv", ["c6", "c10"])
def test_hundred_steps_l2(orc, deriv):
    n = 24
    (dg, do), Q0, _ = descs(orc, cases.taylor_green, n=n)
    if deriv == "c10":
        dg.deriv = cl.lele_d1_10()
        do.deriv = orc.lele_d1_10()
    S, O = both(orc, (dg, do), Q0)
    rg = S.run(1e9, 100)
    ro = O.run(1e9, 100)[1]
    assert rg.steps == ro.steps == 100
    assert abs(rg.t - ro.t) <= 1e-12 * ro.t
    sl = (slice(None),) + cl.interior_slices(dg)
    a, b = S.get_state()[sl], O.get_state()[sl]
    rel = np.linalg.norm(a - b) / np.linalg.norm(b)
    assert rel < 1e-10, rel


def test_sod_on_gpu_matches_measured_and_oracle(orc):
    pair, Q0, tfin = descs(orc, cases.sod)
    S, O = both(orc, pair, Q0)
    res = S.run(tfin, 100_000)
    O.run(tfin, 100_000)
    assert abs(res.t - tfin) < 1e-12
    S.max_rate()
    xs = cl.coords(pair[0])[0]
    rho = S.field(abi.CLES_FIELD_RHO)[0, 0, 4:-4]
    u = S.field(abi.CLES_FIELD_U)[0, 0, 4:-4]
    p = S.field(abi.CLES_FIELD_P)[0, 0, 4:-4]
    er, eu, ep = ref.riemann_profile(xs, tfin, 0.5, (1.0, 0.0, 1.0), (0.125, 0.0, 0.1), 1.4)
    assert round(ref.l1(rho, er), 4) == 0.0029 and round(ref.l1(u, eu), 4) == 0.0046 and round(ref.l1(p, ep), 4) == 0.0025
    sl = (slice(None),) + cl.interior_slices(pair[0])
    a, b = S.get_state()[sl], O.get_state()[sl]
    assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-9


def test_shu_osher_on_gpu(orc):
    pair, Q0, tfin = descs(orc, cases.shu_osher)
    S, O = both(orc, pair, Q0)
    S.run(tfin, 2_000_000)
    O.run(tfin, 2_000_000)
    sl = (slice(None),) + cl.interior_slices(pair[0])
    a, b = S.get_state()[sl], O.get_state()[sl]
    assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-8


def test_run_failure_and_retry_on_gpu():
    sch = (cl.lele_d1_6(), cl.compact_filter(0.45))
    desc, Q0, tfin = cases.noh_planar(sch, cfl=0.3)
    S = cl.Solver(desc)
    S.set_state(Q0)
    with pytest.raises(cl.SolverFailure) as ei:
        S.run(tfin, 20_000)
    assert ei.value.reason in ("negative_density", "dt_collapse")
    desc, Q0, tfin = cases.noh_planar(sch, cfl=0.9, control=cl.StepControl(retries=5, savepoint_interval=20))
    S = cl.Solver(desc)
    S.set_state(Q0)
    res = S.run(tfin, 20_000)
    assert abs(res.t - tfin) < 1e-9 * tfin and res.cfl <= 0.45 + 1e-12
    S.max_rate()
    xs = cl.coords(desc)[0]
    rho = S.field(abi.CLES_FIELD_RHO)[0, 0, 4:-4]
    core = (xs >= 0.06) & (xs <= 0.14)
    assert abs(rho[core].mean() / 4 - 1) < 0.05


def test_freestream_and_conservation_on_gpu():
    d = cl.solver_desc((24, 12, 12), (1.0, 1.0, 1.0), cl.PER3, cl.lele_d1_6(), cl.compact_filter(0.45),
                       art=cl.ArtParams(enabled=False))
    S = cl.Solver(d)
    S.set_state(cl.initialize(d, lambda x, y, z: cl.Prim(u=(0.0, 0.0, 0.0), p=1.0 + 0 * x, rho=1.0 + 0 * x)))
    assert np.abs(S.compute_rhs(layout="interior")).max() < 1e-8
    d = cl.solver_desc((16, 16, 16), (2 * np.pi,) * 3, cl.PER3, cl.lele_d1_6(), cl.compact_filter(0.45),
                       transport=cl.Transport(mu0=1e-3), art=cl.ArtParams(enabled=False))
    S = cl.Solver(d)
    S.set_state(cl.initialize(d, lambda x, y, z: cl.Prim(
        u=(0.1 * np.sin(x) * np.cos(y), -0.1 * np.cos(x) * np.sin(y), 0.05 * np.sin(z)),
        p=1 + 0.05 * np.cos(x) * np.cos(z), rho=1 + 0.1 * np.sin(y) + 0 * x)))
    dQ = S.compute_rhs(layout="interior")
    for c in range(5):
        assert abs(dQ[c].sum()) < 1e-8 * 16 ** 3


def test_diagnostics_parity(orc):
    pair, Q0, _ = descs(orc, cases.taylor_green, n=32)
    S, O = both(orc, pair, Q0)
    assert abs(S.kinetic_energy() - O.kinetic_energy()) < 1e-13 * O.kinetic_energy()
    eg, eo = S.dissipation_rate(), O.dissipation_rate()
    assert abs(eg - eo) < 1e-11 * abs(eo)


def test_mixed_precision_rhs_close(orc):
    pair, Q0, _ = descs(orc, cases.taylor_green, n=32)
    dg = pair[0]
    dg.precision = abi.CLES_PREC_MIXED
    S, O = both(orc, (dg, pair[1]), Q0)
    dQo = O.compute_rhs()
    errs = rhs_errors(S.compute_rhs(), dQo, _interior(dg), O.rhs_scales(cl.grid_spacing(dg)))
    # FP32 fields and line solves: a few single-precision ulps of the terms
    assert max(errs) < 2e-6, errs


def test_body_forces_match_oracle(orc):
    # ConstantBodyForce sources (src/sources.jl:42-82): the reference's known
    # answer on a uniform state (test/runtests.jl:374-388), then a stratified
    # box under gravity against the oracle: RHS to 1e-12, 20 steps to 1e-10
    force = cl.ConstantBodyForce((1.0, 2.0, -3.0))
    d = cl.solver_desc((12, 12, 12), (2 * np.pi,) * 3, cl.PER3, cl.lele_d1_6(), cl.compact_filter(0.45),
                       art=cl.ArtParams(enabled=False), sources=(force,))
    S = cl.Solver(d)
    S.set_state(cl.initialize(d, lambda x, y, z: cl.Prim(u=(0.5 + 0 * x, 0.25 + 0 * y, -0.1 + 0 * z),
                                                         p=1.0 + 0 * x, rho=2.0 + 0 * x)))
    dQ = _interior(d)(S.compute_rhs())
    assert np.allclose(dQ[1], 2.0, atol=1e-10) and np.allclose(dQ[2], 4.0, atol=1e-10)
    assert np.allclose(dQ[3], -6.0, atol=1e-10) and np.allclose(dQ[4], 2.6, atol=1e-10)
    g = (cl.ConstantBodyForce((0.0, -1.0, 0.0)), cl.ConstantBodyForce((0.05, 0.0, 0.0)))
    PER = (cl.PeriodicBC(), cl.PeriodicBC())
    bcs = (PER, (cl.SlipWallBC(), cl.SlipWallBC()), PER)
    ic = lambda x, y, z: cl.Prim(u=(0.1 * np.sin(x), 0.0 * y, 0.05 * np.cos(z)), p=2.0 - 0.3 * y / np.pi + 0 * x,
                                 rho=1.0 + 0.1 * np.cos(x) + 0 * z)
    pair = [cl.solver_desc((16, 24, 12), (2 * np.pi, 2 * np.pi, 2 * np.pi), bcs, *sch, art=cl.ArtParams(enabled=True),
                           sources=g) for sch in ((cl.lele_d1_6(), cl.compact_filter(0.45)),
                                                  (orc.lele_d1_6(), orc.compact_filter(0.45)))]
    Q0 = cl.initialize(pair[0], ic)
    S, O = both(orc, pair, Q0)
    S.apply_bcs()
    O.apply_bcs()
    errs = rhs_errors(S.compute_rhs(), O.compute_rhs(), _interior(pair[0]), O.rhs_scales(cl.grid_spacing(pair[0])))
    assert max(errs) < 1e-12, errs
    S.run(1e9, 20)
    assert O.run(1e9, 20)[0] == 0
    it = _interior(pair[0])
    a, b = it(S.get_state()), it(O.get_state())
    assert np.linalg.norm(a - b) <= 1e-10 * np.linalg.norm(b)
