"""Device parity of the curvilinear metrics, stretching and coordinate folds.

* the reference's own known answers on the device: a uniform state gives
  dQ ~ 0 in every metric, with stretching and with folds
  (test/runtests.jl:305-330), and rigid rotation has zero strain
  (test/runtests.jl:285-303);
* the velocity gradients (1/h scaling, curvature terms, fold parities) match
  the oracle to 1e-12 of their scale;
* the RHS matches the oracle per component to 1e-12 of the component's RHS
  scale, and 20 steps to 1e-10 in relative L2 (momentum against the momentum
  vector), in FP64, with and without artificial properties (one step for the
  two ill-conditioned cases named at ILL_CONDITIONED);
* the mixed form stays within FP32 rounding of the oracle, and graph mode
  reproduces the stepped run bitwise.
"""
import math

import numpy as np
import pytest

import compactles_b200 as cl

pytestmark = pytest.mark.gpu

PER = (cl.PeriodicBC(), cl.PeriodicBC())


def _ic_axisym(r, t, z):
    g = np.exp(-4 * r ** 2)
    return cl.Prim(u=(0.2 * r * g, 0.1 * r * g * (1 + 0 * t), 0.05 * np.cos(2 * np.pi * z / 0.5) + 0 * r),
                   p=1.0 + 0.1 * g * np.cos(2 * np.pi * z / 0.5), rho=1.0 + 0.05 * g + 0 * z)


def _ic_plane(r, t, z):
    # theta-dependent scalars; theta-independent velocity components (radial
    # inflow plus swirl), whose antipodal continuation the paired fold
    # reproduces for either parity
    x, y = r * np.cos(t), r * np.sin(t)
    g = np.exp(-4 * r ** 2)
    return cl.Prim(u=(-0.2 * r * g + 0 * t, 0.1 * r * g + 0 * t, 0 * r + 0 * z),
                   p=1.0 + 0.1 * np.exp(-5 * ((x - 0.2) ** 2 + y ** 2)),
                   rho=1.0 + 0.05 * np.exp(-4 * ((x + 0.1) ** 2 + y ** 2)))


def _ic_sphere(r, t, p):
    g = np.exp(-4 * r ** 2)
    return cl.Prim(u=(0.1 * r * g + 0 * t, 0.05 * r * g * np.sin(t), 0.02 * r * g * np.sin(t) * np.cos(p)),
                   p=1.0 + 0.1 * g + 0 * p, rho=1.0 + 0.05 * g * (1 + 0.2 * np.cos(t)) + 0 * p)


def _ic_annulus(r, t, z):
    return cl.Prim(u=(0.05 * np.sin(np.pi * (r - 0.2)) * np.cos(t), 0.3 * r + 0.05 * np.sin(2 * t),
                      0.05 * np.cos(2 * np.pi * z / 0.5) + 0 * r),
                   p=1.0 + 0.1 * np.exp(-10 * (r - 0.7) ** 2) * np.cos(t), rho=1.0 + 0 * r + 0 * z)


def _ic_stretched(x, y, z):
    return cl.Prim(u=(0.1 * np.sin(np.pi * x) * np.cos(2 * np.pi * y), 0.05 * np.cos(np.pi * x) + 0 * y,
                      0.02 * np.sin(2 * np.pi * z) + 0 * x),
                   p=1.0 + 0.1 * np.exp(-20 * (x - 0.4) ** 2) + 0 * y, rho=1.0 + 0.05 * np.cos(np.pi * x) + 0 * z)


CASES = {
    "stretched": dict(n=(40, 16, 12), L=(1.0, 1.0, 1.0), metric=None,
                      bcs=((cl.SlipWallBC(), cl.SlipWallBC()), PER, PER), ic=_ic_stretched,
                      stretch=(cl.sine_cluster(0.0, 1.0, 0.4, 0.4), None, None)),
    "annulus": dict(n=(32, 24, 12), L=(1.0, 2 * math.pi, 0.5), metric=cl.CylindricalMetric(),
                    bcs=((cl.SlipWallBC(), cl.SlipWallBC()), PER, PER), ic=_ic_annulus, origin=(0.2, 0.0, 0.0)),
    "axis_axisym": dict(n=(40, 1, 12), L=(1.0, 1.0, 0.5), metric=cl.CylindricalMetric(),
                        bcs=((cl.AxisBC(), cl.SlipWallBC()), PER, PER), ic=_ic_axisym),
    "axis_resolved": dict(n=(32, 16, 1), L=(1.0, 2 * math.pi, 1.0), metric=cl.CylindricalMetric(),
                          bcs=((cl.AxisBC(), cl.SlipWallBC()), PER, PER), ic=_ic_plane),
    "sphere": dict(n=(24, 16, 12), L=(1.0, math.pi, 2 * math.pi), metric=cl.SphericalMetric(),
                   bcs=((cl.OriginBC(), cl.SlipWallBC()), (cl.PoleBC(), cl.PoleBC()), PER), ic=_ic_sphere),
    "sphere_axisym": dict(n=(24, 16, 1), L=(1.0, math.pi, 2 * math.pi), metric=cl.SphericalMetric(),
                          bcs=((cl.OriginBC(), cl.SlipWallBC()), (cl.PoleBC(), cl.PoleBC()), PER),
                          ic=lambda r, t, p: _ic_sphere(r, t, 0 * p)),
}


def _pair(orc, case, art=False, precision="fp64", mu0=1e-3, eos=None, ic=None):
    c = CASES[case]

    def mk(sch, prec):
        return cl.solver_desc(c["n"], c["L"], c["bcs"], *sch, eos=eos, art=cl.ArtParams(enabled=art),
                              transport=cl.Transport(mu0=mu0), origin=c.get("origin", (0.0, 0.0, 0.0)),
                              metric=c["metric"], stretch=c.get("stretch", (None, None, None)), cfl=0.4,
                              precision=prec)
    dg = mk((cl.lele_d1_6(), cl.compact_filter(0.45)), precision)
    do = mk((orc.lele_d1_6(), orc.compact_filter(0.45)), "fp64")
    Q0 = cl.initialize(dg, ic or c["ic"], eos=eos)
    S = cl.Solver(dg)
    S.set_state(Q0)
    O = orc.Solver(do)
    O.set_state(Q0)
    return S, O, dg


def _it(d):
    sl = cl.interior_slices(d)
    return lambda A: A[(slice(None),) + sl]


@pytest.mark.parametrize("case", ["stretched", "annulus", "axis_axisym", "axis_resolved", "sphere"])
def test_freestream_on_device(orc, case):
    uniform = lambda x, y, z: cl.Prim(u=(0.0, 0.0, 0.0), p=1.0 + 0 * x, rho=1.0 + 0 * x)
    S, O, d = _pair(orc, case, mu0=0.0, ic=uniform)
    S.apply_bcs()
    dQ = _it(d)(S.compute_rhs())
    assert np.abs(dQ).max() < 1e-8


def test_rigid_rotation_zero_strain_on_device(orc):
    d = cl.solver_desc((32, 16, 12), (1.0, 2 * math.pi, 0.5), ((cl.SlipWallBC(), cl.SlipWallBC()), PER, PER),
                       cl.lele_d1_6(), cl.compact_filter(0.45), art=cl.ArtParams(enabled=False),
                       metric=cl.CylindricalMetric(), origin=(0.2, 0.0, 0.0))
    S = cl.Solver(d)
    S.set_state(cl.initialize(d, lambda r, t, z: cl.Prim(u=(0.0 * r, 0.3 * r, 0.0 * r), p=1.0 + 0 * r,
                                                         rho=1.0 + 0 * r)))
    S.compute_rhs()
    sl = cl.interior_slices(d)
    g = [[S.field(cl.abi.CLES_FIELD_GRAD_U0 + 3 * a + b)[sl] for b in range(3)] for a in range(3)]
    smax = max(float(np.abs(0.5 * (g[a][b] + g[b][a])).max()) for a in range(3) for b in range(3))
    assert smax < 1e-8


@pytest.mark.parametrize("case", list(CASES))
def test_gradients_match_oracle(orc, case):
    S, O, d = _pair(orc, case)
    S.compute_rhs()
    O.compute_rhs()
    sl = cl.interior_slices(d)
    gs = [S.field(cl.abi.CLES_FIELD_GRAD_U0 + e)[sl] for e in range(9)]
    go = [O.field(cl.abi.CLES_FIELD_GRAD_U0 + e)[sl] for e in range(9)]
    scale = max(float(np.abs(g).max()) for g in go)
    for e in range(9):
        assert np.abs(gs[e] - go[e]).max() <= 1e-12 * scale, e


# With artificial properties on, the paired-fold cases are ill-conditioned: in
# the oracle alone a 1e-15 perturbation of the initial state grows to 2e-8
# (resolved axis, 3 steps) and 1.6e-4 (sphere, 20 steps) in relative L2, while
# every other case stays near 1e-13.  Those two are checked over one step.
ILL_CONDITIONED = {("axis_resolved", True), ("sphere", True)}


@pytest.mark.parametrize("case", list(CASES))
@pytest.mark.parametrize("art", [False, True])
def test_rhs_and_steps_match_oracle(orc, case, art):
    steps = 1 if (case, art) in ILL_CONDITIONED else 20
    S, O, d = _pair(orc, case, art=art)
    it = _it(d)
    S.apply_bcs()
    O.apply_bcs()
    dQo = it(O.compute_rhs())
    dQ = it(S.compute_rhs())
    sc = O.rhs_scales(cl.grid_spacing(d))
    for c in range(dQo.shape[0]):
        ref = max(np.abs(dQo[c]).max(), sc[c])
        assert np.abs(dQ[c] - dQo[c]).max() <= 1e-12 * ref, c
    S.run(1e9, steps)
    rc, _ = O.run(1e9, steps)
    assert rc == 0
    a, b = it(S.get_state()), it(O.get_state())
    mom = math.sqrt(sum(np.linalg.norm(b[c]) ** 2 for c in (1, 2, 3)))
    for c in range(b.shape[0]):
        ref = mom if c in (1, 2, 3) else np.linalg.norm(b[c])
        assert np.linalg.norm(a[c] - b[c]) <= 1e-10 * ref, c
    # the step sizes come from rate reductions that round differently
    assert S.t == pytest.approx(O.clock()[0], rel=1e-9)


def test_two_species_axis(orc):
    two = cl.IdealMixture([cl.IdealSpecies("a", 1.0, 1.4), cl.IdealSpecies("b", 0.25, 1.4)])

    def ic(r, t, z):
        g = np.exp(-4 * r ** 2)
        y0 = 0.5 + 0.3 * g * np.cos(2 * np.pi * z / 0.5)
        return cl.Prim(Y=(y0, 1 - y0), u=(0.2 * r * g, 0.1 * r * g, 0.05 * np.cos(2 * np.pi * z / 0.5) + 0 * r),
                       p=1.0 + 0.1 * g + 0 * z, T_ion=1.0 + 0 * r + 0 * z)
    S, O, d = _pair(orc, "axis_axisym", art=True, eos=two, ic=ic)
    it = _it(d)
    dQo = it(O.compute_rhs())
    dQ = it(S.compute_rhs())
    sc = O.rhs_scales(cl.grid_spacing(d))
    for c in range(dQo.shape[0]):
        ref = max(np.abs(dQo[c]).max(), sc[c])
        assert np.abs(dQ[c] - dQo[c]).max() <= 1e-12 * ref, c


@pytest.mark.parametrize("case", ["axis_resolved", "sphere"])
def test_mixed_precision_geometry(orc, case):
    S, O, d = _pair(orc, case, art=True, precision="mixed")
    it = _it(d)
    dQo = it(O.compute_rhs())
    dQ = it(S.compute_rhs())
    sc = O.rhs_scales(cl.grid_spacing(d))
    errs = []
    for c in range(dQo.shape[0]):
        diff, den = float(np.abs(dQ[c] - dQo[c]).max()), max(float(np.abs(dQo[c]).max()), sc[c])
        assert den > 0 or diff == 0, c      # a component that vanishes must vanish on the device too
        errs.append(diff / den if den > 0 else 0.0)
    # FP32 fields and line solves, amplified by the 1/r metric factors near the singular set
    assert max(errs) < 5e-5, errs
    # ten steps without artificial properties (well conditioned, see above)
    S, O, d = _pair(orc, case, art=False, precision="mixed")
    S.run(1e9, 10)
    O.run(1e9, 10)
    a, b = it(S.get_state()), it(O.get_state())
    rel = float(np.linalg.norm(a - b) / np.linalg.norm(b))
    assert rel <= 1e-5, rel


def test_graph_mode_geometry(orc):
    S, _, _ = _pair(orc, "axis_resolved", art=True)
    R, _, _ = _pair(orc, "axis_resolved", art=True)
    S.run(1e9, 12)
    R.run_graph(1e9, 12)
    assert np.array_equal(S.get_state(), R.get_state())
    assert S.t == R.t


def test_geometry_setup_errors():
    d = cl.solver_desc((16, 8, 1), (1.0, 1.0, 1.0), ((cl.AxisBC(), cl.SlipWallBC()), PER, PER),
                       cl.lele_d1_6(), cl.compact_filter(0.45))
    with pytest.raises(cl.ClesError, match="AxisBC requires CylindricalMetric"):
        cl.Solver(d)
    # a characteristic face needs a unit normal scale factor: not a theta face (src/nscbc.jl:309-323)
    d = cl.solver_desc((16, 16, 8), (1.0, 1.0, 1.0), (PER, (cl.NSCBCOutflowBC(pinf=1.0), cl.SlipWallBC()), PER),
                       cl.lele_d1_6(), cl.compact_filter(0.45), metric=cl.CylindricalMetric(), origin=(0.5, 0.0, 0.0))
    with pytest.raises(cl.ClesError, match="periodic radial|scale factor"):
        cl.Solver(d)
    d = cl.solver_desc((16, 16, 8), (1.0, 1.0, 1.0), ((cl.SlipWallBC(), cl.SlipWallBC()),
                                                      (cl.NSCBCOutflowBC(pinf=1.0), cl.SlipWallBC()), PER),
                       cl.lele_d1_6(), cl.compact_filter(0.45), metric=cl.CylindricalMetric(), origin=(0.5, 0.0, 0.0))
    with pytest.raises(cl.ClesError, match="scale factor is one"):
        cl.Solver(d)


@pytest.mark.parametrize("case", ["stretched", "annulus", "axis_axisym", "axis_resolved", "sphere"])
def test_dissipation_rate_matches_oracle(orc, case):
    # dissipation_rate (src/diagnostics.jl:354-378): J-weighted volume
    # integrals, unit quadrature weight on a folded edge
    S, O, d = _pair(orc, case, art=True)
    ds, do = S.dissipation_rate(), O.dissipation_rate()
    assert abs(ds - do) <= 1e-11 * abs(do)
