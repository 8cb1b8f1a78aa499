"""Oracle pins for the curvilinear metrics, stretching and coordinate folds.

Each case is one of the reference's own known-answer tests
(test/runtests.jl:171-330) run through the oracle's restatement of
src/metric.jl, src/folds.jl and the fold-aware plans of src/operators.jl /
src/operators_banded.jl, with the reference's tolerances:

* C10 and C6 derivatives through an axis fold of odd and even fields;
* the resolved-theta axis (antipodal pairing, local);
* spherical origin + poles on a smooth Gaussian;
* rigid rotation in cylindrical coordinates has zero strain;
* a uniform state gives dQ ~ 0 in every metric, with stretching and folds.

Plus the setup-time errors of Solver(...) (src/rhs.jl:143-190).
"""
import math

import numpy as np
import pytest

import compactles_b200 as cl

PER = (cl.PeriodicBC(), cl.PeriodicBC())


def _solver(orc, n, L, bcs, metric=None, origin=(0.0, 0.0, 0.0), deriv=None, stretch=(None, None, None),
            art=False, mu0=0.0):
    d = cl.solver_desc(n, L, bcs, deriv or orc.lele_d1_6(), orc.compact_filter(0.45),
                       art=cl.ArtParams(enabled=art), origin=origin, metric=metric, stretch=stretch,
                       transport=cl.Transport(mu0=mu0))
    return orc.Solver(d), d


def _fill(S, d, fn):
    f = np.zeros(S.field_shape)
    x, y, z = cl.coords(d)
    f[cl.interior_slices(d)] = np.broadcast_to(fn(x[None, None, :], y[None, :, None], z[:, None, None]),
                                               (d.n_global[2], d.n_global[1], d.n_global[0]))
    return f


def _ferr(S, d, f, fn):
    x, y, z = cl.coords(d)
    want = np.broadcast_to(fn(x[None, None, :], y[None, :, None], z[:, None, None]),
                           (d.n_global[2], d.n_global[1], d.n_global[0]))
    return float(np.abs(f[cl.interior_slices(d)] - want).max())


def test_c10_through_axis_fold(orc):
    # test/runtests.jl:171-188
    S, d = _solver(orc, (64, 1, 12), (1.0, 1.0, 0.5), ((cl.AxisBC(), cl.SlipWallBC()), PER, PER),
                   metric=cl.CylindricalMetric(), deriv=orc.lele_d1_10())
    f = _fill(S, d, lambda r, t, z: r * np.exp(-4 * r ** 2))
    df = S.deriv(f, 1, -1)
    assert _ferr(S, d, df, lambda r, t, z: (1 - 8 * r ** 2) * np.exp(-4 * r ** 2)) < 5e-6
    f = _fill(S, d, lambda r, t, z: np.exp(-4 * r ** 2))
    df = S.deriv(f, 1, 1)
    assert _ferr(S, d, df, lambda r, t, z: -8 * r * np.exp(-4 * r ** 2)) < 2e-5


def test_axisymmetric_axis_manufactured(orc):
    # test/runtests.jl:231-248
    S, d = _solver(orc, (64, 1, 12), (1.0, 1.0, 0.5), ((cl.AxisBC(), cl.SlipWallBC()), PER, PER),
                   metric=cl.CylindricalMetric())
    h, shift, _ = S.spacing()
    assert h[0] == 1.0 / 63.5 and shift[0] == h[0] / 2
    f = _fill(S, d, lambda r, t, z: r * np.exp(-4 * r ** 2))
    df = S.deriv(f, 1, -1)
    assert _ferr(S, d, df, lambda r, t, z: (1 - 8 * r ** 2) * np.exp(-4 * r ** 2)) < 5e-6
    f = _fill(S, d, lambda r, t, z: np.exp(-4 * r ** 2))
    df = S.deriv(f, 1, 1)
    assert _ferr(S, d, df, lambda r, t, z: -8 * r * np.exp(-4 * r ** 2)) < 2e-5


def test_resolved_theta_axis_pairing(orc):
    # test/runtests.jl:250-267
    S, d = _solver(orc, (48, 16, 1), (1.0, 2 * math.pi, 1.0), ((cl.AxisBC(), cl.SlipWallBC()), PER, PER),
                   metric=cl.CylindricalMetric())
    f = _fill(S, d, lambda r, t, z: r * np.cos(t) * np.exp(-4 * r ** 2))
    df = S.deriv(f, 1, -1)
    assert _ferr(S, d, df, lambda r, t, z: np.cos(t) * (1 - 8 * r ** 2) * np.exp(-4 * r ** 2)) < 1e-5
    f = _fill(S, d, lambda r, t, z: np.exp(-4 * r ** 2) * (1 + 0.5 * np.cos(2 * t)))
    df = S.deriv(f, 1, 1)
    assert _ferr(S, d, df, lambda r, t, z: -8 * r * np.exp(-4 * r ** 2) * (1 + 0.5 * np.cos(2 * t))) < 1e-4


def test_spherical_origin_and_poles(orc):
    # test/runtests.jl:269-283
    S, d = _solver(orc, (40, 16, 12), (1.0, math.pi, 2 * math.pi),
                   ((cl.OriginBC(), cl.SlipWallBC()), (cl.PoleBC(), cl.PoleBC()), PER),
                   metric=cl.SphericalMetric())
    f = _fill(S, d, lambda r, t, p: np.exp(-4 * r ** 2))
    df = S.deriv(f, 1, 1)
    assert _ferr(S, d, df, lambda r, t, p: -8 * r * np.exp(-4 * r ** 2)) < 1e-4
    df = S.deriv(f, 2, 1)
    assert _ferr(S, d, df, lambda r, t, p: 0.0 * r) < 1e-8


def test_rigid_rotation_zero_strain(orc):
    # test/runtests.jl:285-303
    S, d = _solver(orc, (32, 16, 12), (1.0, 2 * math.pi, 0.5), ((cl.SlipWallBC(), cl.SlipWallBC()), PER, PER),
                   metric=cl.CylindricalMetric(), origin=(0.2, 0.0, 0.0))
    Q = cl.initialize(d, lambda r, t, z: cl.Prim(u=(0.0 * r, 0.3 * r, 0.0 * r), p=1.0 + 0 * r, rho=1.0 + 0 * r))
    S.set_state(Q)
    S.compute_rhs()
    sl = cl.interior_slices(d)
    g = [[S.field(cl.abi.CLES_FIELD_GRAD_U0 + 3 * a + b)[sl] for b in range(3)] for a in range(3)]
    smax = max(float(np.abs(0.5 * (g[a][b] + g[b][a])).max()) for a in range(3) for b in range(3))
    assert smax < 1e-8


FREESTREAM = [
    ("cartesian", (24, 12, 12), (1.0, 1.0, 1.0), None, cl.PER3, {}),
    ("stretched", (24, 12, 12), (1.0, 1.0, 1.0), None, ((cl.SlipWallBC(), cl.SlipWallBC()), PER, PER),
     {"stretch": (cl.sine_cluster(0.0, 1.0, 0.5, 0.4), None, None)}),
    ("cylindrical", (24, 12, 12), (1.0, 2 * math.pi, 0.5), cl.CylindricalMetric(),
     ((cl.SlipWallBC(), cl.SlipWallBC()), PER, PER), {"origin": (0.2, 0.0, 0.0)}),
    ("axisymmetric axis", (32, 1, 12), (1.0, 1.0, 0.5), cl.CylindricalMetric(),
     ((cl.AxisBC(), cl.SlipWallBC()), PER, PER), {}),
    ("resolved axis", (24, 16, 1), (1.0, 2 * math.pi, 1.0), cl.CylindricalMetric(),
     ((cl.AxisBC(), cl.SlipWallBC()), PER, PER), {}),
    ("spherical origin+poles", (24, 12, 12), (1.0, math.pi, 2 * math.pi), cl.SphericalMetric(),
     ((cl.OriginBC(), cl.SlipWallBC()), (cl.PoleBC(), cl.PoleBC()), PER), {}),
]


@pytest.mark.parametrize("case", FREESTREAM, ids=[c[0] for c in FREESTREAM])
def test_freestream_preservation(orc, case):
    # test/runtests.jl:305-330
    _, n, L, metric, bcs, kw = case
    S, d = _solver(orc, n, L, bcs, metric=metric, **kw)
    Q = cl.initialize(d, lambda x, y, z: cl.Prim(u=(0.0, 0.0, 0.0), p=1.0 + 0 * x, rho=1.0 + 0 * x))
    S.set_state(Q)
    S.apply_bcs()
    dQ = S.compute_rhs()
    assert np.abs(dQ[(slice(None),) + cl.interior_slices(d)]).max() < 1e-8


def test_stretched_geometry_and_derivative(orc):
    # A Stretch composes with the metric through the mapping Jacobian
    # (src/metric.jl:47-63, :109-140): 1/h_1 = 1/x'(xi), and the scaled
    # derivative is the physical one.
    st = cl.sine_cluster(0.0, 2.0, 0.3, 0.5)
    S, d = _solver(orc, (48, 12, 1), (1.0, 1.0, 1.0), ((cl.SlipWallBC(), cl.SlipWallBC()), PER, PER),
                   stretch=(st, None, None))
    h, _, _ = S.spacing()
    assert h[0] == 1.0 / 47
    xi = np.arange(48) * (1.0 / 47)
    sl = cl.interior_slices(d)
    ih = S.geometry("inv_h1")[sl]
    assert np.allclose(ih[0, 0, :], 1.0 / st.dxdxi(xi), rtol=1e-15)
    assert np.array_equal(cl.coords(d)[0], st.x(xi))
    f = _fill(S, d, lambda x, y, z: np.sin(2 * x) + 0 * y)
    df = S.deriv(f, 1, 1)
    # the one-sided closure rows are the least accurate on the mapped profile
    err = np.abs(df[sl][0, 0] - 2 * np.cos(2 * cl.coords(d)[0]))
    assert err.max() < 3e-3 and err[4:-4].max() < 5e-5


def test_spherical_gcl_cot_over_r(orc):
    # gcl_cotr! (src/metric.jl:154-170): cot(theta)/r is redefined as
    # inv_J D_theta(A_theta), O(h^4) from the analytic value
    S, d = _solver(orc, (24, 32, 1), (1.0, math.pi, 1.0), ((cl.OriginBC(), cl.SlipWallBC()),
                                                             (cl.PoleBC(), cl.PoleBC()), PER),
                   metric=cl.SphericalMetric())
    sl = cl.interior_slices(d)
    r, t, _ = cl.coords(d)
    ctr = S.geometry("cot_over_r")[sl][0]
    want = np.cos(t)[:, None] / (r[None, :] * np.sin(t)[:, None])
    assert np.abs(ctr - want).max() / np.abs(want).max() < 1e-3
    assert not np.array_equal(ctr, want)


@pytest.mark.parametrize("bad,msg", [
    (dict(n=(16, 1, 8), L=(1.0, 1.0, 1.0), bcs=((cl.AxisBC(), cl.SlipWallBC()), PER, PER), metric=None),
     "AxisBC requires CylindricalMetric"),
    (dict(n=(16, 1, 8), L=(1.0, 1.0, 1.0), bcs=((cl.AxisBC(), cl.SlipWallBC()), PER, PER),
          metric=cl.CylindricalMetric(), origin=(0.1, 0.0, 0.0)), "AxisBC requires origin"),
    (dict(n=(16, 7, 1), L=(1.0, 2 * math.pi, 1.0), bcs=((cl.AxisBC(), cl.SlipWallBC()), PER, PER),
          metric=cl.CylindricalMetric()), "even θ point count"),
    (dict(n=(16, 8, 1), L=(1.0, math.pi, 1.0), bcs=(PER, (cl.PoleBC(), cl.SlipWallBC()), PER),
          metric=cl.SphericalMetric()), "PoleBC must be applied at both ends"),
    (dict(n=(16, 8, 1), L=(1.0, 3.0, 1.0), bcs=(PER, (cl.PoleBC(), cl.PoleBC()), PER),
          metric=cl.SphericalMetric()), "PoleBC requires the θ domain"),
    (dict(n=(16, 8, 1), L=(1.0, 1.0, 1.0), bcs=(PER, PER, PER), stretch=(cl.sine_cluster(0, 1, 0.5, 0.2), None, None)),
     "stretched dimensions must be non-periodic"),
    (dict(n=(16, 1, 8), L=(1.0, 1.0, 1.0), bcs=((cl.AxisBC(), cl.SlipWallBC()), PER, PER),
          metric=cl.CylindricalMetric(), stretch=(cl.sine_cluster(0, 1, 0.5, 0.2), None, None)),
     "folded dimensions cannot be stretched"),
])
def test_setup_errors(orc, bad, msg):
    kw = dict(bad)
    n, L, bcs = kw.pop("n"), kw.pop("L"), kw.pop("bcs")
    with pytest.raises(ValueError, match=msg):
        _solver(orc, n, L, bcs, **kw)
