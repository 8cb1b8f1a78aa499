"""The host side of initialize! (conserved_from_prim, Prim) against the
reference's round-trip test (test/runtests.jl:1352-1389, the ideal-mixture
parts: StiffenedGas is outside this path), and the curvature term of the
oracle's max_rate (test/runtests.jl:641-665): swirl through a collapsed
angular dimension must shorten dt in cylindrical and spherical metrics;
and the oracle's volume quadrature, which the dissipation-rate diagnostic
rests on (test/runtests.jl:955-990)."""
import numpy as np
import pytest

import compactles_b200 as cl


def test_conserved_from_prim_round_trip():
    eos = cl.IdealMixture([cl.IdealSpecies("a", 1.0, 1.4), cl.IdealSpecies("b", 0.2, 1.09)])
    assert eos.nspecies == 2 and cl.single_species().nspecies == 1
    q = cl.conserved_from_prim(eos, cl.Prim(u=(0.3, -0.1, 0.2), p=0.8, T_ion=1.7, Y=(0.35, 0.65)))
    rho = q[0] + q[1]
    assert abs(q[0] / rho - 0.35) < 1e-12
    assert abs(q[2] / rho - 0.3) < 1e-12
    Rm = 0.35 * eos.Rk[0] + 0.65 * eos.Rk[1]
    assert abs(rho * Rm * 1.7 - 0.8) < 1e-12
    rho0 = 0.8 / (Rm * 1.7)
    for alt in (cl.Prim(u=(0.3, -0.1, 0.2), rho=rho0, T_ion=1.7, Y=(0.35, 0.65)),
                cl.Prim(u=(0.3, -0.1, 0.2), p=0.8, rho=rho0, Y=(0.35, 0.65))):
        got = cl.conserved_from_prim(eos, alt)
        assert np.allclose(got, q, rtol=1e-14, atol=0)
    ideal = cl.single_species(gamma=1.4, R=287.0)
    a = cl.conserved_from_prim(ideal, cl.Prim(rho=1000.0, T_ion=300.0))
    b = cl.conserved_from_prim(ideal, cl.Prim(p=1000.0 * 287.0 * 300.0, T_ion=300.0))
    assert np.allclose(a, b, rtol=1e-12, atol=0)
    for bad in ({"p": 1.0}, {"rho": 1.0}, {"p": 1.0, "rho": 1.0, "T_ion": 1.0}):
        with pytest.raises(ValueError):
            cl.Prim(**bad)


@pytest.mark.parametrize("metric", ["cylindrical", "spherical"])
def test_swirl_through_a_collapsed_angle_shortens_dt(orc, metric):
    m = cl.CylindricalMetric() if metric == "cylindrical" else cl.SphericalMetric()

    def rate(uang):
        d = cl.solver_desc((64, 1, 1), (1.0, 1.0, 1.0), ((cl.SlipWallBC(), cl.SlipWallBC()), cl.PER3[1], cl.PER3[2]),
                           orc.lele_d1_6(), orc.compact_filter(0.45), metric=m, origin=(0.5, np.pi / 2, 0.0),
                           art=cl.ArtParams(enabled=False))
        S = orc.Solver(d)
        S.set_state(cl.initialize(d, lambda r, t, p: cl.Prim(u=(0.0 * r, uang + 0 * r, uang + 0 * r), p=1.0 + 0 * r,
                                                              rho=1.0 + 0 * r)))
        return S.max_rate()[0]

    # dt = cfl / rate: a larger rate is a shorter step
    assert rate(2.0) > rate(0.0)


def test_cartesian_rate_has_no_curvature_term(orc):
    # the same swirl on a Cartesian grid changes only the advective part
    def rate(w):
        d = cl.solver_desc((64, 1, 1), (1.0, 1.0, 1.0), ((cl.SlipWallBC(), cl.SlipWallBC()), cl.PER3[1], cl.PER3[2]),
                           orc.lele_d1_6(), orc.compact_filter(0.45), art=cl.ArtParams(enabled=False))
        S = orc.Solver(d)
        S.set_state(cl.initialize(d, lambda x, y, z: cl.Prim(u=(0.0 * x, w + 0 * x, w + 0 * x), p=1.0 + 0 * x,
                                                              rho=1.0 + 0 * x)))
        return S.max_rate()[0]

    # collapsed y and z carry no advective rate either, so the swirl is invisible
    assert rate(2.0) == rate(0.0)


def test_volume_quadrature(orc):
    # test/runtests.jl:955-990: Cartesian exact (half weights on node-centred
    # walls), the cylindrical axis fold O(h^2) at the outer wall only
    PER, WALLS = cl.PER3[1], (cl.SlipWallBC(), cl.SlipWallBC())
    d = cl.solver_desc((24, 16, 12), (2.0, 1.0, 0.5), (WALLS, PER, PER), orc.lele_d1_6(), orc.compact_filter(0.45),
                       art=cl.ArtParams(enabled=False))
    S = orc.Solver(d)
    ones = np.ones(S.field_shape)
    assert abs(S.volume_integral(ones) - 1.0) < 1e-12
    lin = np.zeros(S.field_shape)
    x = cl.coords(d)[0]
    lin[cl.interior_slices(d)] = x[None, None, :]
    assert abs(S.volume_integral(lin) - 1.0) < 1e-12
    dc = cl.solver_desc((64, 1, 12), (1.0, 1.0, 1.0), ((cl.AxisBC(), cl.SlipWallBC()), PER, PER), orc.lele_d1_6(),
                        orc.compact_filter(0.45), metric=cl.CylindricalMetric(), art=cl.ArtParams(enabled=False))
    Sc = orc.Solver(dc)
    v = Sc.volume_integral(np.ones(Sc.field_shape))
    h = cl.grid_spacing(dc)[0]
    assert abs(v - 0.5) <= 1e-3 * 0.5
    assert v - 0.5 < h * h


def test_slip_wall_box_has_no_flow_through_its_walls():
    """The closed-line benchmark box: every face a slip wall, and the field's
    momentum normal to each face zero on that face."""
    n = 24
    desc, Q0, _ = cl.scenarios.slip_wall_box((cl.lele_d1_6(), cl.compact_filter(0.45)), n)
    assert tuple(desc.n_global) == (n, n, n)
    Qi = Q0[(slice(None),) + cl.interior_slices(desc)]      # [comp][z][y][x]
    assert Qi.shape == (5, n, n, n)
    scale = np.abs(Qi[1:4]).max()
    assert scale > 0.5
    for comp, axis in ((1, 3), (2, 2), (3, 1)):             # rho u on x faces, rho v on y, rho w on z
        for end in (0, n - 1):
            face = np.take(Qi[comp], end, axis=axis - 1)
            assert np.abs(face).max() <= 1e-12 * scale
    assert np.allclose(Qi[0], 1.0)
