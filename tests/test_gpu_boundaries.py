"""Device parity of the boundary conditions beyond periodic / slip wall:
NoSlipWallBC, ExtrapolationBC, NSCBC outflow and inflow, SwitchableBC.

* enforcement (apply_bcs) equals the oracle's to a few ulp (the device
  contracts products and sums into FMAs);
* the RHS with characteristic faces matches the oracle per component to 1e-12
  of the component's RHS scale, and 20 steps to 1e-10 in relative L2
  (momentum components against the momentum vector);
* the measured shock/interface case with the switching upstream face meets
  the reference's bounds on the device too, and the switched face forwards to
  its `after` condition exactly.
"""
import math

import numpy as np
import pytest

import compactles_b200 as cl
import test_oracle_boundaries as ob

pytestmark = pytest.mark.gpu

PER = (cl.PeriodicBC(), cl.PeriodicBC())


def _pair(orc, n, L, bcs, ic, eos=None, art=False, cfl=0.5):
    eos = eos or cl.single_species()

    def mk(sch):
        return cl.solver_desc(n, L, bcs, *sch, eos=eos, art=cl.ArtParams(enabled=art), cfl=cfl)
    dg = mk((cl.lele_d1_6(), cl.compact_filter(0.45)))
    do = mk((orc.lele_d1_6(), orc.compact_filter(0.45)))
    Q0 = cl.initialize(dg, ic, eos=eos)
    S = cl.Solver(dg)
    S.set_state(Q0)
    O = orc.Solver(do)
    O.set_state(Q0)
    return S, O, dg


def _it(d):
    sl = cl.interior_slices(d)
    return lambda A: A[(slice(None),) + sl]


@pytest.mark.parametrize("bc", ["noslip_adiabatic", "noslip_iso", "extrapolation"])
def test_enforcement_matches_oracle(orc, bc):
    face = {"noslip_adiabatic": cl.NoSlipWallBC(), "noslip_iso": cl.NoSlipWallBC(Twall=2.5),
            "extrapolation": cl.ExtrapolationBC()}[bc]
    two = cl.IdealMixture([cl.IdealSpecies("a", 1.0, 1.4), cl.IdealSpecies("b", 0.4, 1.6)])
    S, O, d = _pair(orc, (24, 12, 10), (1.0, 0.4, 0.4), ((face, face), PER, PER),
                    lambda x, y, z: cl.Prim(Y=(0.3 + 0.4 * x, 0.7 - 0.4 * x), u=(0.3 + x, -0.2 * np.cos(y), 0.1 + 0 * z),
                                            p=1.0 + 0.2 * x, T_ion=1.0 + 0.1 * np.sin(z)), eos=two)
    S.apply_bcs()
    O.apply_bcs()
    it = _it(d)
    assert np.allclose(it(S.get_state()), it(O.get_state()), rtol=1e-14, atol=0)


def _nscbc_case(case):
    two = cl.IdealMixture([cl.IdealSpecies("a", 1.0, 1.4), cl.IdealSpecies("b", 0.25, 1.4)])
    bcs = ((cl.NSCBCInflowBC(u=(0.4, 0.05, 0.0), T_ion=1.1, Y=(0.8, 0.2)), cl.NSCBCOutflowBC(pinf=1.0, sigma=0.3)),
           PER, PER)

    def ic(x, y, z):
        return cl.Prim(Y=(0.5 + 0.3 * np.cos(3 * x), 0.5 - 0.3 * np.cos(3 * x)),
                       u=(0.3 + 0.1 * np.sin(2 * np.pi * y), 0.05 * np.cos(4 * x), 0 * x + 0 * z),
                       p=1.0 + 0.1 * np.exp(-30 * (x - 0.7) ** 2), T_ion=1.0 + 0.05 * x)
    n, L = ((48, 16, 1), (1.0, 0.5, 0.5)) if case == "2d" else ((24, 12, 10), (1.0, 0.5, 0.4))
    return n, L, bcs, ic, two


@pytest.mark.parametrize("case", ["2d", "3d"])
@pytest.mark.parametrize("art", [False, True])
def test_nscbc_rhs_and_steps_match_oracle(orc, case, art):
    n, L, bcs, ic, eos = _nscbc_case(case)
    S, O, d = _pair(orc, n, L, bcs, ic, eos=eos, art=art)
    it = _it(d)
    S.apply_bcs()
    O.apply_bcs()
    dQo = it(O.compute_rhs())
    dQ = it(S.compute_rhs())
    sc = O.rhs_scales(cl.grid_spacing(d))
    for c in range(dQo.shape[0]):
        ref = max(np.abs(dQo[c]).max(), sc[c])
        assert np.abs(dQ[c] - dQo[c]).max() <= 1e-12 * ref, c
    S.run(1e9, 20)
    rc, _ = O.run(1e9, 20)
    assert rc == 0
    a, b = it(S.get_state()), it(O.get_state())
    mom = math.sqrt(sum(np.linalg.norm(b[c]) ** 2 for c in (2, 3, 4)))
    for c in range(b.shape[0]):
        ref = mom if c in (2, 3, 4) else np.linalg.norm(b[c])
        assert np.linalg.norm(a[c] - b[c]) <= 1e-10 * ref, c


def test_switchable_on_device():
    def mk(xbc):
        d = cl.solver_desc((16, 12, 12), (1.0, 1.0, 1.0), (xbc, PER, PER), cl.lele_d1_6(), cl.compact_filter(0.45),
                           art=cl.ArtParams(enabled=False), cfl=0.4)
        S = cl.Solver(d)
        S.set_state(cl.initialize(d, lambda x, y, z: cl.Prim(u=(0.2 + 0 * x, 0.0, 0.0),
                                                             p=1 + 0.1 * np.exp(-40 * (x - 0.5) ** 2),
                                                             rho=1.0 + 0 * x)))
        return S
    ref = mk((cl.SlipWallBC(), cl.SlipWallBC()))
    ref.run(1e9, 12)
    sw = (cl.SwitchableBC(cl.SlipWallBC(), cl.ExtrapolationBC()), cl.SwitchableBC(cl.SlipWallBC(), cl.ExtrapolationBC()))
    wrap = mk(sw)
    wrap.run(1e9, 12)
    assert np.array_equal(wrap.get_state(), ref.get_state())
    assert not wrap.switched(1, 1)
    s2 = mk(sw)
    s2.run(1e9, 4)
    s2.switch_bc(1, 1)
    s2.switch_bc(1, 2)
    assert s2.switched(1, 1) and s2.switched(1, 2)
    s2.run(1e9, 12)
    assert not np.array_equal(s2.get_state(), ref.get_state())
    with pytest.raises(cl.ClesError):
        ref.switch_bc(1, 1)


def test_switching_case_on_device():
    schemes = (cl.lele_d1_6(), cl.compact_filter(0.45))
    m = ob.switching_case(cl.Solver, schemes)
    ob.check_switching(m)
    s_sw = m["s_sw"]
    s_p, _ = ob.build_case(cl.Solver, schemes, (ob.outflow(), ob.downstream()))
    s_p.set_state(s_sw.get_state())
    s_p.set_clock(*s_sw.clock())
    s_sw.apply_bcs()
    s_p.apply_bcs()
    assert np.array_equal(s_sw.get_state(), s_p.get_state())
    a, b = s_sw.compute_rhs(), s_p.compute_rhs()
    assert np.abs(a).max() > 1
    assert np.array_equal(a, b)
