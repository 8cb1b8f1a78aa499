"""Function-valued boundary faces on the device: DirichletBC(fun) and
NSCBCInflowBC(target=fun) evaluated at the RK stage times
(src/problem.jl:194-207, src/nscbc.jl:250-260).

* the Noh battery (test/validation.jl:217-233) in planar, cylindrical-axis
  and spherical-origin geometry meets the reference's bounds on the device,
  and 50 steps of each match the oracle to 1e-10;
* an oscillating piston (examples/piston_driver.jl) with an NSCBC outflow,
  and an NSCBC inflow with a pulsed target, match the oracle per RHS to
  1e-12 and over 40 steps to 1e-10;
* a face function that returns a constant gives the constant face bitwise;
* graph mode refuses a solver with a face function.
"""
import math

import numpy as np
import pytest

import compactles_b200 as cl
from compactles_b200 import noh

pytestmark = pytest.mark.gpu


def _state_close(a, b, tol):
    mom = math.sqrt(sum(np.linalg.norm(b[c]) ** 2 for c in (1, 2, 3)))
    for c in range(b.shape[0]):
        ref = mom if c in (1, 2, 3) else np.linalg.norm(b[c])
        assert np.linalg.norm(a[c] - b[c]) <= tol * ref, c


@pytest.mark.parametrize("nu", [1, 2, 3])
def test_noh_battery_on_device(nu):
    d, ic, tf = noh.noh_desc(cl, nu, (cl.lele_d1_6(), cl.compact_filter(0.45)))
    S = cl.Solver(d)
    S.set_state(cl.initialize(d, ic))
    S.run(tf, noh.NMAX)
    assert not S.face_errors and S.t >= tf * (1 - 1e-9)
    S.compute_rhs()
    sl = cl.interior_slices(d)
    rho = S.field(cl.abi.CLES_FIELD_RHO)[sl][0, 0]
    noh.check_noh(cl.coords(d)[0], rho, nu)


@pytest.mark.parametrize("nu", [1, 2, 3])
def test_noh_steps_match_oracle(orc, nu):
    dg, ic, _ = noh.noh_desc(cl, nu, (cl.lele_d1_6(), cl.compact_filter(0.45)))
    do, _, _ = noh.noh_desc(cl, nu, (orc.lele_d1_6(), orc.compact_filter(0.45)))
    Q0 = cl.initialize(dg, ic)
    S = cl.Solver(dg)
    S.set_state(Q0)
    O = orc.Solver(do)
    O.set_state(Q0)
    S.run(1e9, 50)
    assert O.run(1e9, 50)[0] == 0
    it = lambda A: A[(slice(None),) + cl.interior_slices(dg)]
    _state_close(it(S.get_state()), it(O.get_state()), 1e-10)


def _piston(sch, target=False):
    p0, r0, g = 1.0, 1.0, 1.4
    c0 = math.sqrt(g * p0 / r0)
    A, f = 0.2 * c0, 2.0
    PER = (cl.PeriodicBC(), cl.PeriodicBC())
    if target:
        # subsonic inflow relaxing toward a pulsed velocity and temperature
        lo = cl.NSCBCInflowBC(u=(0.3, 0.0, 0.0), T_ion=1.0,
                              target=lambda x, y, z, t: cl.Prim(u=(0.3 + 0.1 * np.sin(2 * np.pi * f * t) + 0 * y,
                                                                   0.02 * np.sin(2 * np.pi * y / 0.25), 0.0 * y),
                                                                T_ion=1.0 + 0.05 * np.cos(2 * np.pi * y / 0.25),
                                                                p=1.0 + 0 * y))
        ic = lambda x, y, z: cl.Prim(u=(0.3 + 0 * x, 0.0 * y, 0.0 * z), p=p0 + 0 * x, rho=r0 + 0 * x)
    else:
        # examples/piston_driver.jl: an oscillating full-state driver
        lo = cl.DirichletBC(lambda x, y, z, t: cl.Prim(u=(A * math.sin(2 * math.pi * f * t) + 0 * y, 0.0 * y, 0.0 * y),
                                                       p=p0 + 0 * y, rho=r0 + 0 * y))
        ic = lambda x, y, z: cl.Prim(u=(0.0 * x, 0.0 * y, 0.0 * z), p=p0 + 0 * x, rho=r0 + 0 * x)
    bcs = ((lo, cl.NSCBCOutflowBC(pinf=p0)), PER, PER)
    d = cl.solver_desc((96, 12, 1), (2.0, 0.25, 1.0), bcs, *sch, eos=cl.single_species(gamma=g),
                       art=cl.ArtParams(enabled=True), cfl=0.5)
    return d, ic


@pytest.mark.parametrize("target", [False, True])
def test_piston_and_inflow_target_match_oracle(orc, target):
    dg, ic = _piston((cl.lele_d1_6(), cl.compact_filter(0.45)), target)
    do, _ = _piston((orc.lele_d1_6(), orc.compact_filter(0.45)), target)
    Q0 = cl.initialize(dg, ic)
    S = cl.Solver(dg)
    S.set_state(Q0)
    O = orc.Solver(do)
    O.set_state(Q0)
    it = lambda A: A[(slice(None),) + cl.interior_slices(dg)]
    for s in (S, O):
        s.set_clock(0.13, 0, 0.5)   # a stage time where the functions are far from their t = 0 values
    S.apply_bcs()
    O.apply_bcs()
    dQo = it(O.compute_rhs())
    dQ = it(S.compute_rhs())
    sc = O.rhs_scales(cl.grid_spacing(dg))
    for c in range(dQo.shape[0]):
        ref = max(np.abs(dQo[c]).max(), sc[c])
        assert np.abs(dQ[c] - dQo[c]).max() <= 1e-12 * ref, c
    S.run(1e9, 40)
    assert O.run(1e9, 40)[0] == 0
    assert not S.face_errors and not O.face_errors
    _state_close(it(S.get_state()), it(O.get_state()), 1e-10)


def test_constant_function_face_is_the_constant_face():
    prim = cl.Prim(rho=1.2, u=(0.3, 0.0, 0.0), p=0.9)
    fun = lambda x, y, z, t: cl.Prim(rho=1.2 + 0 * x, u=(0.3 + 0 * x, 0.0, 0.0), p=0.9 + 0 * x)
    ic = lambda x, y, z: cl.Prim(rho=1.0 + 0.1 * np.cos(np.pi * x), u=(0.1 * np.sin(np.pi * x), 0.0 * y, 0.0 * z),
                                 p=1.0 + 0 * x)
    out = []
    for bc in (cl.DirichletBC(prim), cl.DirichletBC(fun)):
        d = cl.solver_desc((48, 12, 1), (1.0, 0.25, 1.0), ((bc, cl.SlipWallBC()), cl.PER3[1], cl.PER3[2]),
                           cl.lele_d1_6(), cl.compact_filter(0.45))
        S = cl.Solver(d)
        S.set_state(cl.initialize(d, ic))
        S.run(1e9, 15)
        out.append(S.get_state())
    assert np.array_equal(out[0], out[1])


def test_graph_mode_refuses_face_functions():
    d, ic = _piston((cl.lele_d1_6(), cl.compact_filter(0.45)))
    S = cl.Solver(d)
    S.set_state(cl.initialize(d, ic))
    with pytest.raises(cl.ClesError, match="graph mode"):
        S.run_graph(1e9, 3)
