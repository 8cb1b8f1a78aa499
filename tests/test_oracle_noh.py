"""Oracle pin: the reference's Noh validation battery (test/validation.jl:
217-233) in planar, cylindrical-axis and spherical-origin geometry, with the
exact time-dependent inflow as a DirichletBC(fun) evaluated at the stage
times (test/cases.jl:186-236).  The oracle must meet the reference's bounds
on the plateau, the wall heating, the shock radius and the pre-shock error.
"""
import numpy as np
import pytest

import compactles_b200 as cl
from compactles_b200 import noh


@pytest.mark.parametrize("nu", [1, 2, 3])
def test_noh_battery(orc, nu):
    d, ic, tf = noh.noh_desc(cl, nu, (orc.lele_d1_6(), orc.compact_filter(0.45)))
    O = orc.Solver(d)
    O.set_state(cl.initialize(d, ic))
    rc, res = O.run(tf, noh.NMAX)
    assert rc == 0 and not O.face_errors
    assert res.t >= tf * (1 - 1e-9)
    O.compute_rhs()   # refresh the primitives of the final state
    sl = cl.interior_slices(d)
    xs = cl.coords(d)[0]
    rho = O.field(cl.abi.CLES_FIELD_RHO)[sl][0, 0]
    plat, deficit, Rnum, epre = noh.check_noh(xs, rho, nu)
    print(f"nu={nu} plateau {plat:.4f} (exact {4.0 ** nu}) deficit {deficit:+.3f} shock {Rnum:.4f} L1 {epre:.2e}")


def test_face_function_dirichlet_matches_constant(orc):
    # a function that returns a constant Prim gives the constant-state face bitwise
    sch = (orc.lele_d1_6(), orc.compact_filter(0.45))
    prim = cl.Prim(rho=1.2, u=(0.3, 0.0, 0.0), p=0.9)
    bcs_c = ((cl.DirichletBC(prim), cl.SlipWallBC()), cl.PER3[1], cl.PER3[2])
    bcs_f = ((cl.DirichletBC(lambda x, y, z, t: cl.Prim(rho=1.2 + 0 * x, u=(0.3 + 0 * x, 0.0, 0.0), p=0.9 + 0 * x)),
              cl.SlipWallBC()), cl.PER3[1], cl.PER3[2])
    ic = lambda x, y, z: cl.Prim(rho=1.0 + 0.1 * np.cos(np.pi * x), u=(0.1 * np.sin(np.pi * x), 0.0 * y, 0.0 * z),
                                 p=1.0 + 0 * x)
    out = []
    for bcs in (bcs_c, bcs_f):
        d = cl.solver_desc((48, 12, 1), (1.0, 0.25, 1.0), bcs, *sch, art=cl.ArtParams(enabled=True))
        O = orc.Solver(d)
        O.set_state(cl.initialize(d, ic))
        assert O.run(1e9, 15)[0] == 0
        out.append(O.get_state())
    assert np.array_equal(out[0], out[1])
