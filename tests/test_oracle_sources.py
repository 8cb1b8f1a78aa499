"""Oracle pin for the source terms (src/sources.jl): the reference's own
known answer, test/runtests.jl:374-388 -- a uniform state under
ConstantBodyForce((1, 2, -3)) gets dQ momentum = rho g and energy = rho u . g.
"""
import numpy as np

import compactles_b200 as cl


def _uniform_case(lib, forces):
    d = cl.solver_desc((12, 12, 12), (2 * np.pi,) * 3, cl.PER3, lib.lele_d1_6(), lib.compact_filter(0.45),
                       art=cl.ArtParams(enabled=False), sources=forces)
    Q = cl.initialize(d, lambda x, y, z: cl.Prim(u=(0.5 + 0 * x, 0.25 + 0 * y, -0.1 + 0 * z), p=1.0 + 0 * x,
                                                 rho=2.0 + 0 * x))
    return d, Q


def test_body_force_known_answer(orc):
    d, Q = _uniform_case(orc, (cl.ConstantBodyForce((1.0, 2.0, -3.0)),))
    O = orc.Solver(d)
    O.set_state(Q)
    dQ = O.compute_rhs()[(slice(None),) + cl.interior_slices(d)]
    assert np.allclose(dQ[1], 2.0, atol=1e-10) and np.allclose(dQ[2], 4.0, atol=1e-10)
    assert np.allclose(dQ[3], -6.0, atol=1e-10) and np.allclose(dQ[4], 2.6, atol=1e-10)


def test_two_forces_add(orc):
    d, Q = _uniform_case(orc, (cl.ConstantBodyForce((1.0, 0.0, 0.0)), cl.ConstantBodyForce((0.0, 2.0, -3.0))))
    O = orc.Solver(d)
    O.set_state(Q)
    dQ = O.compute_rhs()[(slice(None),) + cl.interior_slices(d)]
    assert np.allclose(dQ[1:5].reshape(4, -1).mean(axis=1), (2.0, 4.0, -6.0, 2.6), atol=1e-10)
