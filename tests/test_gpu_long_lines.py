"""Few long closed x lines, cut into pieces solved side by side on the device
(SigPlan: the reference's P > 1 line solve, src/tridiag.jl:136-170 and
src/banded.jl:177-214, with the pieces of one line in place of ranks).

The 1-D two-species shock tubes of the serving mix reach 8192 cells: one line
per field.  Their right-hand side and steps of run! are compared with the CPU
oracle (its single-rank Thomas solve) at lengths where the pieced form is
used: FP64 per RHS within 1e-12 of the term scale and within 1e-10 relative
L2 after 30 steps (host-stepped and graph mode), the mixed form within 1e-5;
the C10 scheme and a thin 2-D grid of 3 long lines; and lengths on either
side of the threshold (2047 and 2048 cells)."""
import numpy as np
import pytest

import compactles_b200 as cl
import parity
from compactles_b200 import scenarios

pytestmark = pytest.mark.gpu


def _it(desc):
    sl = (slice(None),) + cl.interior_slices(desc)
    return lambda A: A[sl]


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _tube(m, N, precision="fp64", deriv=None):
    sch = (deriv if deriv is not None else m.lele_d1_6(), m.compact_filter(0.45))
    return scenarios.two_species_tube(sch, N, 10.0, 0.5, precision=precision)


@pytest.mark.parametrize("N", [2047, 2048, 4096, 8192])
def test_tube_rhs_and_steps(orc, N):
    dg, Q0, tf = _tube(cl, N)
    do, _, _ = _tube(orc, N)
    it = _it(dg)
    S = cl.Solver(dg)
    O = orc.Solver(do)
    S.set_state(Q0)
    O.set_state(Q0)
    b = O.compute_rhs()
    a = S.compute_rhs()
    plain, term = parity.rhs_errors(it(a), it(b), O.rhs_scales(cl.grid_spacing(dg)))
    parity.record(f"tube N={N} FP64 RHS", plain, term)
    assert max(term) < 1e-12, (plain, term)
    S.set_state(Q0)
    O.set_state(Q0)
    S.run(tf, 30)
    assert O.run(tf, 30)[0] == 0
    rel = _rel(it(S.get_state()), it(O.get_state()))
    # the same history as S (a right-hand side first: max_rate's first step
    # reads the artificial properties it left)
    G = cl.Solver(dg)
    G.set_state(Q0)
    G.compute_rhs()
    G.set_state(Q0)
    G.run_graph(tf, 30)
    relg = _rel(it(G.get_state()), it(O.get_state()))
    parity.record(f"tube N={N} FP64 30 steps", state_l2=rel, graph_l2=relg)
    assert rel < 1e-10 and relg < 1e-10, (rel, relg)


def test_tube_c10_and_mixed(orc):
    dg, Q0, tf = _tube(cl, 5000, deriv=cl.lele_d1_10())
    do, _, _ = _tube(orc, 5000, deriv=orc.lele_d1_10())
    it = _it(dg)
    S, O = cl.Solver(dg), orc.Solver(do)
    S.set_state(Q0)
    O.set_state(Q0)
    S.run(tf, 20)
    assert O.run(tf, 20)[0] == 0
    rel = _rel(it(S.get_state()), it(O.get_state()))
    parity.record("tube N=5000 C10 FP64 20 steps", state_l2=rel)
    assert rel < 1e-10, rel
    dm, Qm, tfm = _tube(cl, 6000, precision="mixed")
    do, _, _ = _tube(orc, 6000)
    S, O = cl.Solver(dm), orc.Solver(do)
    S.set_state(Qm)
    O.set_state(Qm)
    S.run(tfm, 20)
    assert O.run(tfm, 20)[0] == 0
    rel = _rel(_it(dm)(S.get_state()), _it(dm)(O.get_state()))
    parity.record("tube N=6000 mixed 20 steps", state_l2=rel)
    assert rel < 1e-5, rel


def test_thin_grid_of_three_long_lines(orc):
    """apply_along! on a 3000 x 3 grid (three closed x lines, padded layout), every scheme."""
    ng, per = (3000, 3, 1), (0, 1, 1)
    g = orc.grid(ng, per)
    rng = np.random.default_rng(5)
    f = np.zeros(orc.padded_shape(g))
    inner = orc.interior(g, f)
    x = np.arange(ng[0])[None, None, :]
    inner[...] = np.sin(0.01 * x + rng.uniform(0, 6, size=(1, 3, 1))) + 0.1 * rng.standard_normal(inner.shape)
    orc.exchange_halos(g, f)
    for name in ("lele_d1_6", "compact_filter", "lele_d1_10"):
        so = orc.compact_filter(0.45) if name == "compact_filter" else getattr(orc, name)()
        sg = cl.compact_filter(0.45) if name == "compact_filter" else getattr(cl, name)()
        ref = orc.interior(g, orc.Plan(g, so, 1, 0.01).apply(f))
        out = np.zeros_like(f)
        cl.apply_along(out, cl.plan_direction(cl.grid(ng, per), sg, 1, 0.01), f)
        err = np.abs(orc.interior(g, out) - ref).max() / np.abs(ref).max()
        parity.record(f"3000 x 3 {name} apply_along", rel=err)
        assert err < 1e-12, (name, err)
