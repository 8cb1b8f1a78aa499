"""GPU parity of the solver at the sizes the benchmark runs, against the CPU
oracle on identical inputs (the Taylor-Green box of the README quick-start:
rho 1, p 71.43, u = (sin x cos y, -cos x sin y, 0), default numerics).

At 128^3 and 256^3 the step uses kernels that smaller boxes do not reach: the
warp-per-line x kernel (periodic n = 128/256/512) in its subtract-accumulate
flux-divergence store, and the TMA tile kernel with the LSRK stage update
fused into its store at n = 256.  The 64^3 box is the quick-start
configuration itself: its right-hand side is compared at steps 0, 1, 10 and
100 (device and oracle fed the oracle's state at that step), the two
independent 100-step runs are compared in relative L2, and the whole run to
t = 1 (the configuration's end time) is compared in relative L2 and kinetic
energy.

Bounds: per RHS, 1e-12 of each component's term scale (tests/parity.py says
why; the plain relative error is recorded beside it); relative L2 of the state
1e-10 after 10 and 100 steps.  The mixed form (FP32 fields and line solves,
FP64 state and RK update) is held to 2e-6 of the term scale per RHS and to
1e-5 relative L2 of the state after 100 steps (FP32 rounding of the terms,
about 1e-7 of their size, accumulated over 100 updates of size dt * dQ).
"""
import numpy as np
import pytest

import cases
import compactles_b200 as cl
import parity

pytestmark = pytest.mark.gpu


def _descs(orc, n, precision="fp64"):
    dg, Q0, _ = cases.taylor_green((cl.lele_d1_6(), cl.compact_filter(0.45)), n=n, precision=precision)
    do, _, _ = cases.taylor_green((orc.lele_d1_6(), orc.compact_filter(0.45)), n=n)
    return dg, do, Q0


def _interior(desc):
    sl = (slice(None),) + cl.interior_slices(desc)
    return lambda A: A[sl]


def _rhs_pair(S, O, Q, it, h):
    S.set_state(Q)
    O.set_state(Q)
    b = O.compute_rhs()
    a = S.compute_rhs()
    return parity.rhs_errors(it(a), it(b), O.rhs_scales(h))


def _rel_l2(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("n", [128, 256])
def test_tgv_rhs_parity_bench_sizes(orc, n):
    dg, do, Q0 = _descs(orc, n)
    plain, term = _rhs_pair(cl.Solver(dg), orc.Solver(do), Q0, _interior(dg), cl.grid_spacing(dg))
    parity.record(f"TGV {n}^3 FP64 RHS", plain, term)
    assert max(term) < 1e-12, (plain, term)


def test_tgv_rhs_parity_mixed_256(orc):
    dg, do, Q0 = _descs(orc, 256, precision="mixed")
    plain, term = _rhs_pair(cl.Solver(dg), orc.Solver(do), Q0, _interior(dg), cl.grid_spacing(dg))
    parity.record("TGV 256^3 mixed RHS", plain, term)
    assert max(term) < 2e-6, (plain, term)


@pytest.mark.parametrize("n,steps", [(128, 10), (256, 2)])
def test_tgv_steps_bench_sizes(orc, n, steps):
    dg, do, Q0 = _descs(orc, n)
    S = cl.Solver(dg)
    S.set_state(Q0)
    O = orc.Solver(do)
    O.set_state(Q0)
    rg = S.run(1e9, steps)
    rc, ro = O.run(1e9, steps)
    assert rc == 0 and rg.steps == ro.steps == steps
    assert abs(rg.t - ro.t) <= 1e-12 * ro.t
    it = _interior(dg)
    rel = _rel_l2(it(S.get_state()), it(O.get_state()))
    parity.record(f"TGV {n}^3 FP64 {steps} steps", l2=rel)
    assert rel < 1e-10, rel


def test_quickstart_tgv64(orc):
    """The 64^3 quick-start box: RHS at steps 0, 1, 10, 100 and the 100-step state."""
    dg, do, Q0 = _descs(orc, 64)
    it = _interior(dg)
    h = cl.grid_spacing(dg)
    S = cl.Solver(dg)
    S.set_state(Q0)
    O = orc.Solver(do)
    O.set_state(Q0)
    probe_g, probe_o = cl.Solver(dg), orc.Solver(do)
    worst = 0.0
    for k in (0, 1, 10, 100):
        if k:
            rg = S.run(1e9, k)
            rc, ro = O.run(1e9, k)
            assert rc == 0 and S.steps == k and O.clock()[1] == k
            assert abs(S.t - O.clock()[0]) <= 1e-12 * O.clock()[0]
        Qo = O.get_state()
        plain, term = _rhs_pair(probe_g, probe_o, Qo, it, h)
        rel = _rel_l2(it(S.get_state()), it(Qo))
        parity.record(f"TGV 64^3 FP64 step {k} RHS", plain, term, state_l2=rel)
        assert max(term) < 1e-12, (k, plain, term)
        worst = max(worst, rel)
    assert worst < 1e-10, worst


def test_quickstart_tgv64_mixed(orc):
    """The mixed form against the FP64 oracle over 100 steps of the 64^3 box."""
    dg, do, Q0 = _descs(orc, 64, precision="mixed")
    S = cl.Solver(dg)
    S.set_state(Q0)
    O = orc.Solver(do)
    O.set_state(Q0)
    S.run(1e9, 100)
    rc, _ = O.run(1e9, 100)
    assert rc == 0 and S.steps == 100
    it = _interior(dg)
    rel = _rel_l2(it(S.get_state()), it(O.get_state()))
    ke_g, ke_o = S.kinetic_energy(), O.kinetic_energy()
    dt_rel = abs(S.t - O.clock()[0]) / O.clock()[0]
    parity.record("TGV 64^3 mixed vs FP64 oracle, 100 steps", state_l2=rel, ke_rel=abs(ke_g - ke_o) / ke_o,
                  t_rel=dt_rel)
    assert rel < 1e-5, rel
    assert abs(ke_g - ke_o) <= 1e-6 * ke_o


def test_quickstart_tgv64_to_t1(orc):
    """The quick-start configuration as the reference runs it: the 64^3 box to t = 1."""
    dg, do, Q0 = _descs(orc, 64)
    S = cl.Solver(dg)
    S.set_state(Q0)
    O = orc.Solver(do)
    O.set_state(Q0)
    rg = S.run(1.0)
    rc, ro = O.run(1.0)
    assert rc == 0 and rg.steps == ro.steps and abs(rg.t - 1.0) < 1e-12 and abs(ro.t - 1.0) < 1e-12
    it = _interior(dg)
    rel = _rel_l2(it(S.get_state()), it(O.get_state()))
    ke_g, ke_o = S.kinetic_energy(), O.kinetic_energy()
    parity.record(f"TGV 64^3 FP64 to t = 1 ({ro.steps} steps)", state_l2=rel, ke_rel=abs(ke_g - ke_o) / ke_o)
    assert rel < 1e-10, rel
    assert abs(ke_g - ke_o) <= 1e-12 * ke_o
