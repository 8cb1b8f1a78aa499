"""Graph-mode stepping and the continuous-batching server.

* run! as one CUDA-graph launch per step gives the same state as the
  host-stepped loop, bitwise in FP64 (same kernels, same order, the timestep
  and floors evaluated on the device with the same double arithmetic);
* every request served in a mix gives the same state as the same request run
  alone (bitwise in FP64): requests share no buffers and no reductions;
* admission respects the HBM budget, a failing request (negative density)
  fails alone, and queued requests can be cancelled.
"""
import numpy as np
import pytest

import compactles_b200 as cl
from compactles_b200 import scenarios

pytestmark = pytest.mark.gpu

SCH = None


def sch():
    global SCH
    if SCH is None:
        SCH = (cl.lele_d1_6(), cl.compact_filter(0.45))
    return SCH


def _alone(desc, Q0, tfinal, nmax, graph):
    s = cl.Solver(desc)
    s.set_state(Q0)
    res = (s.run_graph if graph else s.run)(tfinal, nmax)
    return s.get_state(), res


@pytest.mark.parametrize("case", ["tgv", "sod_like", "interface"])
def test_graph_mode_equals_host_loop(case):
    if case == "tgv":
        desc, Q0, tf = scenarios.taylor_green_box(sch(), 24)
        nmax = 15
    elif case == "sod_like":
        desc, Q0, tf = scenarios.two_species_tube(sch(), 300, 8.0, 0.4)
        nmax = 80
    else:
        desc, Q0, tf = scenarios.shock_interface_2d(sch(), 96, 32, 1.7, 3)
        nmax = 25
    a, ra = _alone(desc, Q0, tf, nmax, graph=True)
    b, rb = _alone(desc, Q0, tf, nmax, graph=False)
    assert ra.steps == rb.steps == nmax
    assert ra.t == rb.t
    assert np.array_equal(a, b)


def _mix():
    return [
        scenarios.two_species_tube(sch(), 256, 5.0, 0.3) + (60,),
        scenarios.two_species_tube(sch(), 700, 15.0, -0.5) + (60,),
        scenarios.shock_interface_2d(sch(), 80, 32, 2.0, 7) + (20,),
        scenarios.taylor_green_box(sch(), 16) + (12,),
        scenarios.two_species_tube(sch(), 400, 3.0, 0.7) + (10 ** 9,),   # runs to its end time
    ]


def test_server_mix_equals_alone():
    mix = _mix()
    srv = cl.Server(max_active=8)
    ids = [srv.submit(d, Q, tf, nmax) for d, Q, tf, nmax in mix]
    srv.drain()
    for rid, (d, Q, tf, nmax) in zip(ids, mix):
        st = srv.status(rid)
        assert st["state"] == "done", st
        got = srv.fetch(rid)
        want, res = _alone(d, Q, tf, nmax, graph=False)
        assert st["steps"] == res.steps
        assert np.array_equal(got, want)


def test_server_admits_within_hbm_budget():
    mix = _mix()[:3]
    # room for the largest request only: requests run one at a time
    srv = cl.Server(max_active=8)
    ids = [srv.submit(d, Q, tf, nmax) for d, Q, tf, nmax in mix]
    sizes = [srv.status(i)["device_bytes"] for i in ids]
    del srv
    srv = cl.Server(hbm_budget=max(sizes) + 1, max_active=8)
    ids = [srv.submit(d, Q, tf, nmax) for d, Q, tf, nmax in mix]
    max_running = 0
    while True:
        r, q = srv.tick()
        max_running = max(max_running, r)
        if r == 0 and q == 0:
            break
    assert max_running == 1
    for rid, (d, Q, tf, nmax) in zip(ids, mix):
        assert srv.status(rid)["state"] == "done"
        want, _ = _alone(d, Q, tf, nmax, graph=True)
        assert np.array_equal(srv.fetch(rid), want)
    with pytest.raises(cl.ClesError):
        cl.Server(hbm_budget=1024, max_active=2).submit(*mix[0][:3])


def test_failing_request_fails_alone():
    mix = _mix()[:3]
    bad_desc, bad_Q, bad_tf = scenarios.two_species_tube(sch(), 256, 5.0, 0.3)
    bad_Q = bad_Q.copy()
    bad_Q[0, 0, 0, 50] = -1.0     # negative partial density in one cell
    bad_Q[1, 0, 0, 50] = 0.0
    srv = cl.Server(max_active=8)
    ids = [srv.submit(d, Q, tf, nmax) for d, Q, tf, nmax in mix]
    bad = srv.submit(bad_desc, bad_Q, bad_tf, 100)
    srv.drain()
    st = srv.status(bad)
    assert st["state"] == "failed" and st["failure"] == "negative_density"
    with pytest.raises(cl.ClesError):
        srv.fetch(bad)
    for rid, (d, Q, tf, nmax) in zip(ids, mix):
        want, _ = _alone(d, Q, tf, nmax, graph=True)
        assert np.array_equal(srv.fetch(rid), want)


def test_cancel_queued_and_running():
    mix = _mix()[:3]
    srv = cl.Server(max_active=1)
    ids = [srv.submit(d, Q, tf, nmax) for d, Q, tf, nmax in mix]
    srv.tick()                       # admits the first
    srv.cancel(ids[2])               # still queued
    srv.cancel(ids[0])               # running
    srv.drain()
    assert srv.status(ids[0])["state"] == "cancelled"
    assert srv.status(ids[2])["state"] == "cancelled"
    assert srv.status(ids[1])["state"] == "done"


def test_server_curvilinear_request_owns_its_stretch():
    # The server creates a request's solver at admission: a stretched,
    # curvilinear request still matches the same solve run alone after the
    # caller's Stretch samples are gone.
    import gc
    PER = (cl.PeriodicBC(), cl.PeriodicBC())

    def make():
        d = cl.solver_desc((48, 16, 1), (1.0, 2 * np.pi, 1.0), ((cl.SlipWallBC(), cl.SlipWallBC()), PER, PER),
                           cl.lele_d1_6(), cl.compact_filter(0.45), metric=cl.CylindricalMetric(),
                           origin=(0.3, 0.0, 0.0), stretch=(cl.sine_cluster(0.3, 1.3, 0.5, 0.3), None, None))
        Q = cl.initialize(d, lambda r, t, z: cl.Prim(u=(0.0 * r, 0.2 * r + 0 * t, 0.0 * r),
                                                     p=1.0 + 0.1 * np.exp(-20 * (r - 0.8) ** 2) * np.cos(t),
                                                     rho=1.0 + 0 * r))
        return d, Q
    d, Q = make()
    S = cl.Solver(d)
    S.set_state(Q)
    S.run(1e9, 25)
    want = S.get_state()
    srv = cl.Server(max_active=2)
    blocker_d, blocker_Q = make()
    rid0 = srv.submit(blocker_d, blocker_Q, 1e9, 25)
    d2, Q2 = make()
    rid = srv.submit(d2, Q2, 1e9, 25)
    del d2._stretch_keep       # the descriptor's own samples go away before admission
    gc.collect()
    srv.drain()
    assert np.array_equal(srv.fetch(rid), want)
    assert np.array_equal(srv.fetch(rid0), want)
