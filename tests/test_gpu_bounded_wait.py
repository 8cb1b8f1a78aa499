"""The expiry path of the compact kernels' bounded device wait.

Every mbarrier wait in the TMA tile kernels gives up after 2 s, counts the
expiry on the device and returns; the host turns the count into
CLES_ETIMEOUT.  cles_selftest_bounded_wait runs that path with a short limit
on an mbarrier that nothing completes (no copy is in flight), so no GPU is
faulted or held: the call must return CLES_ETIMEOUT, clear the count, and
leave the context usable for the next operator call and run! step."""
import ctypes as C

import numpy as np
import pytest

import compactles_b200 as cl
from compactles_b200 import abi

pytestmark = pytest.mark.gpu


def test_bounded_wait_expiry_returns_etimeout_and_context_survives():
    L = cl.lib()
    ctx = cl.Context(0)
    rc = L.cles_selftest_bounded_wait(ctx.ptr, C.c_int64(1_000_000))   # 1 ms
    assert rc == abi.CLES_ETIMEOUT, rc
    assert "bounded device wait" in L.cles_last_error().decode()
    # the same path a second time: the count was cleared and is set again
    assert L.cles_selftest_bounded_wait(ctx.ptr, C.c_int64(1_000_000)) == abi.CLES_ETIMEOUT
    # out-of-range limits are refused before any launch
    assert L.cles_selftest_bounded_wait(ctx.ptr, C.c_int64(10)) == abi.CLES_EINVAL
    # the context still runs operators, and a run! step reads a clear count
    n = 64
    g = cl.grid((n, n, n), (True, True, True))
    plan = cl.DirPlan(g, cl.lele_d1_6(), 2, 2 * np.pi / n, ctx=ctx)
    f = np.random.default_rng(1).standard_normal(plan.shape())
    out = np.zeros_like(f)
    cl.apply_along(out, plan, f)
    assert np.isfinite(out).all() and np.abs(out).max() > 0
    prob = cl.taylor_green_problem()
    d = cl.solver_desc((32, 32, 32), (2 * np.pi,) * 3, prob.bcs, cl.lele_d1_6(), cl.compact_filter(0.45))
    S = cl.Solver(d, ctx=ctx)
    S.set_state(cl.initialize(d, prob.ic))
    assert S.run(1e9, 2).steps == 2
