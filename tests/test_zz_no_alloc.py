"""cles_max_rate_static, the allocation-free CFL rate reduction, against
cles_max_rate.

The static entry point exists for callers that cannot allocate device memory
(a host framework that owns every allocation, a plugin barred from
allocating after start-up, a fixed HBM budget): it takes only caller-owned
device arrays and keeps its scratch in a library-owned static device array.
This test calls it through the C ABI twice in a row, on two different grids
so that the second call reads fewer partials than the first left behind, and
compares each result with cles_max_rate on the same state to 1e-14 relative
(the per-cell arithmetic is the same, and max/min reductions are exact).  The
test allocates its own device buffers (it is not such a caller).

This file sorts last so that a run stopping at the first failure has already
run every other test; it also passes on its own in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

import cases
import compactles_b200 as cl
from compactles_b200 import abi

pytestmark = pytest.mark.gpu


def _static_rate(torch, solver, desc, stream):
    info = solver.info()
    cells = info.cells
    ns = desc.n_species
    # the solver's conserved state (device, interior layout) and its artificial
    # properties, copied into a caller-owned device block
    Qp = C.POINTER(C.c_double)()
    cl.api._check(cl.lib().cles_state_device(solver.ptr, C.byref(Qp)))
    art = [solver.field(abi.CLES_FIELD_MU_ART, layout="interior"),
           solver.field(abi.CLES_FIELD_BETA_ART, layout="interior"),
           solver.field(abi.CLES_FIELD_KAPPA_ART, layout="interior")]
    art += [solver.field(abi.CLES_FIELD_D_ART0 + k, layout="interior") for k in range(ns)]
    art_dev = torch.tensor(np.stack(art), dtype=torch.float64, device="cuda").contiguous()
    out = torch.full((2,), float("nan"), dtype=torch.float64, device="cuda")
    R = (C.c_double * ns)(*[desc.R[k] for k in range(ns)])
    g = (C.c_double * ns)(*[desc.gamma[k] for k in range(ns)])
    h = cl.grid_spacing(desc)
    inv_h = (C.c_double * 3)(*[1.0 / h[d] if desc.n_global[d] > 1 else 0.0 for d in range(3)])
    torch.cuda.synchronize()
    rc = cl.lib().cles_max_rate_static(C.cast(Qp, C.c_void_p), C.c_void_p(art_dev.data_ptr()), cells, ns, R, g,
                                       inv_h, desc.mu0, desc.Pr, desc.Sc, C.c_void_p(out.data_ptr()),
                                       C.c_void_p(stream))
    cl.api._check(rc)
    torch.cuda.synchronize()
    return out.cpu().numpy()


def _prepared_solver(desc, Q0):
    s = cl.Solver(desc)
    s.set_state(Q0)
    s.compute_rhs()       # fills the artificial properties
    s.run(1e9, 2)         # and moves the state on
    return s


def test_static_rate_matches_max_rate_twice_in_a_row():
    import torch
    stream = torch.cuda.current_stream().cuda_stream
    sch = (cl.lele_d1_6(), cl.compact_filter(0.45))
    # call 1: 48^3 Taylor-Green box (many partials)
    d1, Q1, _ = cases.taylor_green(sch, n=48)
    s1 = _prepared_solver(d1, Q1)
    got1 = _static_rate(torch, s1, d1, stream)
    want1 = s1.max_rate()
    # call 2: a smaller two-species box with walls (fewer partials than call 1 left)
    eos = cl.IdealMixture([cl.IdealSpecies("a", 1.0, 1.4), cl.IdealSpecies("b", 0.3, 1.2)])
    d2 = cl.solver_desc((20, 16, 12), (1.0, 1.2, 0.8), (cl.PER3[0], (cl.SlipWallBC(), cl.SlipWallBC()), cl.PER3[2]),
                        *sch, eos=eos, transport=cl.Transport(mu0=1e-3))
    Q2 = cases.random_smooth_state(d2, seed=5, amp=0.2)
    s2 = _prepared_solver(d2, Q2)
    got2 = _static_rate(torch, s2, d2, stream)
    want2 = s2.max_rate()
    for got, want in ((got1, want1), (got2, want2)):
        assert np.isfinite(got).all()
        assert abs(got[0] - want[0]) <= 1e-14 * abs(want[0])
        assert abs(got[1] - want[1]) <= 1e-14 * abs(want[1])


def test_static_rate_rejects_grids_beyond_its_limit():
    import torch
    stream = torch.cuda.current_stream().cuda_stream
    dummy = torch.zeros(8, dtype=torch.float64, device="cuda")
    one = (C.c_double * 1)(1.0)
    gam = (C.c_double * 1)(1.4)
    inv_h = (C.c_double * 3)(1.0, 1.0, 1.0)
    too_many = 33554432 + 1   # CLES_STATIC_MAX_CELLS + 1; rejected before any launch
    rc = cl.lib().cles_max_rate_static(C.c_void_p(dummy.data_ptr()), C.c_void_p(dummy.data_ptr()), too_many, 1, one,
                                       gam, inv_h, 0.0, 0.7, 0.7, C.c_void_p(dummy.data_ptr()), C.c_void_p(stream))
    assert rc == abi.CLES_EINVAL
    assert "static scratch limit" in cl.lib().cles_last_error().decode()
