"""A whole solver step on a decomposed grid, every rank on one GPU.

The ranks of a process grid run as host threads of this process, each with
its own solver (cles_solver_create_decomposed) and stream, exchanging through
the library's in-process group (cles_local_group_*): the device never waits
on another rank, the threads meet at host barriers.  Each rank's block is
assembled and compared with the oracle's Solver whose derivative and filter
plans along the split dims emulate the same ranks (orc_solver_split: the
reference's LineSolver / BandLineSolver with P > 1, src/tridiag.jl:136-170,
src/banded.jl:177-214, on a Decomp with halos, src/halo.jl:143-194):

* one right-hand side within 1e-12 of each component's term scale (the
  bound of the undecomposed solver tests), plain relative error recorded;
* steps of run! within 1e-10 relative L2, the same number of steps and the
  same clock (max_rate's allreduce of (rate, -rho_min), src/timestep.jl:173);
* the kinetic energy summed over the ranks.

Cases: a Taylor-Green box split along z into 2 (periodic, C6 + C8 filter),
the same box as a 2 x 2 pencil (x and y), a two-species He/CO2 shock-interface
grid split along x into 3 uneven pieces (slip walls: the first and last rank
own the faces; species sensors and their fourth differences across the rank
interfaces), the C10 (pentadiagonal) derivative on a z-split box, and the
mixed form against the FP64 oracle.  Errors: a collapsed or characteristic
split dim is refused, graph mode refuses a decomposed solver, and a rank
that stops makes the others' exchanges fail (CLES_EXCHANGE) instead of
waiting."""
import threading

import numpy as np
import pytest
import torch

import cases
import compactles_b200 as cl
import parity
from compactles_b200 import scenarios

pytestmark = pytest.mark.gpu


class Ranks:
    """Every rank of `dims` on cuda:0, each a solver on its own stream."""

    def __init__(self, desc, dims, Q0, timeout_s=60.0):
        self.desc = desc
        self.decomps = cl.Decomp.all_ranks(desc.n_global, dims)
        self.group = cl.LocalGroup(dims, timeout_s=timeout_s)
        it = Q0[(slice(None),) + cl.interior_slices(desc)]
        self.streams, self.ctxs, self.solvers = [], [], []
        for d in self.decomps:
            st = torch.cuda.Stream()
            ctx = cl.Context(0, stream=st.cuda_stream)
            S = cl.Solver(desc, ctx, decomp=d, exchange=self.group.exchange(d.coords))
            assert S.n_local == d.n_local
            S.set_state(d.block(it), layout="interior")
            self.streams.append(st)
            self.ctxs.append(ctx)
            self.solvers.append(S)

    def each(self, fn):
        """fn(solver) on every rank at once (one thread each); the results in rank order."""
        out = [None] * len(self.solvers)
        errs = []

        def work(i):
            try:
                out[i] = fn(self.solvers[i])
            except BaseException as e:   # noqa: BLE001 - re-raised below
                errs.append(e)
                self.group.abort()

        th = [threading.Thread(target=work, args=(i,)) for i in range(len(self.solvers))]
        for t in th:
            t.start()
        for t in th:
            t.join(timeout=600)
        assert not any(t.is_alive() for t in th)
        if errs:
            raise errs[0]
        return out

    def state(self):
        return cl.assemble(self.decomps, [S.get_state(layout="interior") for S in self.solvers])

    def rhs(self):
        return cl.assemble(self.decomps, self.each(lambda S: S.compute_rhs(layout="interior")))


def _oracle(orc, do, dims, Q0):
    O = orc.Solver(do)
    for k in range(3):
        if dims[k] > 1:
            O.split(k + 1, dims[k])
    O.set_state(Q0)
    return O


def _it(desc):
    sl = (slice(None),) + cl.interior_slices(desc)
    return lambda A: A[sl]


def _rel_l2(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _check(orc, label, dg, do, Q0, dims, steps, rhs_bound=1e-12, l2_bound=1e-10, ke_bound=1e-12, t_bound=1e-12):
    R = Ranks(dg, dims, Q0)
    O = _oracle(orc, do, dims, Q0)
    it = _it(dg)
    plain, term = parity.rhs_errors(R.rhs(), it(O.compute_rhs()), O.rhs_scales(cl.grid_spacing(dg)))
    parity.record(f"{label} decomposed {dims} RHS", plain, term)
    assert max(term) < rhs_bound, (plain, term)
    res = R.each(lambda S: S.run(1e9, steps))
    rc, ro = O.run(1e9, steps)
    assert rc == 0
    assert all(r.steps == steps for r in res)
    assert len({r.t for r in res}) == 1 and abs(res[0].t - ro.t) <= t_bound * ro.t
    rel = _rel_l2(R.state(), it(O.get_state()))
    kes = R.each(lambda S: S.kinetic_energy())
    ke_o = O.kinetic_energy()
    parity.record(f"{label} decomposed {dims} {steps} steps", state_l2=rel, ke_rel=abs(kes[0] - ke_o) / ke_o)
    assert rel < l2_bound, rel
    assert len(set(kes)) == 1 and abs(kes[0] - ke_o) <= ke_bound * ke_o
    return R


def _tgv(orc, n, deriv=None, precision="fp64"):
    dg, Q0, _ = cases.taylor_green((deriv[0] if deriv else cl.lele_d1_6(), cl.compact_filter(0.45)), n=n,
                                   precision=precision)
    do, _, _ = cases.taylor_green((deriv[1] if deriv else orc.lele_d1_6(), orc.compact_filter(0.45)), n=n)
    return dg, do, Q0


def test_tgv_split_z(orc):
    dg, do, Q0 = _tgv(orc, 32)
    _check(orc, "TGV 32^3 FP64", dg, do, Q0, (1, 1, 2), 10)


def test_tgv_pencil_xy(orc):
    dg, do, Q0 = _tgv(orc, 32)
    _check(orc, "TGV 32^3 FP64", dg, do, Q0, (2, 2, 1), 5)


def test_tgv_c10_split_z(orc):
    dg, do, Q0 = _tgv(orc, 32, deriv=(cl.lele_d1_10(), orc.lele_d1_10()))
    _check(orc, "TGV 32^3 C10 FP64", dg, do, Q0, (1, 1, 3), 5)


def test_shock_interface_split_x_uneven(orc):
    dg, Q0, _ = scenarios.shock_interface_2d((cl.lele_d1_6(), cl.compact_filter(0.45)), 100, 48, 2.0, 5)
    do, _, _ = scenarios.shock_interface_2d((orc.lele_d1_6(), orc.compact_filter(0.45)), 100, 48, 2.0, 5)
    R = _check(orc, "shock-interface 100x48 two species FP64", dg, do, Q0, (3, 1, 1), 20)
    assert [d.n_local[0] for d in R.decomps] == [34, 33, 33]


def test_mixed_against_fp64_oracle(orc):
    dg, do, Q0 = _tgv(orc, 32, precision="mixed")
    # the mixed form's dt follows its FP32 sound speed: the clocks agree to ~1e-7
    _check(orc, "TGV 32^3 mixed", dg, do, Q0, (1, 2, 1), 10, rhs_bound=2e-6, l2_bound=1e-5, ke_bound=1e-6,
           t_bound=1e-5)


def test_checkpoint_per_rank(tmp_path, orc):
    dg, do, Q0 = _tgv(orc, 32)
    R = Ranks(dg, (1, 1, 2), Q0)
    R.each(lambda S: S.run(1e9, 3))
    before = R.state()
    prefix = str(tmp_path / "tgv")
    R.each(lambda S: S.save_checkpoint(prefix))
    assert sorted(p.name for p in tmp_path.iterdir()) == ["tgv.r0000.ckpt", "tgv.r0001.ckpt"]
    R2 = Ranks(dg, (1, 1, 2), np.zeros_like(Q0))
    R2.each(lambda S: S.load_checkpoint(prefix))
    np.testing.assert_array_equal(R2.state(), before)
    assert R2.solvers[1].steps == 3
    # a rank of another decomposition cannot read the block
    R3 = Ranks(dg, (1, 2, 1), np.zeros_like(Q0))
    with pytest.raises(cl.ClesError, match="decomposition mismatch"):
        R3.solvers[0].load_checkpoint(prefix)


def test_refusals(orc):
    dg, _, Q0 = _tgv(orc, 32)
    grp = cl.LocalGroup((1, 1, 2))
    d = dg
    d.n_global[2] = 1
    with pytest.raises(cl.ClesError, match="collapsed"):
        cl.Solver(d, decomp=cl.Decomp(d.n_global, (1, 1, 2), (0, 0, 0)), exchange=grp.exchange((0, 0, 0)))
    dg, _, Q0 = _tgv(orc, 32)
    R = Ranks(dg, (1, 1, 2), Q0)
    with pytest.raises(cl.ClesError, match="graph mode"):
        R.solvers[0].run_graph(1.0, 1)


def test_a_piece_below_the_scheme_minimum_is_refused(orc):
    # src/operators.jl:50-53: every rank refuses a split whose smallest piece is too short
    dg, _, Q0 = _tgv(orc, 16)
    grp = cl.LocalGroup((1, 1, 2))
    with pytest.raises(cl.ClesError, match="too small"):
        cl.Solver(dg, decomp=cl.Decomp(dg.n_global, (1, 1, 2), (0, 0, 1)),
                  exchange=grp.exchange((0, 0, 1)))


def test_nscbc_on_a_split_dim_is_refused():
    sch = (cl.lele_d1_6(), cl.compact_filter(0.45))
    d, Q0, _ = scenarios.shock_interface_2d(sch, 64, 32, 2.0, 3)
    d.bc[0][1] = cl.abi.CLES_BC_NSCBC_OUTFLOW
    grp = cl.LocalGroup((2, 1, 1))
    with pytest.raises(cl.ClesError, match="NSCBC"):
        cl.Solver(d, decomp=cl.Decomp(d.n_global, (2, 1, 1), (1, 0, 0)), exchange=grp.exchange((1, 0, 0)))


def test_a_stopped_rank_fails_the_exchange_instead_of_waiting(orc):
    dg, _, Q0 = _tgv(orc, 32)
    R = Ranks(dg, (1, 1, 2), Q0, timeout_s=2.0)
    # rank 1 never joins: rank 0's first exchange gives up after the group's
    # timeout (host barrier), with nothing of rank 0 left waiting on the device
    with pytest.raises(cl.ClesError) as ei:
        R.solvers[0].run(1e9, 1)
    assert ei.value.code == cl.abi.CLES_EXCHANGE
    torch.cuda.synchronize()
    # the context is still usable: an undecomposed solver runs on the same GPU
    S = cl.Solver(dg)
    S.set_state(Q0)
    S.run(1e9, 1)


def test_tgv256_split_z_matches_undecomposed():
    """At the benchmark's 256^3 (tile kernels on every split piece): 2 z-slabs
    against the undecomposed solver, itself parity-tested against the oracle
    at this size."""
    sch = (cl.lele_d1_6(), cl.compact_filter(0.45))
    dg, Q0, _ = scenarios.taylor_green_box(sch, 256, tfinal=1e9)
    S = cl.Solver(dg)
    S.set_state(Q0)
    S.run(1e9, 2)
    ref = S.get_state(layout="interior")
    del S
    torch.cuda.empty_cache()
    R = Ranks(dg, (1, 1, 2), Q0)
    R.each(lambda S: S.run(1e9, 2))
    rel = _rel_l2(R.state(), ref)
    parity.record("TGV 256^3 FP64 decomposed (1, 1, 2) 2 steps vs undecomposed", state_l2=rel)
    assert rel < 1e-12, rel
