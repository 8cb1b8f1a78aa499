"""The exchange of a split line over gloo on CPU (world sizes 2 and 3):
LineExchange moves the halo planes to the right neighbours (the Sendrecv!
pattern of src/halo.jl:143-194, including two ranks that wrap around each
other and a closed end with no neighbour) and all-gathers the interface
values in rank order (src/tridiag.jl:148); split_apply_along runs its
phases in the right order around those exchanges, checked end to end with
a CPU stand-in for the device plan that keeps the C ABI's buffer layout;
and the exchange stays inside a sub-communicator (the reference's
decomp.sub[dim]) on a 2 x 2 grid of four ranks.  The same calls carry
device tensors over NCCL on GPUs."""
import importlib.util
import os
import pathlib
import socket
import sys

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _package():
    # the package directory name is not an identifier: load it by path (as conftest does)
    if "compactles_b200" not in sys.modules:
        pkg = pathlib.Path(__file__).resolve().parent.parent / "compactles.jl_b200"
        spec = importlib.util.spec_from_file_location("compactles_b200", pkg / "__init__.py",
                                                      submodule_search_locations=[str(pkg)])
        mod = importlib.util.module_from_spec(spec)
        sys.modules["compactles_b200"] = mod
        spec.loader.exec_module(mod)
    return sys.modules["compactles_b200"]


def _neighbours(rank, ranks, periodic):
    prev = (rank - 1) % ranks if (periodic or rank > 0) else None
    nxt = (rank + 1) % ranks if (periodic or rank < ranks - 1) else None
    return prev, nxt


def _worker(rank, world, port, periodic, q):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    import torch.distributed as dist
    cl = _package()
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        prev, nxt = _neighbours(rank, world, periodic)
        ex = cl.LineExchange(prev, nxt)
        n = 6
        # planes tagged by owner and end: low planes 100 r + i, high 100 r + 50 + i
        send_lo = torch.arange(n, dtype=torch.float64) + 100 * rank
        send_hi = torch.arange(n, dtype=torch.float64) + 100 * rank + 50
        recv_lo = torch.full((n,), -1.0, dtype=torch.float64)
        recv_hi = torch.full((n,), -1.0, dtype=torch.float64)
        for _ in range(2):   # repeated exchanges stay matched
            ex.halo(send_lo, send_hi, recv_lo, recv_hi)
        iface = torch.full((4,), float(rank), dtype=torch.float64)
        iface_all = torch.zeros(world, 4, dtype=torch.float64)
        ex.gather(iface, iface_all)
        q.put((rank, prev, nxt, recv_lo.tolist(), recv_hi.tolist(), iface_all.tolist()))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,periodic", [(2, True), (2, False), (3, True), (3, False)])
def test_line_exchange_over_gloo(world, periodic):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, world, port, periodic, q)) for r in range(world)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(world))
    n = 6
    for rank, prev, nxt, lo, hi, allv in got:
        # recv_lo holds the previous rank's high planes, recv_hi the next rank's low planes
        assert lo == ([100 * prev + 50 + i for i in range(n)] if prev is not None else [-1.0] * n)
        assert hi == ([100 * nxt + i for i in range(n)] if nxt is not None else [-1.0] * n)
        assert allv == [[float(r)] * 4 for r in range(world)]


def test_single_periodic_rank_is_its_own_neighbour():
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(_free_port())})
    import torch.distributed as dist
    import compactles_b200 as cl
    dist.init_process_group("gloo", rank=0, world_size=1)
    try:
        ex = cl.LineExchange(0, 0)
        lo, hi = torch.arange(4.0), torch.arange(4.0) + 10
        rlo, rhi = torch.zeros(4), torch.zeros(4)
        ex.halo(lo, hi, rlo, rhi)
        assert rlo.tolist() == hi.tolist() and rhi.tolist() == lo.tolist()
        allv = torch.zeros(1, 3)
        ex.gather(torch.ones(3), allv)
        assert allv.tolist() == [[1.0, 1.0, 1.0]]
    finally:
        dist.destroy_process_group()


class _StandInPlan:
    """One rank's piece of a z-split field with the cles_split_* buffer
    conventions (send/recv [count][M][lines], iface [count][2][lines],
    iface_all rank-major), computing on the CPU a stand-in operator that
    reads the halo (a central difference, one-sided at a closed end) and a
    correction that depends on every rank's interface values and their order.
    It checks the orchestration of split_apply_along, not the kernels."""

    M = 2

    def __init__(self, n_global, ranks, rank, periodic, nxy):
        base, rem = divmod(n_global, ranks)
        self.n = base + (1 if rank < rem else 0)
        self.rank, self.ranks, self.nxy = rank, ranks, nxy
        self.prev = (rank - 1) % ranks if (periodic or rank > 0) else None
        self.next = (rank + 1) % ranks if (periodic or rank < ranks - 1) else None

    def buffers(self, count, device):
        lines = self.nxy
        z = lambda *s: torch.zeros(*s, dtype=torch.float64)
        return dict(send_lo=z(count * self.M * lines), send_hi=z(count * self.M * lines),
                    recv_lo=z(count * self.M * lines), recv_hi=z(count * self.M * lines),
                    iface=z(count * 2 * lines), iface_all=z(self.ranks, count * 2 * lines))

    def pack(self, f, b, count=1, field_stride=None):
        M, n = self.M, self.n
        b["send_lo"].copy_(f[M:2 * M].reshape(-1))
        b["send_hi"].copy_(f[n:n + M].reshape(-1))

    def unpack(self, b, f, count=1, field_stride=None):
        M, n = self.M, self.n
        if self.prev is not None:
            f[0:M] = b["recv_lo"].reshape(M, -1)
        if self.next is not None:
            f[n + M:n + 2 * M] = b["recv_hi"].reshape(M, -1)

    def begin(self, f, out, b, count=1, field_stride=None):
        M, n = self.M, self.n
        g = f[M:M + n]
        d = f[M + 1:M + n + 1] - f[M - 1:M + n - 1]
        if self.prev is None:
            d[0] = 2 * (g[1] - g[0])
        if self.next is None:
            d[-1] = 2 * (g[-1] - g[-2])
        out[M:M + n] = d
        b["iface"].copy_(torch.stack([d[0], d[-1]]).reshape(-1))

    def end(self, b, out, count=1, field_stride=None):
        M, n = self.M, self.n
        allv = b["iface_all"].reshape(self.ranks, 2, -1)
        w = torch.arange(1, self.ranks + 1, dtype=torch.float64)[:, None, None]
        out[M:M + n] += (w * allv).sum(dim=(0, 1)) * 1e-3


def _global_standin(F, ranks, periodic):
    n = F.shape[0]
    base, rem = divmod(n, ranks)
    out = np.zeros_like(F)
    heads_tails = []
    off = 0
    for r in range(ranks):
        nr = base + (1 if r < rem else 0)
        idx = np.arange(off, off + nr)
        up = F[(idx + 1) % n]
        dn = F[(idx - 1) % n]
        d = up - dn
        if not periodic and r == 0:
            d[0] = 2 * (F[1] - F[0])
        if not periodic and r == ranks - 1:
            d[-1] = 2 * (F[n - 1] - F[n - 2])
        out[off:off + nr] = d
        heads_tails.append((d[0], d[-1]))
        off += nr
    corr = sum((r + 1) * (h + t) for r, (h, t) in enumerate(heads_tails)) * 1e-3
    return out + corr


def _orchestration_worker(rank, world, port, periodic, q):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    import torch.distributed as dist
    cl = _package()
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        n_global, nxy = 23, 6
        rng = np.random.default_rng(3)
        F = rng.standard_normal((n_global, nxy))
        plan = _StandInPlan(n_global, world, rank, periodic, nxy)
        base, rem = divmod(n_global, world)
        off = rank * base + min(rank, rem)
        M = plan.M
        f = torch.zeros(plan.n + 2 * M, nxy, dtype=torch.float64)
        f[M:M + plan.n] = torch.from_numpy(F[off:off + plan.n])
        out = torch.zeros_like(f)
        ex = cl.LineExchange(plan.prev, plan.next)
        cl.split_apply_along(out, plan, f, ex, bufs=plan.buffers(1, "cpu"))
        q.put((rank, off, out[M:M + plan.n].numpy().tolist()))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,periodic", [(2, True), (2, False), (3, True), (3, False)])
def test_split_apply_along_orchestration_over_gloo(world, periodic):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_orchestration_worker, args=(r, world, port, periodic, q)) for r in range(world)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(world))
    F = np.random.default_rng(3).standard_normal((23, 6))
    ref = _global_standin(F, world, periodic)
    for rank, off, piece in got:
        piece = np.array(piece)
        assert np.allclose(piece, ref[off:off + piece.shape[0]], rtol=0, atol=1e-13), rank


def _subgroup_worker(rank, world, port, q):
    # four ranks on a 2 x 2 grid: rows {0, 1} and {2, 3} each split a
    # periodic line two ways; every rank exchanges within its own row only
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    import torch.distributed as dist
    cl = _package()
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        rows = [dist.new_group([0, 1]), dist.new_group([2, 3])]
        row = rank // 2
        g = rows[row]
        coord = dist.get_rank(g)
        ex = cl.LineExchange((coord - 1) % 2, (coord + 1) % 2, group=g)
        n = 4
        send_lo = torch.arange(n, dtype=torch.float64) + 100 * rank
        send_hi = torch.arange(n, dtype=torch.float64) + 100 * rank + 50
        recv_lo = torch.full((n,), -1.0, dtype=torch.float64)
        recv_hi = torch.full((n,), -1.0, dtype=torch.float64)
        ex.halo(send_lo, send_hi, recv_lo, recv_hi)
        allv = torch.zeros(2, 3, dtype=torch.float64)
        ex.gather(torch.full((3,), float(rank), dtype=torch.float64), allv)
        q.put((rank, recv_lo.tolist(), recv_hi.tolist(), allv.tolist()))
    finally:
        dist.destroy_process_group()


def test_line_exchange_within_a_sub_communicator():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_subgroup_worker, args=(r, 4, port, q)) for r in range(4)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(4))
    for rank, lo, hi, allv in got:
        partner = rank ^ 1              # the other rank of the same row, both neighbours
        assert lo == [100 * partner + 50 + i for i in range(4)]
        assert hi == [100 * partner + i for i in range(4)]
        row0 = 2 * (rank // 2)
        assert allv == [[float(row0)] * 3, [float(row0 + 1)] * 3]
