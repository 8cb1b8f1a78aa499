"""The exchange of a split line over gloo on CPU (world sizes 2 and 3):
LineExchange moves the halo planes to the right neighbours (the Sendrecv!
pattern of src/halo.jl:143-194, including two ranks that wrap around each
other and a closed end with no neighbour) and all-gathers the interface
values in rank order (src/tridiag.jl:148).  The same calls carry device
tensors over NCCL on GPUs."""
import importlib.util
import os
import pathlib
import socket
import sys

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
