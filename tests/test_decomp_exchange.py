"""The exchange of a decomposed solver over gloo on CPU: TorchExchange's three
callbacks, called through their C function pointers exactly as
libcles.so calls them (cles_exchange), with host buffers.

* halo (Sendrecv!, src/halo.jl:143-194): recv_lo gets the previous rank's
  send_hi and recv_hi the next rank's send_lo, along the dim the call names;
  a closed end (-1) receives nothing; two ranks that wrap around each other
  (periodic, 2 ranks) exchange both ends.
* gather (Allgather! on decomp.sub[dim], src/tridiag.jl:148): blocks in
  coordinate order from the ranks of this rank's line only.
* allreduce (src/timestep.jl:173): max of (rate, -rho_min) and sums over
  every rank.

World sizes 2 (dims 2 x 1 x 1) and 4 (a 2 x 2 pencil, both dims split).
Decomp's local_range split is checked against the reference's formula."""
import ctypes as C
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _package():
    # the package directory name is not an identifier: load it by path (as conftest does)
    import importlib.util
    import pathlib
    import sys
    if "compactles_b200" not in sys.modules:
        pkg = pathlib.Path(__file__).resolve().parent.parent / "compactles.jl_b200"
        spec = importlib.util.spec_from_file_location("compactles_b200", pkg / "__init__.py",
                                                      submodule_search_locations=[str(pkg)])
        mod = importlib.util.module_from_spec(spec)
        sys.modules["compactles_b200"] = mod
        spec.loader.exec_module(mod)
    return sys.modules["compactles_b200"]


# spawned workers import this file without the test's conftest
cl = _package()
abi = cl.abi


def _ptr(a):
    return C.c_void_p(a.ctypes.data)


def _worker(rank, world, dims, periodic, port, q):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        dc = cl.Decomp((8, 8, 1), dims, cl.decomp.coords_of(rank, dims))
        ex = cl.TorchExchange(dc)
        st = ex.struct
        out = {"rank": rank, "coords": dc.coords}
        n = 5
        for dim in range(3):
            if dims[dim] == 1:
                continue
            P, me = dims[dim], dc.coords[dim]
            prev = (me - 1) % P if (periodic or me > 0) else -1
            nxt = (me + 1) % P if (periodic or me < P - 1) else -1
            send_lo = np.arange(n, dtype=np.float64) + 1000 * rank + 100 * dim
            send_hi = send_lo + 50
            recv_lo = np.full(n, -1.0)
            recv_hi = np.full(n, -1.0)
            rc = st.halo(None, dim, prev, nxt, _ptr(send_lo), _ptr(send_hi), _ptr(recv_lo), _ptr(recv_hi),
                         send_lo.nbytes, None)
            out[f"halo{dim}"] = (rc, prev, nxt, recv_lo.copy(), recv_hi.copy())
            local = np.full(3, 10.0 * rank + dim)
            allb = np.zeros(3 * P)
            rc = st.gather(None, dim, _ptr(local), _ptr(allb), local.nbytes, None)
            out[f"gather{dim}"] = (rc, allb.copy())
        v = (C.c_double * 2)(float(rank + 1), -float(10 - rank))
        rc = st.allreduce(None, abi.CLES_REDUCE_MAX, v, 2)
        out["max"] = (rc, v[0], v[1])
        s = (C.c_double * 1)(float(rank) + 0.5)
        rc = st.allreduce(None, abi.CLES_REDUCE_SUM, s, 1)
        out["sum"] = (rc, s[0])
        out["errors"] = [repr(e) for e in ex.errors]
        q.put(out)
    finally:
        dist.destroy_process_group()


def _run(dims, periodic):
    world = dims[0] * dims[1] * dims[2]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, dims, periodic, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    return {r["rank"]: r for r in res}


def _expect_halo(res, dims, dim, rank):
    r = res[rank]
    rc, prev, nxt, rlo, rhi = r[f"halo{dim}"]
    assert rc == 0
    n = len(rlo)
    base = np.arange(n, dtype=np.float64) + 100 * dim
    c = list(r["coords"])
    if prev >= 0:
        c[dim] = prev
        src = cl.decomp.rank_of(c, dims)
        np.testing.assert_array_equal(rlo, base + 1000 * src + 50)   # the previous rank's send_hi
    else:
        assert (rlo == -1).all()
    c = list(r["coords"])
    if nxt >= 0:
        c[dim] = nxt
        src = cl.decomp.rank_of(c, dims)
        np.testing.assert_array_equal(rhi, base + 1000 * src)        # the next rank's send_lo
    else:
        assert (rhi == -1).all()


@pytest.mark.parametrize("periodic", [False, True])
def test_exchange_two_ranks(periodic):
    dims = (2, 1, 1)
    res = _run(dims, periodic)
    for rank in res:
        assert not res[rank]["errors"]
        _expect_halo(res, dims, 0, rank)
        rc, allb = res[rank]["gather0"]
        assert rc == 0
        np.testing.assert_array_equal(allb, np.repeat([0.0, 10.0], 3))
        assert res[rank]["max"] == (0, 2.0, -9.0)
        assert res[rank]["sum"] == (0, 2.0)


def test_exchange_pencil_four_ranks():
    dims = (2, 2, 1)
    res = _run(dims, True)
    for rank in res:
        assert not res[rank]["errors"]
        for dim in (0, 1):
            _expect_halo(res, dims, dim, rank)
            rc, allb = res[rank][f"gather{dim}"]
            assert rc == 0
            c = list(res[rank]["coords"])
            want = []
            for r in range(2):
                c[dim] = r
                want += [10.0 * cl.decomp.rank_of(c, dims) + dim] * 3
            np.testing.assert_array_equal(allb, want)
        assert res[rank]["max"] == (0, 4.0, -7.0)
        assert res[rank]["sum"] == (0, 8.0)


def test_local_range_and_blocks():
    # local_range (src/decomposition.jl:73-78): the first N mod P ranks get one more point
    assert [cl.local_range(10, 3, r) for r in range(3)] == [(4, 0), (3, 4), (3, 7)]
    ds = cl.Decomp.all_ranks((10, 7, 1), (3, 2, 1))
    assert [d.coords for d in ds][:4] == [(0, 0, 0), (1, 0, 0), (2, 0, 0), (0, 1, 0)]
    Q = np.random.default_rng(1).standard_normal((5, 1, 7, 10))
    blocks = [d.block(Q) for d in ds]
    assert sum(b.size for b in blocks) == Q.size
    np.testing.assert_array_equal(cl.assemble(ds, blocks), Q)
