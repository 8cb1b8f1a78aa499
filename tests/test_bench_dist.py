"""The multi-rank path of bench.py on CPU: world_size 2 over gloo checks the
max-over-ranks timing and the whole-job aggregation that the NCCL run uses
(replicas, weak scaling; no data-path collective)."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

import bench


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ.update({"RANK": str(rank), "LOCAL_RANK": str(rank), "WORLD_SIZE": str(world),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    d = bench.Dist(backend="gloo")
    d.barrier()
    local_ms = 100.0 * (rank + 1)     # rank 1 is the slow one
    mx = d.max(local_ms)
    v = bench.aggregate(cells=1000, steps=10, world=d.world, max_ms=mx)
    q.put((rank, d.world, mx, v))
    d.close()


def test_two_rank_max_and_aggregate():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    for rank, world, mx, v in got:
        assert world == 2
        assert mx == 200.0                       # max over ranks, not the local time
        assert v == pytest.approx(2 * 1000 * 10 / 0.2)


def test_single_process_defaults():
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        os.environ.pop(k, None)
    d = bench.Dist()
    assert d.world == 1 and d.rank == 0 and d.max(3.5) == 3.5
    d.close()


def test_parse_rejects_short_warmup():
    with pytest.raises(SystemExit):
        bench.parse(["--warmup", "2"])
    a = bench.parse([])
    assert a.gpus == 1 and a.warmup >= 3 and a.n == 256
