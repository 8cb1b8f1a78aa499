"""Split-line operator benchmark on one GPU: a 256^3 box of 5 FP64 fields cut
into P slabs along one dimension, every rank's phases run in turn on the
same device (pack, unpack, local solve, correction), timed with CUDA events
on the launching stream, beside the undecomposed plan on the same fields.

The exchanges between phases are device copies here (one GPU); on P GPUs
they are NCCL send/recv of the halo planes and an all-gather of the
interface values, whose sizes per rank and application are reported so
their NVLink time can be estimated (bytes / 770 GB/s measured peer copy).

  python compactles.jl_b200/splitbench.py [--n 256] [--fields 5] [--ranks 2 4] [--dims 3] [--reps 5]

Algorithmic bytes: the local solve and the correction each read and write
every field once (2 * 8 * points per field); pack and unpack move 2M planes.
"""
import argparse
import importlib.util
import json
import math
import pathlib
import sys

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
NVLINK_GBS = 770.0


def _package():
    if "compactles_b200" in sys.modules:
        return sys.modules["compactles_b200"]
    spec = importlib.util.spec_from_file_location("compactles_b200", HERE / "__init__.py",
                                                  submodule_search_locations=[str(HERE)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["compactles_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def local_range(N, P, r):
    base, rem = divmod(N, P)
    return base + (1 if r < rem else 0), r * base + min(r, rem)


def _field(torch, shape, count, seed):
    g = torch.Generator(device="cuda").manual_seed(seed)
    return torch.rand((count,) + shape, generator=g, device="cuda", dtype=torch.float64)


def bench_case(cl, torch, n, fields, P, dim, reps, periodic=True):
    nh = 4
    d0 = dim - 1
    h = 2 * math.pi / n
    scheme = cl.lele_d1_6()
    st = torch.cuda.current_stream()
    ranks = []
    for r in range(P):
        nr, _ = local_range(n, P, r)
        nl = [n, n, n]
        nl[d0] = nr
        plan = cl.SplitPlan(scheme, nl, dim, h, n, P, r, periodic, n_halo=nh)
        f = _field(torch, plan.shape(), fields, 7 + r)
        ranks.append(dict(plan=plan, f=f, out=torch.empty_like(f), bufs=plan.buffers(fields, "cuda"),
                          fs=int(np.prod(plan.shape())), pts=n * n * nr))

    def phase(name, fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        fn()
        e1.record(st)
        return name, e0, e1

    def one():
        ev = []
        for R in ranks:
            ev.append(phase("pack", lambda R=R: R["plan"].pack(R["f"], R["bufs"], fields, R["fs"])))
        for R in ranks:
            p, b = R["plan"], R["bufs"]
            if p.prev is not None:
                b["recv_lo"].copy_(ranks[p.prev]["bufs"]["send_hi"])
            if p.next is not None:
                b["recv_hi"].copy_(ranks[p.next]["bufs"]["send_lo"])
        for R in ranks:
            ev.append(phase("unpack", lambda R=R: R["plan"].unpack(R["bufs"], R["f"], fields, R["fs"])))
        for R in ranks:
            ev.append(phase("local", lambda R=R: R["plan"].begin(R["f"], R["out"], R["bufs"], fields, R["fs"])))
        allv = torch.stack([R["bufs"]["iface"] for R in ranks])
        for R in ranks:
            R["bufs"]["iface_all"].copy_(allv)
            ev.append(phase("correct", lambda R=R: R["plan"].end(R["bufs"], R["out"], fields, R["fs"])))
        return ev

    for _ in range(2):
        one()
    torch.cuda.synchronize()
    tot = {"pack": 0.0, "unpack": 0.0, "local": 0.0, "correct": 0.0}
    for _ in range(reps):
        ev = one()
        torch.cuda.synchronize()
        for name, e0, e1 in ev:
            tot[name] += e0.elapsed_time(e1)
    ms = {k: v / reps for k, v in tot.items()}

    # the undecomposed plan over the same points (one padded n^3 block)
    g = cl.grid((n, n, n), (1, 1, 1) if periodic else tuple(0 if k == d0 else 1 for k in range(3)), nh)
    plan = cl.DirPlan(g, scheme, dim, h, ctx=ranks[0]["plan"].ctx)
    F = _field(torch, plan.shape(), fields, 99)
    O = torch.empty_like(F)
    fs = int(np.prod(plan.shape()))
    L = cl.lib()
    import ctypes as C

    def single():
        cl.api._check(L.cles_apply_along_batch(plan.ptr, C.c_void_p(F.data_ptr()), C.c_void_p(O.data_ptr()), fields, fs))

    for _ in range(3):
        single()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(reps):
        single()
    e1.record(st)
    torch.cuda.synchronize()
    ms_single = e0.elapsed_time(e1) / reps

    pts = n ** 3 * fields
    alg = 2 * 8 * pts
    info = ranks[0]["plan"].info
    lines = n * n
    halo_bytes = 2 * info.M * lines * 8 * fields          # sent per interior rank and application
    gather_bytes = 2 * info.q * lines * 8 * fields * (P - 1)   # received per rank
    split_ms = sum(ms.values())
    return dict(n=n, fields=fields, ranks=P, dim=dim, periodic=periodic,
                ms=dict((k, round(v, 4)) for k, v in ms.items()), split_ms=round(split_ms, 4),
                single_ms=round(ms_single, 4), split_over_single=round(split_ms / ms_single, 3),
                local_GBs=round(alg / (ms["local"] * 1e-3) / 1e9, 1),
                correct_GBs=round(alg / (ms["correct"] * 1e-3) / 1e9, 1),
                single_GBs=round(alg / (ms_single * 1e-3) / 1e9, 1),
                per_rank_exchange_bytes=dict(halo_send=halo_bytes, gather_recv=gather_bytes),
                nvlink_ms_estimate=round((halo_bytes + gather_bytes) / (NVLINK_GBS * 1e9) * 1e3, 4),
                per_gpu_ms_estimate=round(split_ms / P + (halo_bytes + gather_bytes) / (NVLINK_GBS * 1e9) * 1e3, 4))


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--fields", type=int, default=5)
    ap.add_argument("--ranks", type=int, nargs="+", default=[2, 4])
    ap.add_argument("--dims", type=int, nargs="+", default=[1, 2, 3])
    ap.add_argument("--reps", type=int, default=5)
    a = ap.parse_args(argv)
    import torch
    cl = _package()
    for dim in a.dims:
        for P in a.ranks:
            print(json.dumps(bench_case(cl, torch, a.n, a.fields, P, dim, a.reps)), flush=True)


if __name__ == "__main__":
    main()
