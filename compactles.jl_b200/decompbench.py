"""Whole run! steps on a decomposed grid, every rank on one GPU.

The ranks of a process grid run as host threads of one process, each with its
own solver (cles_solver_create_decomposed) and stream, exchanging through the
in-process group (cles_local_group_*: a stream synchronisation and two host
barriers per exchange).  K steps of every rank are timed together (wall
clock between device synchronisations: the ranks share the GPU, so this is
the aggregate cost of the decomposed step on one device), beside the
undecomposed solver on the same grid.  The state after the timed steps is
compared with the undecomposed solver's (relative L2), and the exchange
volume per rank and step is counted, from which its NVLink time on P GPUs is
estimated at the measured 770 GB/s peer copy.

  python compactles.jl_b200/decompbench.py [--n 256] [--grids 1x1x2 1x1x4 2x2x1] [--steps 5] [--warmup 2]
"""
import argparse
import importlib.util
import json
import pathlib
import sys
import threading
import time

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


def _each(solvers, group, fn):
    out, errs = [None] * len(solvers), []

    def work(i):
        try:
            out[i] = fn(solvers[i])
        except BaseException as e:   # noqa: BLE001 - re-raised below
            errs.append(e)
            group.abort()

    th = [threading.Thread(target=work, args=(i,)) for i in range(len(solvers))]
    for t in th:
        t.start()
    for t in th:
        t.join()
    if errs:
        raise errs[0]
    return out


def exchange_bytes(desc, dc, fp_bytes, ncons, deriv_M=2, filt_M=4, q=1):
    """Bytes one rank receives per step: per stage the split applications
    (velocity gradients 3 fields, dT 1, the two sensors' smoothing 2, the flux
    divergence ncons; halo 2 M planes and the gathered heads and tails of
    every rank), the delta4 halos (2 fields, 2 planes per end), then the
    FP64 state filter (ncons fields)."""
    total = 0
    for k in range(3):
        if dc.dims[k] == 1:
            continue
        lines = 1
        for e in range(3):
            if e != k:
                lines *= dc.n_local[e]
        P = dc.dims[k]

        def app(count, M, el):
            return el * count * lines * (2 * M + 2 * q * P)
        stage = (app(3, deriv_M, fp_bytes) + app(1, deriv_M, fp_bytes) + app(2, filt_M, fp_bytes)
                 + app(ncons, deriv_M, fp_bytes) + fp_bytes * 2 * lines * 2 * 2)
        total += 5 * stage + app(ncons, filt_M, 8)
    return total


def main(argv=None):
    p = argparse.ArgumentParser()
    p.add_argument("--n", type=int, default=256)
    p.add_argument("--grids", nargs="+", default=["1x1x2", "1x1x4", "2x2x1"])
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=2)
    p.add_argument("--precision", choices=["fp64", "mixed"], default="fp64")
    a = p.parse_args(argv)
    import torch
    cl = _package()
    torch.cuda.set_device(0)
    sch = (cl.lele_d1_6(), cl.compact_filter(0.45))
    desc, Q0, _ = cl.scenarios.taylor_green_box(sch, a.n, tfinal=1e9, precision=a.precision)
    it = Q0[(slice(None),) + cl.interior_slices(desc)]
    cells = a.n ** 3
    el = 8 if a.precision == "fp64" else 4

    # the undecomposed solver on the same grid
    S = cl.Solver(desc)
    S.set_state(Q0)
    S.run(1e9, a.warmup)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    S.run(1e9, a.warmup + a.steps)
    torch.cuda.synchronize()
    single_ms = (time.perf_counter() - t0) * 1e3 / a.steps
    ref = S.get_state(layout="interior")
    del S
    torch.cuda.empty_cache()
    print(json.dumps({"grid": [a.n] * 3, "precision": a.precision, "ranks": 1, "ms_per_step": single_ms,
                      "cell_steps_per_s": cells / (single_ms * 1e-3)}), flush=True)

    for g in a.grids:
        dims = tuple(int(v) for v in g.split("x"))
        ds = cl.Decomp.all_ranks(desc.n_global, dims)
        group = cl.LocalGroup(dims, timeout_s=120.0)
        streams, ctxs, solvers = [], [], []
        for d in ds:
            st = torch.cuda.Stream()
            ctx = cl.Context(0, stream=st.cuda_stream)
            R = cl.Solver(desc, ctx, decomp=d, exchange=group.exchange(d.coords))
            R.set_state(d.block(it), layout="interior")
            streams.append(st)
            ctxs.append(ctx)
            solvers.append(R)
        _each(solvers, group, lambda R: R.run(1e9, a.warmup))
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        _each(solvers, group, lambda R: R.run(1e9, a.warmup + a.steps))
        torch.cuda.synchronize()
        ms = (time.perf_counter() - t0) * 1e3 / a.steps
        got = cl.assemble(ds, [R.get_state(layout="interior") for R in solvers])
        rel = float(np.linalg.norm(got - ref) / np.linalg.norm(ref))
        xb = exchange_bytes(desc, ds[0], el, desc.n_species + 4)
        print(json.dumps({"grid": [a.n] * 3, "precision": a.precision, "dims": list(dims), "ranks": len(ds),
                          "ms_per_step_all_ranks_one_gpu": ms, "over_undecomposed": ms / single_ms,
                          "cell_steps_per_s_one_gpu": cells / (ms * 1e-3),
                          "state_rel_l2_vs_undecomposed": rel,
                          "exchange_bytes_per_rank_step": xb,
                          "nvlink_ms_per_step_estimate": xb / (NVLINK_GBS * 1e9) * 1e3}), flush=True)
        del solvers, ctxs, group
        torch.cuda.empty_cache()


if __name__ == "__main__":
    main()
