"""Ensemble workload: many independent 2-D He/CO2 shock-interface solves on one GPU.

64 cases from one seed (default 7): grid (nx, ny, 1) with nx and ny drawn
log-uniform in [128, 1024] x [64, 256] and rounded to even, shock Mach number
uniform in [1.2, 2.5], an 8-mode interface perturbation of its own seed, slip
walls in x, periodic y, run to t_end = 0.5 Lx / c_He
(compactles.jl_b200/scenarios.shock_interface_2d).  Two ways to run the
whole ensemble, each in mixed precision and in FP64 on the same GPU:
  batch   one cles_batch: every case's fields in one arena, one captured
          CUDA graph per composition, a fixed number of launches per step
          for all cases together (line solves from per-grid descriptor
          tables, autotuned lines per CTA); cases retire as they finish;
  server  a cles_server: each case its own solver and stream, one CUDA-graph
          launch per case per step;
  batchesK a cles_server with batching: the cases spread over batches of at
          most K members (default 16), each on its own stream, whose captured
          steps run concurrently.

Reported per mode and precision: aggregate cell-steps/s (sum over cases of
cells x steps, over the wall time of the whole ensemble), solves/s, and per
case the relative L2 difference of the mixed-precision end state from the
FP64 end state (max over conserved components); for the batch, its
compositions, launches per step and the autotuner's choices.

  python compactles.jl_b200/ensemble.py [--cases 64] [--seed 7] [--modes batch,server]
"""
import argparse
import importlib.util
import json
import math
import pathlib
import sys
import time

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent


def _package():
    if "compactles_b200" in sys.modules:
        return sys.modules["compactles_b200"]
    spec = importlib.util.spec_from_file_location("compactles_b200", HERE / "__init__.py",
                                                  submodule_search_locations=[str(HERE)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["compactles_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def draw_cases(n, seed, nx_range=(128, 1024), ny_range=(64, 256)):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        nx = 2 * int(round(math.exp(rng.uniform(*np.log(nx_range))) / 2))
        ny = 2 * int(round(math.exp(rng.uniform(*np.log(ny_range))) / 2))
        out.append((nx, ny, float(rng.uniform(1.2, 2.5)), int(rng.integers(1 << 31))))
    return out


def serve(cl, reqs, max_active, budget, batching=False, batch_members=0):
    srv = cl.Server(hbm_budget=budget, max_active=max_active, batching=batching, batch_members=batch_members)
    t0 = time.perf_counter()
    ids = [srv.submit(desc, Q0, tf) for desc, Q0, tf in reqs]
    srv.drain()
    wall = time.perf_counter() - t0
    states, steps = [], []
    for rid in ids:
        st = srv.status(rid)
        if st["state"] != "done":
            raise RuntimeError(f"request ended {st['state']} ({st['failure']})")
        steps.append(st["steps"])
        states.append(srv.fetch(rid))
    return wall, steps, states


def run_batch(cl, reqs, trace=None):
    B = cl.Batch(reqs[0][0])
    t0 = time.perf_counter()
    ids = [B.add(desc, Q0, tf) for desc, Q0, tf in reqs]
    n = len(reqs)
    while n > 0:
        ts = time.perf_counter()
        n = B.step()
        if trace is not None:
            trace.append((n, time.perf_counter() - ts))
    B.step()
    wall = time.perf_counter() - t0
    states, steps = [], []
    for mid in ids:
        st = B.status(mid)
        if st["state"] != "done":
            raise RuntimeError(f"member ended {st['state']} ({st['failure']})")
        steps.append(st["steps"])
        states.append(B.fetch(mid))
    return wall, steps, states, B.stats()


def rel_l2(a, b, desc):
    sl = (slice(None),) + _package().problem.interior_slices(desc)
    a, b = a[sl], b[sl]
    return max(float(np.linalg.norm(a[c] - b[c]) / max(np.linalg.norm(b[c]), 1e-300)) for c in range(a.shape[0]))


def main(argv=None):
    p = argparse.ArgumentParser()
    p.add_argument("--cases", type=int, default=64)
    p.add_argument("--seed", type=int, default=7)
    p.add_argument("--max-active", type=int, default=64)
    p.add_argument("--budget-gb", type=float, default=100.0)
    p.add_argument("--precisions", default="mixed,fp64")
    p.add_argument("--modes", default="batch,server")
    a = p.parse_args(argv)
    cl = _package()
    sch = (cl.lele_d1_6(), cl.compact_filter(0.45))
    cases = draw_cases(a.cases, a.seed)
    # warm the library outside the measurement
    for prec in ("fp64", "mixed"):
        wd = cl.scenarios.shock_interface_2d(sch, 64, 32, 1.5, 1, precision=prec)
        s = cl.Solver(wd[0])
        s.set_state(wd[1])
        s.run_graph(wd[2], 5)
        del s
        wb = cl.Batch(wd[0])
        wb.add(*wd)
        wb.run(5)
        del wb
    res, states = {}, {}
    for mode in a.modes.split(","):
        for prec in a.precisions.split(","):
            reqs = [cl.scenarios.shock_interface_2d(sch, nx, ny, M, sd, precision=prec) for nx, ny, M, sd in cases]
            extra = {}
            if mode == "batch":
                trace = []
                wall, steps, st, bstats = run_batch(cl, reqs, trace)
                # where the time goes: batch steps by the number of members still running
                bands = {}
                for lo, hi in ((33, 10 ** 9), (9, 32), (2, 8), (0, 1)):
                    sel = [dt for n, dt in trace if lo <= n <= hi]
                    bands[f"{lo}-{hi if hi < 10 ** 9 else 'all'} running"] = {
                        "steps": len(sel), "s": sum(sel), "ms_per_step": 1e3 * sum(sel) / max(len(sel), 1)}
                extra = {"compositions": bstats["compositions"], "launches_per_step": bstats["launches_per_step"],
                         "batch_steps": bstats["steps"], "time_by_members_running": bands}
            elif mode.startswith("batches"):
                # a cles_server with batching: the cases spread over batches of at
                # most k members, each on its own stream, stepped concurrently
                k = int(mode[len("batches"):] or 16)
                wall, steps, st = serve(cl, reqs, a.max_active, int(a.budget_gb * (1 << 30)), True, k)
            else:
                wall, steps, st = serve(cl, reqs, a.max_active, int(a.budget_gb * (1 << 30)))
            cs = sum(nx * ny * k for (nx, ny, _, _), k in zip(cases, steps))
            res[f"{mode}_{prec}"] = {"wall_s": wall, "cell_steps": cs, "cell_steps_per_s": cs / wall,
                                     "solves_per_s": len(cases) / wall, "steps_total": int(sum(steps)), **extra}
            states[(mode, prec)] = (reqs, st)
    out = {"workload": f"{a.cases} 2-D He/CO2 shock-interface cases, seed {a.seed}, "
                       "nx 128-1024, ny 64-256, t_end 0.5 Lx/c_He",
           "results": res}
    for mode in a.modes.split(","):
        if (mode, "mixed") in states and (mode, "fp64") in states:
            f, m = states[(mode, "fp64")], states[(mode, "mixed")]
            errs = [rel_l2(x, y, r[0]) for r, x, y in zip(f[0], m[1], f[1])]
            out[f"{mode}_mixed_vs_fp64_rel_l2"] = {"max": max(errs), "median": float(np.median(errs))}
            out[f"{mode}_mixed_speedup"] = (res[f"{mode}_mixed"]["cell_steps_per_s"] /
                                            res[f"{mode}_fp64"]["cell_steps_per_s"])
    if ("batch", "fp64") in states and ("server", "fp64") in states:
        b, s_ = states[("batch", "fp64")], states[("server", "fp64")]
        errs = [rel_l2(x, y, r[0]) for r, x, y in zip(b[0], b[1], s_[1])]
        out["batch_vs_server_fp64_rel_l2_max"] = max(errs)
        for prec in a.precisions.split(","):
            out[f"batch_over_server_{prec}"] = (res[f"batch_{prec}"]["cell_steps_per_s"] /
                                                res[f"server_{prec}"]["cell_steps_per_s"])
    print(json.dumps(out), flush=True)
    return out


if __name__ == "__main__":
    main()
