"""Serving benchmark: a seeded Poisson stream of independent solves.

The request mix is one third each of 1-D two-species shock tubes, 2-D He/CO2
shock-interface cases and Taylor-Green boxes (compactles.jl_b200/scenarios).
The stream is processed two ways on the same GPU:

* one at a time: each request to completion with the plain FP64 host-stepped
  run! loop (cles_run), in arrival order; its time-to-solution follows from
  the measured service times of the sequential queue;
* served: requests are submitted to a cles_server when their arrival time
  comes and advanced by continuous batching.  Without --batching each
  request has its own solver (one graph launch per request per tick, steps of
  different requests overlapping on the device); with --batching requests of
  one physics class share a batch (one captured step advances all of them).

--load sets the arrival rate as a multiple of the one-at-a-time capacity
(1.5 by default, the latency case); --load inf submits every request at time
zero, which measures the server's capacity.  Reported: solves/s and p50/p99
time-to-solution of both, and whether every served result equals the same
request run alone: bitwise against the one-at-a-time run without batching.
With batching the relative L2 distance to the one-at-a-time (one-grid
solver) run is reported and held to 1e-10, and bitwise equality with the
request alone in a batch of its own is reported beside it: a batch's
autotuner picks each class's launch form (batched kernels or per-member
kernels) from the batch's composition, and the two forms round differently,
so a request alone and in the mix agree bitwise only where the choices
coincide (under a fixed form they always do).

  python compactles.jl_b200/serving.py [--requests 24] [--scale small|full] [--load 1.5|inf] [--batching]
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


def make_requests(cl, n, seed, scale):
    """The seeded request mix.  scale 'full' uses the sizes of the serving
    workload (tubes N 256-8192, 2-D cases 128x64-1024x256, 64^3 boxes to t=1);
    'small' shrinks every size so the whole comparison runs in about a minute."""
    rng = np.random.default_rng(seed)
    sch = (cl.lele_d1_6(), cl.compact_filter(0.45))
    reqs = []
    for i in range(n):
        kind = i % 3
        if kind == 0:
            lo, hi = (256, 8192) if scale == "full" else (256, 1024)
            N = int(round(math.exp(rng.uniform(math.log(lo), math.log(hi)))))
            desc, Q0, tf = cl.scenarios.two_species_tube(sch, N, rng.uniform(2, 20), rng.uniform(-0.8, 0.8))
            name = f"tube N={N}"
        elif kind == 1:
            if scale == "full":
                nx = 2 * int(round(math.exp(rng.uniform(math.log(128), math.log(1024)))) / 2)
                ny = 2 * int(round(math.exp(rng.uniform(math.log(64), math.log(256)))) / 2)
            else:
                nx = 2 * int(round(math.exp(rng.uniform(math.log(64), math.log(160)))) / 2)
                ny = 2 * int(round(math.exp(rng.uniform(math.log(32), math.log(64)))) / 2)
            desc, Q0, tf = cl.scenarios.shock_interface_2d(sch, nx, ny, rng.uniform(1.2, 2.5),
                                                           int(rng.integers(1 << 30)))
            if scale != "full":
                tf *= 0.25
            name = f"interface {nx}x{ny}"
        else:
            n3 = 64 if scale == "full" else 24
            desc, Q0, tf = cl.scenarios.taylor_green_box(sch, n3, tfinal=1.0 if scale == "full" else 0.1)
            name = f"tgv {n3}^3"
        reqs.append((name, desc, Q0, tf))
    return reqs


def one_at_a_time(cl, reqs):
    out, service = [], []
    for name, desc, Q0, tf in reqs:
        t0 = time.perf_counter()
        s = cl.Solver(desc)
        s.set_state(Q0)
        s.run(tf)
        out.append(s.get_state())
        del s
        service.append(time.perf_counter() - t0)
    return out, service


def alone_in_batch(cl, reqs):
    out = []
    for name, desc, Q0, tf in reqs:
        B = cl.Batch(desc)
        mid = B.add(desc, Q0, tf)
        B.run()
        out.append(B.fetch(mid))
        del B
    return out


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def served(cl, reqs, arrivals, max_active, budget, batching=False):
    srv = cl.Server(hbm_budget=budget, max_active=max_active, batching=batching)
    ids = [None] * len(reqs)
    t0 = time.perf_counter()
    nxt = 0
    while True:
        now = time.perf_counter() - t0
        while nxt < len(reqs) and arrivals[nxt] <= now:
            name, desc, Q0, tf = reqs[nxt]
            ids[nxt] = srv.submit(desc, Q0, tf)
            nxt += 1
        r, q = srv.tick()
        if r == 0 and q == 0:
            if nxt == len(reqs):
                break
            time.sleep(max(0.0, min(0.01, arrivals[nxt] - (time.perf_counter() - t0))))
    # server times are relative to its creation; convert to this clock
    done = []
    results = []
    for i, rid in enumerate(ids):
        st = srv.status(rid)
        if st["state"] != "done":
            raise RuntimeError(f"request {i} ended {st['state']}")
        done.append(st["done_s"])
        results.append(srv.fetch(rid))
    offset = 0.0  # the server was created right before t0
    return results, [d + offset for d in done]


def main(argv=None):
    p = argparse.ArgumentParser()
    p.add_argument("--requests", type=int, default=24)
    p.add_argument("--scale", choices=["small", "full"], default="small")
    p.add_argument("--seed", type=int, default=11)
    p.add_argument("--max-active", type=int, default=64)
    p.add_argument("--budget-gb", type=float, default=60.0)
    p.add_argument("--load", default="1.5", help="offered load over the one-at-a-time capacity, or inf")
    p.add_argument("--batching", action="store_true")
    a = p.parse_args(argv)
    cl = _package()
    reqs = make_requests(cl, a.requests, a.seed, a.scale)
    # warm the library (first-launch setup) outside the measurement
    w = cl.scenarios.two_species_tube((cl.lele_d1_6(), cl.compact_filter(0.45)), 128, 2.0, 0.1)
    s = cl.Solver(w[0]); s.set_state(w[1]); s.run(w[2], 5); s.run_graph(w[2], 10); del s
    base, service = one_at_a_time(cl, reqs)
    rng = np.random.default_rng(a.seed + 1)
    if a.load == "inf":
        arrivals = np.zeros(len(reqs))
    else:
        lam = float(a.load) * len(reqs) / sum(service)     # offered load over one-at-a-time capacity
        arrivals = np.cumsum(rng.exponential(1.0 / lam, size=len(reqs)))
        arrivals -= arrivals[0]
    # one at a time on the same arrival stream
    fin, tts_base = [], []
    t = 0.0
    for i in range(len(reqs)):
        t = max(t, arrivals[i]) + service[i]
        fin.append(t)
        tts_base.append(t - arrivals[i])
    res, done = served(cl, reqs, list(arrivals), a.max_active, int(a.budget_gb * (1 << 30)), a.batching)
    tts = [done[i] - arrivals[i] for i in range(len(reqs))]
    extra = {}
    if a.batching:
        alone = alone_in_batch(cl, reqs)
        extra["bitwise_equal_alone_in_batch"] = all(np.array_equal(res[i], alone[i]) for i in range(len(reqs)))
        extra["max_rel_l2_vs_one_grid_solver"] = max(rel_l2(res[i], base[i]) for i in range(len(reqs)))
        same = extra["max_rel_l2_vs_one_grid_solver"] <= 1e-10
    else:
        same = all(np.array_equal(res[i], base[i]) for i in range(len(reqs)))
    out = {
        "workload": f"{len(reqs)} requests ({a.scale}): tubes / 2-D shock-interface / TGV boxes, Poisson seed {a.seed}",
        "offered_load": ("every request at time zero (capacity)" if a.load == "inf"
                         else f"{a.load}x one-at-a-time capacity"),
        "batching": a.batching,
        "served": {"solves_per_s": len(reqs) / max(done), "p50_s": float(np.percentile(tts, 50)),
                   "p99_s": float(np.percentile(tts, 99))},
        "one_at_a_time": {"solves_per_s": len(reqs) / fin[-1], "p50_s": float(np.percentile(tts_base, 50)),
                          "p99_s": float(np.percentile(tts_base, 99)), "service_s_total": sum(service)},
        "speedup_solves_per_s": (len(reqs) / max(done)) / (len(reqs) / fin[-1]),
        # no schedule finishes before its longest request does alone: the
        # capacity ratio over one-at-a-time is at most total / longest
        "longest_request_alone_s": max(service),
        "speedup_bound_total_over_longest": sum(service) / max(service),
        "results_equal_alone": same,
        **extra,
    }
    print(json.dumps(out), flush=True)
    return out


if __name__ == "__main__":
    main()
