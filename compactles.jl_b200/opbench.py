"""Compact-operator microbenchmark: directional C6 / C10 derivatives and the C8
filter applied to batches of 256^3 fields, periodic and wall-bounded, FP64 and
FP32, timed with CUDA events on the launching stream.

Fields are seeded sums of 16 Fourier modes, f = sum_m a_m/|k_m|^2 cos(k_m.x + phi_m)
with integer wavenumber components uniform in 1..32 (random sign),
a_m ~ N(0, 1), phi_m ~ U[0, 2pi), seed 20261203 + field index.

  python compactles.jl_b200/opbench.py [--n 256] [--fields 5] [--reps 5]
  python compactles.jl_b200/opbench.py --ncu-case      # 3 + 3 launches for an ncu capture
  python compactles.jl_b200/opbench.py --ncu-case closed   # the same on closed lines
  python compactles.jl_b200/opbench.py --ncu-case periodic --ncu-scheme c10 --ncu-dtype f32

Algorithmic bytes per launch: every field read once and written once,
2 * sizeof(T) * n^3 per field.  FP32 cases also report their error against
the FP64 plan on the same fields (max over the batch, relative to the FP64
maximum).  Parity of the FP64 plans with the CPU oracle on these fields is
checked in tests/test_gpu_opbench.py.
"""
import argparse
import importlib.util
import json
import math
import pathlib
import sys

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
ROOT = HERE.parent


def _package():
    if "compactles_b200" in sys.modules:
        return sys.modules["compactles_b200"]
    spec = importlib.util.spec_from_file_location("compactles_b200", HERE / "__init__.py",
                                                  submodule_search_locations=[str(HERE)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["compactles_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def fourier_field(n, seed, periodic, torch, dtype):
    """One seeded 16-mode field on n^3 (periodic: [0,2pi), closed: [0,2pi] with n-1 cells)."""
    rng = np.random.default_rng(seed)
    L = 2 * math.pi
    h = L / n if periodic else L / (n - 1)
    x = torch.arange(n, device="cuda", dtype=torch.float64) * h
    f = torch.zeros((n, n, n), device="cuda", dtype=torch.float64)
    for _ in range(16):
        k = rng.integers(1, 33, size=3) * rng.choice([-1, 1], size=3)
        a = rng.standard_normal()
        ph = rng.uniform(0, 2 * math.pi)
        kk = float(np.dot(k, k))
        f += (a / kk) * torch.cos(k[0] * x[None, None, :] + k[1] * x[None, :, None] + k[2] * x[:, None, None] + ph)
    return f.to(dtype), h


def run(args):
    import torch
    cl = _package()
    from compactles_b200 import abi
    C = cl.api.C
    torch.cuda.set_device(0)
    st = torch.cuda.current_stream()
    ctx = cl.Context(0, stream=st.cuda_stream)
    n, nf = args.n, args.fields
    schemes = {"c6": cl.lele_d1_6(), "c10": cl.lele_d1_10(), "filter": cl.compact_filter(0.45)}
    results = []
    cases = [(p, dt) for p in (True, False) for dt in ("f64", "f32")]
    if args.ncu_case:
        cases = [(args.ncu_case != "closed", args.ncu_dtype)]
        schemes = {args.ncu_scheme: schemes[args.ncu_scheme]}
    if getattr(args, "cases", None):
        cases = args.cases
    if getattr(args, "schemes", None):
        schemes = {k: schemes[k] for k in args.schemes}
    for periodic, dts in cases:
        tdtype = torch.float64 if dts == "f64" else torch.float32
        fields, hs = zip(*[fourier_field(n, 20261203 + i, periodic, torch, tdtype) for i in range(nf)])
        h = hs[0]
        fin = torch.stack(fields)
        fout = torch.empty_like(fin)
        fin64 = fin.double() if dts == "f32" and not args.ncu_case else None
        fref = torch.empty_like(fin64) if fin64 is not None else None
        el = fin.element_size()
        for sname, sch in schemes.items():
            for dim in (1, 2, 3):
                g = cl.grid((n, n, n), (periodic,) * 3)
                plan = cl.plan_direction(g, sch, dim, h, dtype=dts, layout="interior", ctx=ctx)

                def launch():
                    cl.api._check(cl.lib().cles_apply_along_batch(plan.ptr, C.c_void_p(fin.data_ptr()),
                                                                  C.c_void_p(fout.data_ptr()), nf, n ** 3))
                if args.ncu_case:
                    launch()          # one warm launch per direction first
                    continue
                for _ in range(2):
                    launch()
                torch.cuda.synchronize()
                ev = [torch.cuda.Event(enable_timing=True) for _ in range(2 * args.reps)]
                for r in range(args.reps):
                    ev[2 * r].record()
                    launch()
                    ev[2 * r + 1].record()
                torch.cuda.synchronize()
                ms = [ev[2 * r].elapsed_time(ev[2 * r + 1]) for r in range(args.reps)]
                avg = float(np.mean(ms))
                gbs = 2 * el * nf * n ** 3 / (avg / 1e3) / 1e9
                rec = {"scheme": sname, "dim": dim, "periodic": periodic, "dtype": dts, "fields": nf, "n": n,
                       "ms": avg, "GB/s": gbs}
                if fin64 is not None:
                    p64 = cl.plan_direction(g, sch, dim, h, dtype="f64", layout="interior", ctx=ctx)
                    cl.api._check(cl.lib().cles_apply_along_batch(p64.ptr, C.c_void_p(fin64.data_ptr()),
                                                                  C.c_void_p(fref.data_ptr()), nf, n ** 3))
                    torch.cuda.synchronize()
                    rec["rel_err_vs_fp64"] = float((fout.double() - fref).abs().max() / fref.abs().max())
                if args.keep:
                    rec["out"] = fout.clone()
                    rec["in"] = fin
                    rec["h"] = h
                results.append(rec)
                print(json.dumps({k: v for k, v in rec.items() if k not in ("out", "in")}), flush=True)
        if args.ncu_case:
            # the captured launches: one per direction
            for dim in (1, 2, 3):
                g = cl.grid((n, n, n), (periodic,) * 3)
                plan = cl.plan_direction(g, schemes[args.ncu_scheme], dim, h, dtype=dts, layout="interior", ctx=ctx)
                cl.api._check(cl.lib().cles_apply_along_batch(plan.ptr, C.c_void_p(fin.data_ptr()),
                                                              C.c_void_p(fout.data_ptr()), nf, n ** 3))
            torch.cuda.synchronize()
            print("ncu case done")
    return results


if __name__ == "__main__":
    p = argparse.ArgumentParser()
    p.add_argument("--n", type=int, default=256)
    p.add_argument("--fields", type=int, default=5)
    p.add_argument("--reps", type=int, default=5)
    p.add_argument("--ncu-case", nargs="?", const="periodic", default=None, choices=["periodic", "closed"],
                   help="3 + 3 launches (one warm, one captured per direction) for an ncu capture")
    p.add_argument("--ncu-scheme", choices=["c6", "c10", "filter"], default="c6")
    p.add_argument("--ncu-dtype", choices=["f64", "f32"], default="f64")
    p.add_argument("--keep", action="store_true", help=argparse.SUPPRESS)
    run(p.parse_args())
