"""Curvilinear-grid step benchmark: the full run! step (BCs, max_rate, five
LSRK stages, filter) on 256^3 grids with the reference's geometry features,
timed with CUDA events on the solver's stream, beside the Cartesian
Taylor-Green step of the same size.

Workloads (all synthetic, seeded by their analytic initial conditions):

  cylinder_axis     (r, theta, z) over [0, 1] x [0, 2 pi) x [0, 1): AxisBC at
                    r = 0 with theta resolved (paired fold), slip wall at r = 1;
                    a swirling jet with a theta-dependent density perturbation
  spherical_shell   (r, theta, phi) over [0.5, 1.5] x [0.3, pi - 0.3] x
                    [0, 2 pi): slip walls in r and theta (metric terms, no fold)
  stretched_channel Cartesian, x clustered by sine_cluster(0, 1, 0.5, 0.4)
                    between slip walls, periodic in y and z

  python compactles.jl_b200/geobench.py [--n 256] [--steps 5] [--warmup 3] [--workload all]

Each line reports cell-steps/s, ms per step, the compact kernels' share of
the step and their HBM throughput (algorithmic bytes over CUDA-event time).
"""
import argparse
import importlib.util
import json
import math
import pathlib
import sys

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


def workloads(cl, n):
    PER = (cl.PeriodicBC(), cl.PeriodicBC())
    sch = (cl.lele_d1_6(), cl.compact_filter(0.45))
    out = {}

    def jet(r, t, z):
        g = np.exp(-8 * r ** 2)
        x, y = r * np.cos(t), r * np.sin(t)
        return cl.Prim(u=(0.05 * r * g * np.cos(2 * np.pi * z), 0.3 * r * g + 0 * t, 0.5 * g + 0 * z),
                       p=1.0 + 0 * r + 0 * z, rho=1.0 + 0.1 * np.exp(-10 * ((x - 0.3) ** 2 + y ** 2)) + 0 * z)
    out["cylinder_axis"] = (cl.solver_desc((n, n, n), (1.0, 2 * math.pi, 1.0), ((cl.AxisBC(), cl.SlipWallBC()), PER, PER),
                                           *sch, metric=cl.CylindricalMetric(), transport=cl.Transport(mu0=1e-4)), jet)

    def shell(r, t, p):
        return cl.Prim(u=(0.0 * r, 0.1 * np.sin(2 * (t - 0.3)) + 0 * p, 0.2 * r * np.sin(t) + 0 * p),
                       p=1.0 + 0.05 * np.exp(-20 * (r - 1.0) ** 2) * np.cos(p), rho=1.0 + 0 * r + 0 * t)
    out["spherical_shell"] = (cl.solver_desc((n, n, n), (1.0, math.pi - 0.6, 2 * math.pi),
                                             ((cl.SlipWallBC(), cl.SlipWallBC()), (cl.SlipWallBC(), cl.SlipWallBC()), PER),
                                             *sch, metric=cl.SphericalMetric(), origin=(0.5, 0.3, 0.0),
                                             transport=cl.Transport(mu0=1e-4)), shell)

    def channel(x, y, z):
        return cl.Prim(u=(0.1 * np.sin(np.pi * x) * np.cos(2 * np.pi * y), 0.5 * np.sin(np.pi * x) + 0 * z,
                          0.05 * np.sin(2 * np.pi * z) + 0 * x), p=1.0 + 0 * x + 0 * y, rho=1.0 + 0 * x + 0 * z)
    out["stretched_channel"] = (cl.solver_desc((n, n, n), (1.0, 1.0, 1.0), ((cl.SlipWallBC(), cl.SlipWallBC()), PER, PER),
                                               *sch, stretch=(cl.sine_cluster(0.0, 1.0, 0.5, 0.4), None, None),
                                               transport=cl.Transport(mu0=1e-4)), channel)
    out["cartesian_tgv"] = (cl.problem_desc(cl.taylor_green_problem(), cl.Numerics(n_global=(n, n, n)), *sch),
                            cl.taylor_green_problem().ic)
    return out


def time_case(cl, torch, desc, ic, steps, warmup, peak):
    ctx = cl.Context(torch.cuda.current_device(), stream=torch.cuda.current_stream().cuda_stream)
    S = cl.Solver(desc, ctx=ctx)
    S.set_state(cl.initialize(desc, ic))
    S.run(1e9, warmup)
    torch.cuda.synchronize()
    cl.profile_enable(True)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    res = S.run(1e9, warmup + steps)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    prof = cl.profile_read()
    cl.profile_enable(False)
    assert res.steps == steps, res.steps
    cells = S.info().cells
    cms = sum(v[1] for v in prof.values())
    cbytes = sum(v[2] for v in prof.values())
    Q = S.get_state()
    assert np.isfinite(Q).all()
    del S
    return dict(cell_steps_per_s=cells * steps / (ms * 1e-3), ms_per_step=ms / steps,
                compact_share=cms / ms, compact_GBs=cbytes / (cms * 1e-3) / 1e9 if cms else None,
                compact_frac_of_peak=(cbytes / (cms * 1e-3) / 1e9 / peak) if cms and peak else None)


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default="all")
    a = ap.parse_args(argv)
    import torch
    cl = _package()
    peak = None
    mp = HERE.parent / "MEASURED_PEAKS.json"
    if mp.exists():
        peak = json.loads(mp.read_text()).get("hbm_gbs")
    for name, (desc, ic) in workloads(cl, a.n).items():
        if a.workload != "all" and name != a.workload:
            continue
        r = time_case(cl, torch, desc, ic, a.steps, a.warmup, peak)
        print(json.dumps(dict(workload=name, n=a.n, steps=a.steps, warmup=a.warmup, dtype="f64", **r)), flush=True)


if __name__ == "__main__":
    main()
