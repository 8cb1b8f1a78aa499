"""Taylor-Green energy histories on the device: FP64 against mixed precision.

Two cases:

* ``readme64``: the case behind the README's quoted dissipation peak
  (docs/figures/readme_header.jl:24-95): Re 1600 (mu0 = 1/1600), c0 = 10,
  p = c0^2/gamma + (cos 2x + cos 2y)(cos 2z + 2)/16, 64^3, artificial
  properties off, cfl 0.6, filter every step, run to t = 12 with nmax 10000
  (scaled by n/64 on finer grids);
  kinetic energy every 10 steps, the centred difference of it, a 5-point mean,
  and its maximum.  The README quotes eps = 0.01265 at t = 9.13
  (README.md:13-16).
* ``inviscid``: the quick-start Taylor-Green vortex (README.md:31-39: p0 71.43,
  mu0 0, artificial properties on, cfl 0.5) on n^3 to t = 10; kinetic energy
  every step, ``dissipation_rate`` every 100 steps, and the windowed -dKE/dt
  of bench/tgv_energy.jl:168-172 (window 250 steps either side, clamped to a
  eighth of the samples).

Each case runs in FP64 and in mixed precision and the script prints one JSON
line with both peaks and the relative differences between them.

  python compactles.jl_b200/tgv_study.py --case readme64
  python compactles.jl_b200/tgv_study.py --case inviscid --n 256
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


def re1600_problem(cl, c0=10.0, gamma=1.4):
    """The Re 1600 Taylor-Green vortex of examples/taylor_green.jl:22-37."""
    two_pi = 2 * math.pi
    p0 = c0 * c0 / gamma
    return cl.problem.Problem(
        domain=((0.0, two_pi),) * 3, bcs=cl.problem.PER3, name="taylor_green_re1600",
        eos=cl.problem.single_species(gamma=gamma), transport=cl.problem.Transport(mu0=1.0 / 1600.0),
        ic=lambda x, y, z: cl.problem.Prim(
            u=(np.sin(x) * np.cos(y) * np.cos(z), -np.cos(x) * np.sin(y) * np.cos(z), 0.0 * x),
            p=p0 + (np.cos(2 * x) + np.cos(2 * y)) * (np.cos(2 * z) + 2) / 16.0, rho=1.0 + 0.0 * x))


def make_solver(cl, case, n, precision):
    if case == "readme64":
        prob = re1600_problem(cl)
        num = cl.problem.Numerics(n_global=(n, n, n), art=cl.problem.ArtParams(enabled=False), cfl=0.6,
                                  filter_interval=1, precision=precision)
    else:
        prob = cl.problem.taylor_green_problem()
        num = cl.problem.Numerics(n_global=(n, n, n), precision=precision)
    desc = cl.problem.problem_desc(prob, num, cl.lele_d1_6(), cl.compact_filter(0.45))
    s = cl.Solver(desc)
    s.set_state(cl.problem.initialize(desc, prob.ic, eos=prob.eos))
    return s


def readme_peak(times, energy):
    """Centred difference of KE and a 5-point mean (docs/figures/readme_header.jl:78-90)."""
    t = np.asarray(times)
    e = np.asarray(energy)
    d = np.empty_like(e)
    d[0] = -(e[1] - e[0]) / (t[1] - t[0])
    d[1:-1] = -(e[2:] - e[:-2]) / (t[2:] - t[:-2])
    d[-1] = -(e[-1] - e[-2]) / (t[-1] - t[-2])
    m = np.array([d[max(0, i - 2):min(len(d), i + 3)].mean() for i in range(len(d))])
    k = int(np.argmax(m))
    return float(m[k]), float(t[k]), m


def windowed_peak(times, energy, window=250):
    """Peak of windowed_rate (bench/tgv_energy.jl:168-172) with the window clamp."""
    t = np.asarray(times)
    e = np.asarray(energy)
    w = min(window, len(t) // 8)
    best, tbest = -np.inf, float("nan")
    for i in range(len(t)):
        lo, hi = max(i - w, 0), min(i + w, len(t) - 1)
        if hi <= lo:
            continue
        r = -(e[hi] - e[lo]) / (t[hi] - t[lo])
        if r > best:
            best, tbest = r, t[i]
    return float(best), float(tbest)


def run_case(cl, case, n, precision, tfinal=None):
    s = make_solver(cl, case, n, precision)
    t0 = time.perf_counter()
    if case == "readme64":
        tfinal = 12.0 if tfinal is None else tfinal
        times, energy = [0.0], [s.kinetic_energy()]
        nmax = 10_000 * max(1, n // 64)   # the README run's cap at 64^3, scaled with the step count
        while s.t < tfinal and s.steps < nmax:
            s.run(tfinal, min(nmax, s.steps + 10))
            if s.steps % 10 == 0:
                times.append(s.t)
                energy.append(s.kinetic_energy())
        if times[-1] < s.t:
            times.append(s.t)
            energy.append(s.kinetic_energy())
        peak, tpeak, _ = readme_peak(times, energy)
        out = {"eps_peak": peak, "t_peak": tpeak}
    else:
        tfinal = 10.0 if tfinal is None else tfinal
        times, energy, eps = [0.0], [s.kinetic_energy()], []
        while s.t < tfinal:
            s.run(tfinal, s.steps + 1)
            times.append(s.t)
            energy.append(s.kinetic_energy())
            if s.steps % 100 == 0:
                eps.append((s.t, s.dissipation_rate()))
        peak, tpeak = windowed_peak(times, energy)
        ek = max(eps, key=lambda v: v[1]) if eps else (float("nan"), float("nan"))
        out = {"dkedt_peak": peak, "t_dkedt_peak": tpeak, "eps_sampled_peak": ek[1], "t_eps_sampled_peak": ek[0]}
    wall = time.perf_counter() - t0
    out.update({"steps": s.steps, "t_end": s.t, "ke_end": energy[-1], "wall_s": wall,
                "cell_steps_per_s": n ** 3 * s.steps / wall})
    return out, np.asarray(times), np.asarray(energy)


def main(argv=None):
    p = argparse.ArgumentParser()
    p.add_argument("--case", choices=["readme64", "inviscid"], default="readme64")
    p.add_argument("--n", type=int, default=None)
    p.add_argument("--tfinal", type=float, default=None)
    p.add_argument("--precisions", default="fp64,mixed")
    a = p.parse_args(argv)
    cl = _package()
    n = a.n or (64 if a.case == "readme64" else 256)
    res, hist = {}, {}
    for prec in a.precisions.split(","):
        res[prec], t, e = run_case(cl, a.case, n, prec, a.tfinal)
        hist[prec] = (t, e)
    out = {"case": a.case, "n": n, "results": res}
    if "fp64" in res and "mixed" in res:
        f, m = res["fp64"], res["mixed"]
        keys = ["eps_peak"] if a.case == "readme64" else ["dkedt_peak", "eps_sampled_peak"]
        out["mixed_vs_fp64"] = {k: abs(m[k] - f[k]) / abs(f[k]) for k in keys}
        out["mixed_vs_fp64"]["ke_end"] = abs(m["ke_end"] - f["ke_end"]) / abs(f["ke_end"])
        (tf, ef), (tm, em) = hist["fp64"], hist["mixed"]
        k = min(len(ef), len(em))
        # KE histories at matching sample indices (the step sequences differ slightly)
        out["mixed_vs_fp64"]["ke_max_rel_at_matching_samples"] = float(
            np.max(np.abs(np.interp(tf[:k], tm, em) - ef[:k]) / np.abs(ef[:k])))
    if a.case == "readme64":
        out["readme"] = {"eps_peak": 0.01265, "t_peak": 9.13}
    print(json.dumps(out), flush=True)
    return out


if __name__ == "__main__":
    main()
