"""Benchmark: cell-steps/s of the 256^3 Taylor-Green step on B200.

Workload: the README quick-start Taylor-Green vortex (rho = 1, p = 71.43,
u = (sin x cos y, -cos x sin y, 0) on [0, 2pi)^3, periodic) with the
reference's default numerics (Lele C6 derivatives, C8 filter every step,
Cook artificial properties, LSRK(5,4), cfl 0.5) at 256^3.  One step is one
run! iteration: boundary conditions, max_rate (with its host read of the
rate), five RK stages and filter_state!.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun (N > 1) every rank advances its own 256^3 box (replicas,
weak scaling); the time is the max over ranks.  `--impl reference` times the
CPU oracle (the FP64 restatement of the reference; the Julia reference cannot
run on this machine) on every host core, on the same 256^3 box.
"""
import argparse
import importlib.util
import json
import math
import os
import pathlib
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parent
METRIC = "cell-steps/s 256³ TGV (mixed vs FP64, same GPU); ensemble solves/s + p99 lat"
UNIT = "cell-steps/s"
WORKLOAD = "taylor_green_256^3: README IC (rho 1, p 71.43), C6 deriv + C8 filter every step, Cook art, LSRK(5,4), cfl 0.5"


def _package():
    if "compactles_b200" in sys.modules:
        return sys.modules["compactles_b200"]
    pkg = ROOT / "compactles.jl_b200"
    spec = importlib.util.spec_from_file_location("compactles_b200", pkg / "__init__.py",
                                                  submodule_search_locations=[str(pkg)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["compactles_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def parse(argv=None):
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--n", type=int, default=256, help="grid points per dimension")
    p.add_argument("--cpu-n", type=int, default=128, help="grid of the one-thread CPU sample")
    p.add_argument("--cpu-steps", type=int, default=3, help="timed steps of the all-core CPU sample")
    p.add_argument("--e2e-steps", type=int, default=5)
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-mixed", action="store_true")
    a = p.parse_args(argv)
    if a.warmup < 3:
        p.error("--warmup must be >= 3")
    return a


# ----------------------------------------------------------- distribution ----
class Dist:
    """Rank bookkeeping: torchrun env or a single process."""

    def __init__(self, backend=None):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local_rank = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        if self.world > 1:
            import datetime

            import torch.distributed as dist
            if backend is None:
                import torch
                backend = "nccl" if torch.cuda.is_available() else "gloo"
            os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
            dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=600))
            self.pg = dist
            self.backend = backend

    def barrier(self):
        if self.pg:
            if getattr(self, "backend", "") == "nccl":
                import torch
                self.pg.barrier(device_ids=[torch.cuda.current_device()])
            else:
                self.pg.barrier()

    def max(self, x):
        """Max of a float over ranks."""
        if not self.pg:
            return float(x)
        import torch
        dev = "cuda" if getattr(self, "backend", "") == "nccl" else "cpu"
        t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


def aggregate(cells, steps, world, max_ms):
    """Whole-job cell-steps/s of `world` replicas each doing cells*steps in max_ms."""
    return world * cells * steps / (max_ms / 1e3)


# ----------------------------------------------------------------- clocks ----
class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
        except Exception:
            self.proc = None

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.th.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


# ------------------------------------------------------------------ cases ----
def tgv_desc(cl, n, precision="fp64"):
    prob = cl.taylor_green_problem()
    tp = 2 * math.pi
    return cl.solver_desc((n, n, n), (tp, tp, tp), prob.bcs, cl.lele_d1_6(), cl.compact_filter(0.45),
                          precision=precision), prob


def measured_peaks():
    try:
        return json.loads((ROOT / "MEASURED_PEAKS.json").read_text()), "measured"
    except Exception:
        return {"hbm_gbs": 6650.0}, "fallback"


# DRAM traffic over algorithmic bytes of the C6 compact kernels on 5 FP64
# fields of 256^3, from one ncu capture of the operator benchmark
# (dram__bytes_read.sum + dram__bytes_write.sum; x / y / z 0.963 / 0.958 /
# 0.959).  Traffic grows in proportion to fields x points, so a launch's
# traffic is this ratio times its algorithmic bytes.
NCU_TRAFFIC_RATIO = 0.960


def ncu_traffic():
    """Per-launch DRAM bytes of the compact kernel, as a ratio to its algorithmic bytes (one ncu capture)."""
    return {"traffic_ratio": NCU_TRAFFIC_RATIO,
            "note": "dram__bytes_read.sum + dram__bytes_write.sum over algorithmic bytes, from one ncu capture "
                    "of the C6 compact kernels on 5 FP64 fields of 256^3 (x/y/z: 0.963/0.958/0.959); the "
                    "per-launch traffic is this ratio times the average algorithmic bytes of the timed launches "
                    "(traffic grows in proportion to fields x points)"}


# -------------------------------------------------------------- our arm ------
def time_solver(cl, torch, desc, Q0, steps, warmup, dist, profile=False):
    ctx = cl.Context(torch.cuda.current_device(), stream=torch.cuda.current_stream().cuda_stream)
    S = cl.Solver(desc, ctx=ctx)
    S.set_state(Q0)
    S.run(1e9, warmup)
    cells = S.info().cells
    dist.barrier()
    torch.cuda.synchronize()
    launches0 = cl.kernel_launches()
    if profile:
        cl.profile_enable(True)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    sampler = ClockSampler(torch.cuda.current_device())
    sampler.start()
    time.sleep(0.3)
    e0.record()
    res = S.run(1e9, warmup + steps)
    e1.record()
    torch.cuda.synchronize()
    clocks = sampler.stop()
    ms = e0.elapsed_time(e1)
    launches = cl.kernel_launches() - launches0
    prof = cl.profile_read() if profile else None
    if profile:
        cl.profile_enable(False)
    dist.barrier()
    assert res.steps == steps, res.steps
    ke = S.kinetic_energy()
    del S
    return dict(ms=ms, cells=cells, launches=launches, prof=prof, clocks=clocks, ke=ke, ctx=ctx)


def time_e2e(cl, torch, desc, Q0, steps, dist):
    """Through the public host-buffer call: per step H2D of the state from pinned
    padded host memory, one run! step, D2H of the state."""
    ctx = cl.Context(torch.cuda.current_device(), stream=torch.cuda.current_stream().cuda_stream)
    S = cl.Solver(desc, ctx=ctx)
    Qh = torch.empty(Q0.shape, dtype=torch.float64, pin_memory=True).numpy()
    Qh[...] = Q0
    for _ in range(2):
        S.step_host(Qh, 1e9)
    dist.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        S.step_host(Qh, 1e9)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    info = S.info()
    # host to device: each component's whole padded block (contiguous copy,
    # interior gathered on the device); device to host: the interior, plus the
    # 16-byte rate read of the step
    h2d = int(Qh.nbytes)
    d2h = info.cells * info.n_cons * 8 + 16
    del S
    return ms, (h2d, d2h)


def _oracle_tgv(n):
    cl = _package()          # first: the oracle shares the package's descriptor structs
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as orc
    prob = cl.taylor_green_problem()
    tp = 2 * math.pi
    desc = cl.solver_desc((n, n, n), (tp, tp, tp), prob.bcs, orc.lele_d1_6(), orc.compact_filter(0.45))
    O = orc.Solver(desc)
    O.set_state(cl.initialize(desc, prob.ic))
    return orc, O


def cpu_sample(n, steps, threads=None):
    """The oracle on the host cores: `steps` run! steps of the n^3 box after one
    warm-up step, on `threads` OpenMP threads (None: every host core)."""
    orc, O = _oracle_tgv(n)
    threads = orc.set_threads(threads or os.cpu_count() or 1)
    O.run(1e9, 1)
    t0 = time.perf_counter()
    O.run(1e9, 1 + steps)
    dt = time.perf_counter() - t0
    orc.set_threads(os.cpu_count() or 1)
    return n ** 3 * steps / dt, threads, dt


def run_ours(a):
    import torch
    cl = _package()
    dist = Dist()
    torch.cuda.set_device(dist.local_rank)
    desc, prob = tgv_desc(cl, a.n)
    Q0 = cl.initialize(desc, prob.ic)
    r = time_solver(cl, torch, desc, Q0, a.steps, a.warmup, dist, profile=True)
    max_ms = dist.max(r["ms"])
    value = aggregate(r["cells"], a.steps, dist.world, max_ms)
    out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": dist.world, "steps": a.steps,
           "warmup": a.warmup, "ms_per_step": max_ms / a.steps, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f64", "data": "synthetic (analytic Taylor-Green initial condition)",
           "config": {"workload": WORKLOAD, "grid": [a.n] * 3, "form": "fp64 drop-in",
                      "parallelism": f"replicas x{dist.world}" if dist.world > 1 else "single GPU",
                      "l2": "inputs larger than L2: state 5 x 256^3 FP64 = 671 MB, working set ~8.6 GB"},
           "gpu_launches": r["launches"], "clocks": r["clocks"]}
    # roofline of the dominant kernel: the compact line-solve operator
    peaks, src = measured_peaks()
    prof = r["prof"] or {}
    tot_ms = sum(v[1] for v in prof.values())
    tot_b = sum(v[2] for v in prof.values())
    nl = sum(v[0] for v in prof.values())
    if tot_ms > 0:
        achieved = tot_b / (tot_ms / 1e3) / 1e9
        peak = float(peaks.get("hbm_gbs", 6650.0))
        traffic = ncu_traffic()
        per_launch = tot_b / nl
        out["roofline"] = {"bound": "hbm", "kernel": "k_compact (all directions)", "achieved": achieved,
                           "peak": peak, "unit": "GB/s", "frac": achieved / peak, "peak_source": src,
                           "traffic": (traffic["traffic_ratio"] * per_launch) if traffic else None,
                           "traffic_note": (traffic or {}).get("note"),
                           "algorithmic_bytes_per_launch": tot_b / nl, "avg_launch_ms": tot_ms / nl,
                           "launches": nl, "share_of_step": tot_ms / r["ms"],
                           "per_direction": {k: {"launches": v[0], "ms": v[1], "GB/s": v[2] / (v[1] / 1e3) / 1e9}
                                             for k, v in prof.items()}}
    out["diagnostics"] = {"kinetic_energy_after": r["ke"]}
    if not a.no_mixed:
        try:
            dm, _ = tgv_desc(cl, a.n, precision="mixed")
            rm = time_solver(cl, torch, dm, Q0, a.steps, a.warmup, dist)
            mm = dist.max(rm["ms"])
            vm = aggregate(rm["cells"], a.steps, dist.world, mm)
            out["forms"] = {"fp64": value, "mixed": vm, "mixed_over_fp64": vm / value,
                            "mixed_ms_per_step": mm / a.steps}
        except Exception as e:  # reported, never silently dropped
            out["forms"] = {"fp64": value, "mixed_error": str(e)[:200]}
    if not a.no_e2e:
        k = min(a.e2e_steps, a.steps)
        ms, sb = time_e2e(cl, torch, desc, Q0, k, dist)
        mm = dist.max(ms)
        out["e2e"] = {"value": aggregate(r["cells"], k, dist.world, mm), "unit": UNIT,
                      "h2d_bytes_per_step": sb[0], "d2h_bytes_per_step": sb[1],
                      "how": "cles_step_host: pinned padded host state in, one run! step, state out"}
    if dist.rank == 0 and dist.world == 1 and not a.no_cpu:
        v, th, secs = cpu_sample(a.n, a.cpu_steps)
        v1, _, secs1 = cpu_sample(a.cpu_n, 1, threads=1)
        out["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": th, "kind": "port",
                               "sample": f"{a.cpu_steps} run! steps (after 1 untimed) of the same {a.n}^3 "
                                         f"Taylor-Green case on the CPU oracle (FP64, OpenMP, {th} threads), "
                                         f"{secs:.1f} s",
                               "single_thread": {"value": v1, "unit": UNIT, "cores": 1,
                                                 "sample": f"1 run! step (after 1 untimed) of the same case at "
                                                           f"{a.cpu_n}^3 on one thread, {secs1:.1f} s"}}
    if dist.rank == 0:
        print(json.dumps(out), flush=True)
    dist.close()


def run_reference(a):
    """The oracle on the host cores, every core: W untimed steps, then K timed
    run! steps of the same a.n^3 box the GPU arm times."""
    dist = Dist(backend="gloo")
    if dist.rank != 0:
        dist.close()
        return
    orc, O = _oracle_tgv(a.n)
    threads = orc.set_threads(os.cpu_count() or 1)
    O.run(1e9, a.warmup)
    t0 = time.perf_counter()
    O.run(1e9, a.warmup + a.steps)
    secs = time.perf_counter() - t0
    value = a.n ** 3 * a.steps / secs
    out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": dist.world, "steps": a.steps,
           "warmup": a.warmup, "ms_per_step": 1e3 * secs / a.steps, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (analytic Taylor-Green)",
           "impl": "reference",
           "config": {"workload": WORKLOAD, "grid": [a.n] * 3, "form": "fp64 CPU"},
           "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                            "sample": f"{a.steps} timed run! steps (after {a.warmup} untimed) of the same "
                                      f"{a.n}^3 Taylor-Green case on the FP64 CPU oracle, {secs:.1f} s; the Julia "
                                      f"reference itself cannot run on this machine"},
           "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)
    dist.close()


def main(argv=None):
    a = parse(argv)
    if a.impl == "reference":
        run_reference(a)
    else:
        run_ours(a)


if __name__ == "__main__":
    main()
