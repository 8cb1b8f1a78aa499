"""One run! step of a solver between cudaProfilerStart / cudaProfilerStop, for
an ncu launch list of every kernel the step runs (ncu --profile-from-start off).

Cases:
  tgv        the README Taylor-Green box on an n^3 periodic grid (default 192:
             5 FP64 fields of 283 MB, larger than the 126 MB L2; the working
             set is about 3.6 GB), single species, artificial properties on;
  interface  a 2-D He/CO2 shock-interface grid (n x n/2, two species, slip
             walls in x): adds the species sensors and diffusion fluxes;
  batch      the 64-case ensemble of 2-D shock-interface grids in one batch;
  tube       a 1-D two-species shock tube of n cells (pressure ratio 10,
             Atwood 0.5): one line, the latency-bound end of the serving mix.

  python compactles.jl_b200/stepprof.py [--case tgv|interface|batch|tube] [--n 192] [--precision fp64|mixed]
"""
import argparse
import importlib.util
import pathlib
import sys

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


def main(argv=None):
    p = argparse.ArgumentParser()
    p.add_argument("--case", choices=["tgv", "interface", "batch", "tube"], default="tgv")
    p.add_argument("--n", type=int, default=192)
    p.add_argument("--precision", choices=["fp64", "mixed"], default="fp64")
    a = p.parse_args(argv)
    import torch
    cl = _package()
    sch = (cl.lele_d1_6(), cl.compact_filter(0.45))
    torch.cuda.set_device(0)
    if a.case == "batch":
        sys.path.insert(0, str(HERE))
        import ensemble
        reqs = [cl.scenarios.shock_interface_2d(sch, nx, ny, M, sd, precision=a.precision)
                for nx, ny, M, sd in ensemble.draw_cases(64, 7)]
        B = cl.Batch(reqs[0][0])
        for d, Q0, tf in reqs:
            B.add(d, Q0, tf)
        for _ in range(3):
            B.step()
        torch.cuda.synchronize()
        torch.cuda.cudart().cudaProfilerStart()
        B.step()
    else:
        if a.case == "tgv":
            desc, Q0, tf = cl.scenarios.taylor_green_box(sch, a.n, tfinal=1e9, precision=a.precision)
        elif a.case == "tube":
            desc, Q0, tf = cl.scenarios.two_species_tube(sch, a.n, 10.0, 0.5, precision=a.precision)
        else:
            desc, Q0, tf = cl.scenarios.shock_interface_2d(sch, a.n, a.n // 2, 2.0, 5, precision=a.precision)
        S = cl.Solver(desc)
        S.set_state(Q0)
        S.run(tf, 2)
        torch.cuda.synchronize()
        torch.cuda.cudart().cudaProfilerStart()
        S.run(tf, 3)
    torch.cuda.synchronize()
    torch.cuda.cudart().cudaProfilerStop()
    print("profiled one step", flush=True)


if __name__ == "__main__":
    main()
