"""Regenerates the golden fixtures in this folder from a CompactLES.jl checkout.

The reference stores two high-resolution profiles produced by its own solver
(test/refs/shu_osher.csv: Shu-Osher at t=1.8 run at N=3200 and interpolated
to N=800; test/refs/woodward_colella.csv: Woodward-Colella at t=0.038, same
construction).  They are the only stored outputs of the reference for this
path, so they are copied here unchanged (data only) and the tests read them
from here; nothing reads the reference tree at test time.

usage: python tests/golden/make_golden.py /path/to/CompactLES.jl
"""
import pathlib
import shutil
import sys

HERE = pathlib.Path(__file__).resolve().parent


def main(ref_root):
    src = pathlib.Path(ref_root) / "test" / "refs"
    for name in ("shu_osher.csv", "woodward_colella.csv"):
        shutil.copyfile(src / name, HERE / name)
        print("wrote", HERE / name)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py <root of the CompactLES.jl source tree>")
    main(sys.argv[1])
