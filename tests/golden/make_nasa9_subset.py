"""Generate tests/golden/nasa9_subset.json: the NASA-9 records of a few gases
as parsed from the NASA CEA thermo.inp database that ships with the
reference (data/thermo.inp), in the tabulated (formation) enthalpy gauge.

The coefficient file itself is not copied; the fixture holds the parsed
numbers for the species the thermodynamic tests use, with each record's
specific gas constant R = 1000 R_u / M.  Run from the repository root:

    python tests/golden/make_nasa9_subset.py <CompactLES.jl source tree>/data/thermo.inp
"""
import importlib.util
import json
import pathlib
import sys

ROOT = pathlib.Path(__file__).resolve().parents[2]
SPECIES = ["He", "CO2", "Air", "N2", "O2", "Jet-A(g)", "ALOCL", "SnCL2"]


def main(path):
    spec = importlib.util.spec_from_file_location("nasa9", ROOT / "compactles.jl_b200" / "nasa9.py")
    n9 = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(n9)
    out = []
    for sp in n9.read_nasa9(SPECIES, path, reference="formation"):
        out.append({"name": sp.name, "R": sp.R,
                    "intervals": [{"Tmin": iv.Tmin, "Tmax": iv.Tmax, "a": list(iv.a), "b1": iv.b1}
                                  for iv in sp.intervals]})
    dst = pathlib.Path(__file__).with_name("nasa9_subset.json")
    dst.write_text(json.dumps({"source": "NASA CEA thermo.inp (Glenn Research Center), formation gauge",
                               "species": out}, indent=1))
    print("wrote", dst)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_nasa9_subset.py <CompactLES.jl source tree>/data/thermo.inp")
    main(sys.argv[1])
