"""CPU-only checks of the C ABI: the library loads without a GPU, exports every
entry point include/cles.h declares, its descriptor structs have the layout
the ctypes mirror assumes, and its scheme presets equal the oracle's
restatement of src/kernels.jl / src/kernels_banded.jl.  Host-only entry points
(presets, defaults, check_step) are exercised; nothing here touches CUDA."""
import ctypes as C
import pathlib
import re
import subprocess

import numpy as np
import pytest

import compactles_b200 as cl
from compactles_b200 import abi

ROOT = pathlib.Path(__file__).resolve().parent.parent
HEADER = ROOT / "include" / "cles.h"


def declared_symbols():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(cles_[a-z0-9_]+)\s*\(", text)))


def test_library_loads_and_exports_every_declared_symbol():
    L = cl.lib()
    missing = [s for s in declared_symbols() if not hasattr(L, s)]
    assert not missing, missing
    assert len(declared_symbols()) >= 30


def test_struct_layout_matches_the_c_header(tmp_path):
    src = tmp_path / "sz.c"
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "cles.h"\n'
                   "int main(void){printf(\"%zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu\\n\","
                   "sizeof(cles_scheme), sizeof(cles_grid), sizeof(cles_step_control), sizeof(cles_solver_desc),"
                   "sizeof(cles_solver_info), sizeof(cles_run_result), offsetof(cles_solver_desc, deriv),"
                   "offsetof(cles_solver_desc, precision), sizeof(cles_split_desc), sizeof(cles_split_info),"
                   "offsetof(cles_split_info, prev), sizeof(cles_decomp), offsetof(cles_decomp, rank),"
                   "sizeof(cles_exchange), offsetof(cles_exchange, allreduce));return 0;}\n")
    exe = tmp_path / "sz"
    subprocess.run(["gcc", "-I", str(HEADER.parent), str(src), "-o", str(exe)], check=True)
    got = list(map(int, subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()))
    want = [C.sizeof(abi.cles_scheme), C.sizeof(abi.cles_grid), C.sizeof(abi.cles_step_control),
            C.sizeof(abi.cles_solver_desc), C.sizeof(abi.cles_solver_info), C.sizeof(abi.cles_run_result),
            abi.cles_solver_desc.deriv.offset, abi.cles_solver_desc.precision.offset, C.sizeof(abi.cles_split_desc),
            C.sizeof(abi.cles_split_info), abi.cles_split_info.prev.offset, C.sizeof(abi.cles_decomp),
            abi.cles_decomp.rank.offset, C.sizeof(abi.cles_exchange), abi.cles_exchange.allreduce.offset]
    assert got == want


def _scheme_tuple(s):
    q, M, nc = s.q, s.M, s.nc
    return (q, [s.lhs[i] for i in range(q)], s.a0, M, [s.coeffs[i] for i in range(M)], s.symmetric, nc,
            [[s.clo_lhs[j][t] for t in range(2 * q + 1)] for j in range(nc)],
            [[s.clo_rhs[j][t] for t in range(s.clo_len[j])] for j in range(nc)])


@pytest.mark.parametrize("name", ["lele_d1_6", "pade_d1_4", "compact_filter", "lele_d1_10"])
def test_library_presets_equal_oracle(orc, name):
    mine = getattr(cl, name)()
    theirs = getattr(orc, name)()
    assert _scheme_tuple(mine) == _scheme_tuple(theirs)


def test_filter_closure_consistency():
    # every filter row's RHS sums to 1 + 2 alpha_f (src/kernels.jl:96)
    s = cl.compact_filter(0.45)
    for j in range(1, s.nc):
        assert abs(sum(s.clo_rhs[j][t] for t in range(s.clo_len[j])) - 1.9) < 1e-15
    assert abs(s.a0 + 2 * sum(s.coeffs[m] for m in range(s.M)) - 1.9) < 1e-15


def test_desc_default_matches_numerics_defaults():
    d = abi.cles_solver_desc()
    cl.lib().cles_solver_desc_default(C.byref(d))
    assert d.cfl == 0.5 and d.filter_interval == 1 and d.art_enabled == 1 and d.n_halo == 4
    assert (d.C_mu, d.C_beta, d.C_kappa, d.C_D) == (0.002, 1.0, 0.01, 0.01)
    assert d.control.dt_min_ratio == 1e-8 and d.control.landing_steps == 2 and d.control.savepoint_interval == 25
    assert d.mu0 == 0.0 and d.Pr == 0.7 and d.Sc == 0.7


def test_check_step_in_the_library_matches_the_oracle(orc):
    c = abi.step_control_default()
    rng = np.random.default_rng(1)
    for dt, rho, seen in [(1e-3, 1.0, 1.0), (float("nan"), 1.0, 1.0), (1e-3, -1e-9, 1.0), (1e-50, 1.0, 1.0),
                          (1e-40, 1.0, 1.0), (1e-9, 1.0, 0.0)] + [tuple(rng.uniform(-1, 1, 3)) for _ in range(20)]:
        assert cl.check_step(c, dt, rho, seen) == orc.check_step(c, dt, rho, seen)


def test_context_creation_fails_loudly_without_a_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is visible")
    with pytest.raises(cl.ClesError):
        cl.Context(0)
