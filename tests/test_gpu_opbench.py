"""The operator microbenchmark's seeded Fourier fields (periodic and closed,
C6 / C10 / C8 filter, every direction) through the batched device plan,
checked against the CPU oracle on whole lines of a thin slab.  FP64 plans
must agree to 1e-12 relative to the oracle's maximum; FP32 plans report
their error against FP64 and must stay below 1e-5."""
import argparse

import numpy as np
import pytest

import compactles_b200 as cl
from compactles_b200 import opbench

pytestmark = pytest.mark.gpu


def _oracle_slab(orc, f, sname, dim, periodic, h):
    # lines along `dim` need their full extent and only a few points across
    sl = [slice(0, 8)] * 3
    sl[3 - dim] = slice(None)            # numpy axes are (z, y, x)
    sub = f[tuple(sl)]
    ng = (sub.shape[2], sub.shape[1], sub.shape[0])
    per = [True, True, True]
    per[dim - 1] = periodic
    g = orc.grid(ng, per)
    F = np.zeros(orc.padded_shape(g))
    orc.interior(g, F)[...] = sub
    orc.exchange_halos(g, F)
    mk = {"c6": orc.lele_d1_6, "c10": orc.lele_d1_10, "filter": lambda: orc.compact_filter(0.45)}[sname]
    return orc.interior(g, orc.Plan(g, mk(), dim, h).apply(F)), tuple(sl)


def test_opbench_fields_match_oracle(orc):
    args = argparse.Namespace(n=64, fields=2, reps=1, ncu_case=False, keep=True, schemes=None,
                              cases=[(True, "f64"), (False, "f64"), (True, "f32"), (False, "f32")])
    recs = opbench.run(args)
    assert len(recs) == 36
    for rec in recs:
        if rec["dtype"] == "f32":
            assert rec["rel_err_vs_fp64"] < 1e-5, rec
            continue
        f = rec["in"][0].double().cpu().numpy()
        got = rec["out"][0].double().cpu().numpy()
        ref, sl = _oracle_slab(orc, f, rec["scheme"], rec["dim"], rec["periodic"], rec["h"])
        err = np.abs(got[sl] - ref).max() / np.abs(ref).max()
        assert err < 1e-12, (rec["scheme"], rec["dim"], rec["periodic"], err)
