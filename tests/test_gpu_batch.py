"""Batched solves (cles_batch_*): many grids of different sizes advanced by one
captured step of O(stages) launches.

Checked here, against the one-grid solver and the CPU oracle on the same
inputs:
* every member of a batch of uneven 2-D He/CO2 shock-interface grids matches
  the one-grid solver and the oracle to 1e-10 relative L2 after 30 steps
  (FP64), and, with a fixed launch form (batched kernels or per-member
  kernels), its results are bitwise the same alone and in the mix; the two
  forms and the autotuner's mix of them agree to 1e-12;
* members with different end times retire as they finish (the composition
  changes and the step is re-captured), each ending exactly at its end time
  with the state of its solo run;
* with the batched form, the kernels in one captured step do not grow with
  the number of members;
* 3-D Taylor-Green boxes and 1-D two-species tubes in batches, FP64 and the
  mixed form (FP32 fields, FP64 state; 1e-5 relative L2 against the FP64
  oracle after 20 steps, FP32 rounding of the terms accumulated over the
  updates), and cancellation of a running member.
"""
import numpy as np
import pytest

import compactles_b200 as cl
import parity
from compactles_b200 import scenarios

pytestmark = pytest.mark.gpu

SHAPES = [(96, 48, 1.5, 11), (128, 64, 2.0, 12), (70, 40, 1.3, 13), (160, 32, 2.4, 14)]


def _rel(a, b, desc):
    sl = (slice(None),) + cl.interior_slices(desc)
    a, b = a[sl], b[sl]
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _cases(m, precision="fp64", shapes=SHAPES):
    sch = (m.lele_d1_6(), m.compact_filter(0.45))
    return [scenarios.shock_interface_2d(sch, nx, ny, M, sd, precision=precision) for nx, ny, M, sd in shapes]


def _batch(reqs, steps=None, strategy="auto"):
    B = cl.Batch(reqs[0][0], strategy=strategy)
    ids = [B.add(d, Q0, tf) for d, Q0, tf in reqs]
    if steps is None:
        assert B.run() == 0
    else:
        B.run(steps)
    return B, ids


def test_batch_matches_solo_and_oracle(orc):
    reqs = _cases(cl)
    B, ids = _batch(reqs, steps=30)
    st = B.stats()
    assert st["members"] == 4 and st["steps"] == 30
    ocases = _cases(orc)
    for k, ((d, Q0, tf), mid) in enumerate(zip(reqs, ids)):
        assert B.status(mid)["steps"] == 30
        got = B.fetch(mid)
        S = cl.Solver(d)
        S.set_state(Q0)
        S.run(tf, 30)
        rs = _rel(got, S.get_state(), d)
        line = {"solo_l2": rs}
        if k in (0, 2):
            O = orc.Solver(ocases[k][0])
            O.set_state(Q0)
            assert O.run(tf, 30)[0] == 0
            ro = _rel(got, O.get_state(), d)
            line["oracle_l2"] = ro
            assert ro < 1e-10, ro
        parity.record(f"batch shock-interface {d.n_global[0]}x{d.n_global[1]} FP64 30 steps", **line)
        assert rs < 1e-10, rs


@pytest.mark.parametrize("strategy", ["batched", "per_member"])
def test_batch_member_alone_equals_in_mix(strategy):
    # with a fixed launch form a member's arithmetic does not depend on the others
    reqs = _cases(cl)
    B, ids = _batch(reqs, steps=12, strategy=strategy)
    for k in (1, 2):
        A, aid = _batch([reqs[k]], steps=12, strategy=strategy)
        assert np.array_equal(A.fetch(aid[0]), B.fetch(ids[k]))


def test_batch_strategies_agree():
    # the batched kernels, the per-member kernels and the autotuner's mix of
    # them give the same states to rounding
    reqs = _cases(cl)
    out = {}
    for strategy in ("batched", "per_member", "auto"):
        B, ids = _batch(reqs, steps=20, strategy=strategy)
        out[strategy] = [B.fetch(i) for i in ids]
        if strategy == "auto":
            assert {t["threads"] for t in B.stats()["tuning"]} <= {0, 128, 256, 512}
    for k, (d, _, _) in enumerate(reqs):
        for strategy in ("per_member", "auto"):
            r = _rel(out[strategy][k], out["batched"][k], d)
            assert r < 1e-12, (strategy, k, r)


def test_batch_members_retire_at_their_end_times():
    reqs = [(d, Q0, 2e-5 * (i + 1)) for i, (d, Q0, _) in enumerate(_cases(cl))]
    B, ids = _batch(reqs)
    st = B.stats()
    assert st["active"] == 0 and st["compositions"] >= 2
    for (d, Q0, tf), mid in zip(reqs, ids):
        s = B.status(mid)
        assert s["state"] == "done" and abs(s["t"] - tf) <= 1e-15 * tf
        S = cl.Solver(d)
        S.set_state(Q0)
        res = S.run(tf)
        assert res.steps == s["steps"]
        assert _rel(B.fetch(mid), S.get_state(), d) < 1e-10


def test_batch_launches_do_not_grow_with_members():
    reqs = _cases(cl)
    B2, _ = _batch(reqs[:2], steps=1, strategy="batched")
    B4, _ = _batch(reqs, steps=1, strategy="batched")
    n2, n4 = B2.stats()["launches_per_step"], B4.stats()["launches_per_step"]
    assert n2 == n4 and 0 < n4 < 200
    tun = B4.stats()["tuning"]
    assert {t["threads"] for t in tun} <= {128, 256, 512} and len(tun) == 6


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batch_taylor_green_boxes(orc, precision):
    reqs = [scenarios.taylor_green_box((cl.lele_d1_6(), cl.compact_filter(0.45)), n, precision=precision)
            for n in (24, 32)]
    B, ids = _batch(reqs, steps=20)
    for (d, Q0, tf), mid, n in zip(reqs, ids, (24, 32)):
        do = scenarios.taylor_green_box((orc.lele_d1_6(), orc.compact_filter(0.45)), n)[0]
        O = orc.Solver(do)
        O.set_state(Q0)
        assert O.run(tf, 20)[0] == 0
        r = _rel(B.fetch(mid), O.get_state(), d)
        parity.record(f"batch TGV {n}^3 {precision} 20 steps", oracle_l2=r)
        assert r < (1e-10 if precision == "fp64" else 1e-5), r


def test_batch_two_species_tubes_and_cancel(orc):
    sch = (cl.lele_d1_6(), cl.compact_filter(0.45))
    reqs = [scenarios.two_species_tube(sch, N, pr, 0.4) for N, pr in ((256, 5.0), (700, 12.0), (333, 3.0))]
    B = cl.Batch(reqs[0][0])
    ids = [B.add(d, Q0, tf) for d, Q0, tf in reqs]
    B.run(10)
    B.cancel(ids[2])
    frozen = B.fetch(ids[2])
    B.run(15)
    assert B.status(ids[2])["state"] == "cancelled" and B.status(ids[2])["steps"] == 10
    assert np.array_equal(B.fetch(ids[2]), frozen)
    osch = (orc.lele_d1_6(), orc.compact_filter(0.45))
    for k in (0, 1):
        d, Q0, tf = reqs[k]
        O = orc.Solver(scenarios.two_species_tube(osch, d.n_global[0], (5.0, 12.0)[k], 0.4)[0])
        O.set_state(Q0)
        assert O.run(tf, 25)[0] == 0
        assert B.status(ids[k])["steps"] == 25
        r = _rel(B.fetch(ids[k]), O.get_state(), d)
        parity.record(f"batch tube N={d.n_global[0]} FP64 25 steps", oracle_l2=r)
        assert r < 1e-10, r


def test_batch_members_with_their_own_gas_constants(orc):
    # species gas constants are per member: tubes of different Atwood numbers
    # share one batch and each matches the oracle
    sch = (cl.lele_d1_6(), cl.compact_filter(0.45))
    osch = (orc.lele_d1_6(), orc.compact_filter(0.45))
    spec = [(300, 4.0, 0.6), (512, 9.0, -0.5), (1000, 15.0, 0.1)]
    reqs = [scenarios.two_species_tube(sch, N, pr, A) for N, pr, A in spec]
    B = cl.Batch(reqs[0][0])
    ids = [B.add(d, Q0, tf) for d, Q0, tf in reqs]
    B.run(40)
    for (N, pr, A), (d, Q0, tf), mid in zip(spec, reqs, ids):
        O = orc.Solver(scenarios.two_species_tube(osch, N, pr, A)[0])
        O.set_state(Q0)
        assert O.run(tf, 40)[0] == 0
        r = _rel(B.fetch(mid), O.get_state(), d)
        parity.record(f"batch tube N={N} Atwood {A} FP64 40 steps", oracle_l2=r)
        assert r < 1e-10, r


def test_batch_rejects_a_member_of_another_class():
    sch = (cl.lele_d1_6(), cl.compact_filter(0.45))
    d0, Q0, tf = scenarios.two_species_tube(sch, 256, 5.0, 0.4)
    d1, Q1, _ = scenarios.two_species_tube(sch, 256, 5.0, 0.4, precision="mixed")
    B = cl.Batch(d0)
    B.add(d0, Q0, tf)
    with pytest.raises(cl.ClesError, match="precision"):
        B.add(d1, Q1, tf)
