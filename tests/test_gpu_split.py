"""Lines split across ranks (cles_split_* through the C ABI) on the device.

The P ranks of a decomposed dimension run in one process on cuda:0: each
rank has its own plan, padded block and exchange buffers, and the two
exchanges of LineExchange (the halo Sendrecv! and the interface Allgather!)
are done as device copies between the ranks' buffers, in the same phases a
multi-process run takes.  No kernel waits on another rank.

* every scheme (C6, C4, C10, C8 filter), every dimension, periodic and
  closed lines, P = 1 (periodic self-neighbour), 2, 3, 4 and uneven splits
  match the oracle's P-rank solve (src/tridiag.jl:136-170,
  src/banded.jl:177-214) to 1e-12 in FP64 and 2e-6 in FP32, and the
  undecomposed device plan to the same bound;
* long split lines (segmented and cyclic-reduction local solves) and
  batches of fields;
* the reference's MPI suite cases (test/mpi_tests.jl:117-192): periodic C6
  and C10 derivatives of sin(3x) cos(2y) split 2, 4 and 8 ways on 72 points,
  closed C6 and C10 cubic exactness with the derivative dimension split;
* the reference's plan-time errors (src/operators.jl:50-53).
"""
import numpy as np
import pytest

import compactles_b200 as cl

pytestmark = pytest.mark.gpu


def _schemes(mod, name):
    return {"c6": mod.lele_d1_6, "c10": mod.lele_d1_10, "filt": lambda: mod.compact_filter(0.45),
            "pade": mod.pade_d1_4}[name]()


def local_range(N, P, r):
    base, rem = divmod(N, P)
    return base + (1 if r < rem else 0), r * base + min(r, rem)


def run_split(f, ng, periodic, dim, P, scheme, h, dtype="f64", n_halo=4):
    """apply_along! of `scheme` along `dim` on the global padded field(s) f
    ((count,) + padded shape, or the padded shape), split P ways."""
    import torch
    single = f.ndim == 3
    F = f[None] if single else f
    count = F.shape[0]
    d0 = dim - 1
    nh = n_halo
    act = [ng[k] > 1 for k in range(3)]
    pad = [nh if act[k] else 0 for k in range(3)]
    tdt = torch.float64 if dtype == "f64" else torch.float32
    ranks = []
    for r in range(P):
        nr, off = local_range(ng[d0], P, r)
        nl = list(ng)
        nl[d0] = nr
        plan = cl.SplitPlan(scheme, nl, dim, h, ng[d0], P, r, periodic, n_halo=nh, dtype=dtype)
        shape = plan.shape()
        loc = np.zeros((count,) + shape)
        # interior of the global field along [off, off + nr) of dim (numpy axes are z, y, x)
        src = [slice(None)] + [slice(pad[k], pad[k] + ng[k]) for k in (2, 1, 0)]
        dst = [slice(None)] + [slice(pad[k], pad[k] + nl[k]) for k in (2, 1, 0)]
        ax = 1 + (2 - d0)
        src[ax] = slice(pad[d0] + off, pad[d0] + off + nr)
        loc[tuple(dst)] = F[tuple(src)]
        ft = torch.tensor(loc, dtype=tdt, device="cuda")
        out = torch.zeros_like(ft)
        bufs = plan.buffers(count, "cuda")
        ranks.append(dict(plan=plan, f=ft, out=out, bufs=bufs, off=off, nr=nr, dst=tuple(dst)))
    for R in ranks:
        R["fs"] = int(np.prod(R["plan"].shape()))
        R["plan"].pack(R["f"], R["bufs"], count, R["fs"])
    # the Sendrecv! of LineExchange.halo
    for R in ranks:
        p, b = R["plan"], R["bufs"]
        if p.prev is not None:
            b["recv_lo"].copy_(ranks[p.prev]["bufs"]["send_hi"])
        if p.next is not None:
            b["recv_hi"].copy_(ranks[p.next]["bufs"]["send_lo"])
    for R in ranks:
        R["plan"].unpack(R["bufs"], R["f"], count, R["fs"])
        R["plan"].begin(R["f"], R["out"], R["bufs"], count, R["fs"])
    # the Allgather! of LineExchange.gather
    allv = torch.stack([R["bufs"]["iface"] for R in ranks])
    for R in ranks:
        R["bufs"]["iface_all"].copy_(allv)
        R["plan"].end(R["bufs"], R["out"], count, R["fs"])
    torch.cuda.synchronize()
    res = np.zeros((count,) + tuple(ng[k] for k in (2, 1, 0)))
    for R in ranks:
        o = R["out"].cpu().numpy().astype(np.float64)[R["dst"]]
        sl = [slice(None)] * 4
        sl[1 + (2 - d0)] = slice(R["off"], R["off"] + R["nr"])
        res[tuple(sl)] = o
    return res[0] if single else res


def _field(orc, g, seed):
    rng = np.random.default_rng(seed)
    f = np.zeros(orc.padded_shape(g))
    inner = orc.interior(g, f)
    z, y, x = np.meshgrid(*[np.arange(s) for s in inner.shape], indexing="ij")
    inner[...] = np.sin(0.3 * x + 0.2 * y + 0.1 * z + rng.uniform(0, 6)) + 0.1 * rng.standard_normal(inner.shape)
    orc.exchange_halos(g, f)
    return f


@pytest.mark.parametrize("scheme", ["c6", "c10", "filt", "pade"])
@pytest.mark.parametrize("dim", [1, 2, 3])
@pytest.mark.parametrize("periodic", [True, False])
def test_split_matches_oracle_fp64(orc, scheme, dim, periodic):
    ng = tuple(50 if k == dim - 1 else 9 for k in range(3))
    per = tuple(1 if (k != dim - 1 or periodic) else 0 for k in range(3))
    g = orc.grid(ng, per)
    f = _field(orc, g, seed=dim + 10 * periodic)
    h = 0.7 / 50
    single = orc.interior(g, orc.Plan(g, _schemes(orc, scheme), dim, h).apply(f))
    for P in (1, 2, 3, 4):
        ref = orc.interior(g, orc.Plan(g, _schemes(orc, scheme), dim, h, P=P).apply(f))
        got = run_split(f, ng, periodic, dim, P, _schemes(cl, scheme), h)
        scale = np.abs(ref).max()
        assert np.abs(got - ref).max() <= 1e-12 * scale, (P, np.abs(got - ref).max() / scale)
        assert np.abs(got - single).max() <= 1e-12 * scale, P


@pytest.mark.parametrize("scheme", ["c6", "c10", "filt"])
@pytest.mark.parametrize("dim", [1, 3])
def test_split_fp32(orc, scheme, dim):
    ng = tuple(96 if k == dim - 1 else 10 for k in range(3))
    for periodic in (True, False):
        per = tuple(1 if (k != dim - 1 or periodic) else 0 for k in range(3))
        g = orc.grid(ng, per)
        f = _field(orc, g, seed=3)
        h = 1.0 / 96
        ref = orc.interior(g, orc.Plan(g, _schemes(orc, scheme), dim, h, P=3).apply(f))
        got = run_split(f, ng, periodic, dim, 3, _schemes(cl, scheme), h, dtype="f32")
        assert np.abs(got - ref).max() <= 2e-6 * np.abs(ref).max()


@pytest.mark.parametrize("case", ["segmented_3d", "long_1d_closed", "long_1d_periodic_c10"])
def test_split_long_lines(orc, case):
    # local pieces of several 32-point segments, and 1-D pieces long enough
    # for the cyclic-reduction interface solve (more than 32 segments)
    if case == "segmented_3d":
        ng, per, dim, P, sch = (20, 250, 18), (1, 0, 1), 2, 3, "c6"
    elif case == "long_1d_closed":
        ng, per, dim, P, sch = (4100, 1, 1), (0, 1, 1), 1, 2, "c6"
    else:
        ng, per, dim, P, sch = (3000, 1, 1), (1, 1, 1), 1, 4, "c10"
    g = orc.grid(ng, per)
    f = _field(orc, g, seed=7)
    h = 1.0 / ng[dim - 1]
    ref = orc.interior(g, orc.Plan(g, _schemes(orc, sch), dim, h, P=P).apply(f))
    got = run_split(f, ng, bool(per[dim - 1]), dim, P, _schemes(cl, sch), h)
    assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()


@pytest.mark.parametrize("scheme", ["c6", "c10", "filt", "pade"])
@pytest.mark.parametrize("dim,P", [(1, 2), (1, 4), (2, 2), (3, 4), (3, 8)])
@pytest.mark.parametrize("periodic", [True, False])
def test_split_tile_path(orc, scheme, dim, P, periodic):
    # pieces of equal 32-point segments (16-point ones for the 32-point pieces
    # of P = 8) and enough line groups for the tile kernels: y/z through TMA
    # boxes that also carry the halo rows, x through cp.async rows widened by
    # the halo elements
    ng = {1: (256, 80, 64), 2: (64, 256, 80), 3: (64, 80, 256)}[dim]
    per = tuple(1 if (k != dim - 1 or periodic) else 0 for k in range(3))
    g = orc.grid(ng, per)
    f = _field(orc, g, seed=11 + dim)
    h = 1.0 / 256
    ref = orc.interior(g, orc.Plan(g, _schemes(orc, scheme), dim, h, P=P).apply(f))
    got = run_split(f, ng, periodic, dim, P, _schemes(cl, scheme), h)
    assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()
    got32 = run_split(f, ng, periodic, dim, P, _schemes(cl, scheme), h, dtype="f32")
    assert np.abs(got32 - ref).max() <= 2e-6 * np.abs(ref).max()


def test_split_batch_of_fields(orc):
    ng, per = (12, 40, 64), (1, 1, 0)
    g = orc.grid(ng, per)
    fs = np.stack([_field(orc, g, seed=s) for s in range(3)])
    h = 1.0 / 63
    got = run_split(fs, ng, False, 3, 4, cl.lele_d1_6(), h)
    for c in range(3):
        ref = orc.interior(g, orc.Plan(g, orc.lele_d1_6(), 3, h, P=4).apply(fs[c]))
        assert np.abs(got[c] - ref).max() <= 1e-12 * np.abs(ref).max()


SPLITN = 72


def _global_field(ng, fn, L, periodic):
    nh = 4
    xs = []
    for k in range(3):
        if ng[k] == 1:
            xs.append(np.zeros(1))
            continue
        h = L[k] / ng[k] if periodic[k] else L[k] / (ng[k] - 1)
        xs.append(np.arange(ng[k]) * h)
    z, y, x = np.meshgrid(xs[2], xs[1], xs[0], indexing="ij")
    f = np.zeros(tuple(n + 2 * nh if n > 1 else 1 for n in reversed(ng)))
    f[tuple(slice(nh, nh + ng[k]) if ng[k] > 1 else slice(None) for k in (2, 1, 0))] = fn(x, y, z)
    return f, (x, y, z)


@pytest.mark.parametrize("P", [2, 4, 8])
def test_reference_mpi_periodic_c6_and_c10(P):
    # test/mpi_tests.jl:117-166: sin(3x) cos(2y), 72 points on the split dim
    fx = lambda x, y, z: np.sin(3 * x) * np.cos(2 * y)
    for scheme, tol, axes in ((cl.lele_d1_6(), 1e-4, (1, 2, 3)), (cl.lele_d1_10(), 1e-8, (1, 2))):
        for ax in axes:
            ng = tuple(SPLITN if k == ax - 1 else 16 for k in range(3))
            f, (x, y, z) = _global_field(ng, fx, (2 * np.pi,) * 3, (1, 1, 1))
            h = 2 * np.pi / ng[ax - 1]
            got = run_split(f, ng, True, ax, P, scheme, h)
            exact = {1: 3 * np.cos(3 * x) * np.cos(2 * y), 2: -2 * np.sin(3 * x) * np.sin(2 * y), 3: 0 * x}[ax]
            assert np.abs(got - exact).max() < (1e-10 if ax == 3 else tol), (ax, P)


@pytest.mark.parametrize("P", [2, 4, 8])
def test_reference_mpi_closed_cubic_exact(P):
    # test/mpi_tests.jl:153-165 (C10) and :181-192 (C6): 1 + 2x + 3x^2 - x^3
    # on [0, 1] between slip walls, x split
    ng = (SPLITN, 12, 12)
    f, (x, y, z) = _global_field(ng, lambda x, y, z: 1 + 2 * x + 3 * x ** 2 - x ** 3, (1.0, 1.0, 1.0), (0, 1, 1))
    exact = 2 + 6 * x - 3 * x ** 2
    for scheme in (cl.lele_d1_6(), cl.lele_d1_10()):
        got = run_split(f, ng, False, 1, P, scheme, 1.0 / (SPLITN - 1))
        assert np.abs(got - exact).max() < 1e-9


def test_split_plan_errors():
    # src/operators.jl:50-53: the smallest local extent decides for every rank
    with pytest.raises(cl.ClesError, match="too small"):
        cl.SplitPlan(cl.compact_filter(0.45), (9, 8, 8), 1, 0.1, 36, 4, 0, True)  # 36 / 4 = 9: fine
        cl.SplitPlan(cl.compact_filter(0.45), (8, 8, 8), 1, 0.1, 35, 4, 3, True)  # 35 / 4 = 8 < 9
    with pytest.raises(cl.ClesError, match="share"):
        cl.SplitPlan(cl.lele_d1_6(), (20, 8, 8), 1, 0.1, 50, 3, 2, True)           # rank 2 of 50 / 3 holds 16
    with pytest.raises(cl.ClesError, match="halo"):
        cl.SplitPlan(cl.compact_filter(0.45), (20, 8, 8), 1, 0.1, 40, 2, 0, True, n_halo=3)
    p = cl.SplitPlan(cl.lele_d1_6(), (20, 8, 8), 1, 0.1, 40, 2, 1, False)
    assert (p.prev, p.next) == (0, None)
    p = cl.SplitPlan(cl.lele_d1_6(), (20, 8, 8), 1, 0.1, 40, 2, 1, True)
    assert (p.prev, p.next) == (0, 0)
