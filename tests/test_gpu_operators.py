"""GPU parity of the directional compact operators (cles_apply_along through
the C ABI) against the CPU oracle on identical seeded inputs.

Tolerances: FP64 plans must agree with the oracle to 1e-12 relative to the
largest output value (the per-RHS bound of the FP64 drop-in); FP32 plans to
2e-6 (single-precision line solves of diagonally dominant systems)."""
import numpy as np
import pytest

import compactles_b200 as cl

pytestmark = pytest.mark.gpu

SCHEMES = ["c6", "c10", "filt", "pade"]


def _schemes(mod, name):
    return {"c6": mod.lele_d1_6, "c10": mod.lele_d1_10, "filt": lambda: mod.compact_filter(0.45),
            "pade": mod.pade_d1_4}[name]()


def _field(orc, g, seed):
    rng = np.random.default_rng(seed)
    f = np.zeros(orc.padded_shape(g))
    inner = orc.interior(g, f)
    # smooth part plus a little noise so every mode is exercised
    z, y, x = np.meshgrid(*[np.arange(s) for s in inner.shape], indexing="ij")
    inner[...] = (np.sin(0.3 * x + 0.2 * y + 0.1 * z + rng.uniform(0, 6)) + 0.1 * rng.standard_normal(inner.shape))
    orc.exchange_halos(g, f)
    return f


@pytest.mark.parametrize("scheme", SCHEMES)
@pytest.mark.parametrize("dim", [1, 2, 3])
@pytest.mark.parametrize("periodic", [True, False])
@pytest.mark.parametrize("n", [12, 40, 256])
def test_apply_along_matches_oracle_fp64(orc, scheme, dim, periodic, n):
    ng = tuple(n if k == dim - 1 else (9 if n == 256 else 11) for k in range(3))
    per = tuple(1 if (k != dim - 1 or periodic) else 0 for k in range(3))
    g = orc.grid(ng, per)
    f = _field(orc, g, seed=n + dim)
    h = 0.7 / n
    ref = orc.interior(g, orc.Plan(g, _schemes(orc, scheme), dim, h).apply(f))
    plan = cl.plan_direction(cl.grid(ng, per), _schemes(cl, scheme), dim, h)
    out = np.zeros_like(f)
    cl.apply_along(out, plan, f)
    got = orc.interior(g, out)
    err = np.abs(got - ref).max() / np.abs(ref).max()
    assert err < 1e-12, err


@pytest.mark.parametrize("scheme", SCHEMES)
@pytest.mark.parametrize("dim", [1, 2, 3])
def test_apply_along_fp32(orc, scheme, dim):
    n = 128
    ng = tuple(n if k == dim - 1 else 10 for k in range(3))
    for periodic in (True, False):
        per = tuple(1 if (k != dim - 1 or periodic) else 0 for k in range(3))
        g = orc.grid(ng, per)
        f = _field(orc, g, seed=dim)
        h = 1.0 / n
        ref = orc.interior(g, orc.Plan(g, _schemes(orc, scheme), dim, h).apply(f))
        plan = cl.plan_direction(cl.grid(ng, per), _schemes(cl, scheme), dim, h, dtype="f32")
        f32 = f.astype(np.float32)
        out = np.zeros_like(f32)
        cl.apply_along(out, plan, f32)
        err = np.abs(orc.interior(g, out).astype(np.float64) - ref).max() / np.abs(ref).max()
        assert err < 2e-6, err


def test_apply_along_device_in_place_and_batch(orc):
    import torch
    n = (64, 48, 40)
    g = orc.grid(n, (1, 0, 1))
    fs = [_field(orc, g, seed=s) for s in range(3)]
    for dim in (1, 2, 3):
        h = 0.05
        refs = [orc.interior(g, orc.Plan(g, orc.lele_d1_6(), dim, h).apply(f)) for f in fs]
        plan = cl.plan_direction(cl.grid(n, (1, 0, 1)), cl.lele_d1_6(), dim, h)
        t = torch.tensor(np.stack(fs), device="cuda")
        st = torch.cuda.current_stream()
        plan.ctx.set_stream(st.cuda_stream)
        cl.api._check(cl.lib().cles_apply_along_batch(plan.ptr, cl.api.C.c_void_p(t.data_ptr()),
                                                      cl.api.C.c_void_p(t.data_ptr()), 3, fs[0].size))
        torch.cuda.synchronize()
        got = t.cpu().numpy()
        plan.ctx.set_stream(None)
        for b in range(3):
            err = np.abs(orc.interior(g, got[b]) - refs[b]).max() / np.abs(refs[b]).max()
            assert err < 1e-12
            # halos are never written
            assert np.array_equal(got[b][:4], fs[b][:4])


def test_spectral_accuracy_on_gpu():
    # test/runtests.jl:86-132 through the GPU plans
    n = 32
    g = cl.grid((n, n, n), (1, 1, 1))
    h = 2 * np.pi / n
    x = np.arange(n) * h
    f = np.zeros((n + 8,) * 3)
    f[4:-4, 4:-4, 4:-4] = np.sin(3 * x)[None, None, :] * np.cos(2 * x)[None, :, None]
    for sch, tol_x, tol_y, meas in ((cl.lele_d1_6(), 1e-4, 2e-5, None), (cl.lele_d1_10(), 1e-7, 1e-8, 2.8e-8)):
        out = np.zeros_like(f)
        cl.apply_along(out, cl.plan_direction(g, sch, 1, h), f)
        ex = np.abs(out[4:-4, 4:-4, 4:-4] - 3 * np.cos(3 * x)[None, None, :] * np.cos(2 * x)[None, :, None]).max()
        assert ex < tol_x
        if meas:
            assert abs(ex - meas) < 0.3e-8
        cl.apply_along(out, cl.plan_direction(g, sch, 2, h), f)
        ey = np.abs(out[4:-4, 4:-4, 4:-4] + 2 * np.sin(3 * x)[None, None, :] * np.sin(2 * x)[None, :, None]).max()
        assert ey < tol_y


def test_plan_errors_match_plan_direction():
    with pytest.raises(cl.ClesError, match="too small"):
        cl.plan_direction(cl.grid((8, 12, 12), (1, 1, 1)), cl.compact_filter(0.45), 1, 0.1)


@pytest.mark.parametrize("scheme", ["c6", "filt", "c10"])
@pytest.mark.parametrize("periodic", [True, False])
@pytest.mark.parametrize("ng,dim", [((1024, 64, 1), 1), ((768, 48, 1), 1), ((8192, 1, 1), 1), ((300, 256, 1), 2),
                                    ((2000, 3, 1), 1), ((9, 9, 1024), 3)])
def test_apply_along_long_lines(orc, scheme, periodic, ng, dim):
    """Line lengths of the 2-D ensemble and the 1-D tubes (up to 8192 cells),
    with the other dimensions collapsed or short."""
    per = tuple(1 if (k != dim - 1 or periodic or ng[k] == 1) else 0 for k in range(3))
    g = orc.grid(ng, per)
    f = _field(orc, g, seed=ng[dim - 1] + dim)
    h = 1.3 / ng[dim - 1]
    ref = orc.interior(g, orc.Plan(g, _schemes(orc, scheme), dim, h).apply(f))
    plan = cl.plan_direction(cl.grid(ng, per), _schemes(cl, scheme), dim, h)
    out = np.zeros_like(f)
    cl.apply_along(out, plan, f)
    got = orc.interior(g, out)
    err = np.abs(got - ref).max() / np.abs(ref).max()
    assert err < 1e-12, err


@pytest.mark.parametrize("scheme", SCHEMES)
@pytest.mark.parametrize("periodic", [True, False])
@pytest.mark.parametrize("dim", [1, 2, 3])
@pytest.mark.parametrize("n", [64, 128, 192, 256])
@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_apply_along_tile_kernels(orc, scheme, periodic, dim, n, dtype):
    """Lines with enough lines per plan for the 32-point segments of the tile
    kernels: TMA tiles for y/z, cp.async transposed tiles for x (closed lines,
    C10, and the periodic tridiagonal ones)."""
    # 96 x 96 lines: at least one group of 32 lines per SM, as the tile kernels require
    ng = tuple(n if k == dim - 1 else 96 for k in range(3))
    per = tuple(1 if (k != dim - 1 or periodic) else 0 for k in range(3))
    g = orc.grid(ng, per)
    f = _field(orc, g, seed=n + 7 * dim)
    h = 0.9 / n
    ref = orc.interior(g, orc.Plan(g, _schemes(orc, scheme), dim, h).apply(f))
    plan = cl.plan_direction(cl.grid(ng, per), _schemes(cl, scheme), dim, h, dtype=dtype)
    fin = f if dtype == "f64" else f.astype(np.float32)
    out = np.zeros_like(fin)
    cl.apply_along(out, plan, fin)
    got = orc.interior(g, out).astype(np.float64)
    err = np.abs(got - ref).max() / np.abs(ref).max()
    # FP32: single-precision inputs and solves; the seeded noise makes the
    # derivative large compared with the field, hence 5e-6 of the maximum
    assert err < (1e-12 if dtype == "f64" else 5e-6), err
