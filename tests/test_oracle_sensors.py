"""The oracle against the reference's known-answer tests of the artificial
properties (test/runtests.jl:543-628):

* with two species, D*_k stays tiny on a smooth composition and switches on
  (more than 100x) at a sharp interface, finite everywhere (:543-566);
* on a solenoidal Taylor-Green field the dilatation sensor's beta* is below
  1e-12 of the strain sensor's, the gated strain removes more than 99 % of
  the total, and mu* is bitwise the same for all three sensors (:568-598);
* on a velocity ramp both compression-keyed sensors give beta* = 0 exactly
  where the flow expands, still switch on where it compresses, and gated
  strain never exceeds strain (:600-626)."""
import numpy as np
import pytest

import compactles_b200 as cl
from compactles_b200 import abi


def _solver(orc, n, L, ic, sensor="strain", eos=None):
    d = cl.solver_desc(n, L, cl.PER3, orc.lele_d1_6(), orc.compact_filter(0.45),
                       art=cl.ArtParams(enabled=True, beta_sensor=sensor), **({"eos": eos} if eos else {}))
    S = orc.Solver(d)
    S.set_state(cl.initialize(d, ic))
    S.compute_rhs()
    return S, cl.interior_slices(d)


def test_multi_species_diffusivity_responds_to_y_gradients(orc):
    eos = cl.IdealMixture([cl.IdealSpecies("a", 1.0, 1.4), cl.IdealSpecies("b", 0.2, 1.09)])
    n, L = (64, 12, 12), (1.0, 0.2, 0.2)
    smooth = lambda x, y, z: cl.Prim(Y=(0.5 + 0.1 * np.sin(2 * np.pi * x) + 0 * y, 0.5 - 0.1 * np.sin(2 * np.pi * x) + 0 * z),
                                     p=1.0 + 0 * x, rho=1.0 + 0 * x)

    def sharp(x, y, z):
        th = cl.tanh_blend(x, 0.5, 0.01) + 0 * y + 0 * z
        return cl.Prim(Y=(1 - th, th), p=1.0 + 0 * x, rho=1.0 + 0 * x)

    out = []
    for ic in (smooth, sharp):
        S, sl = _solver(orc, n, L, ic, eos=eos)
        D = [S.field(abi.CLES_FIELD_D_ART0 + k) for k in range(2)]
        assert all(np.isfinite(Dk).all() for Dk in D)
        out.append(max(Dk.max() for Dk in D))
    assert out[1] > 100 * max(out[0], 1e-14)


def test_compression_keyed_beta_sensors(orc):
    tgv = lambda x, y, z: cl.Prim(rho=1.0 + 0 * x, p=100.0 + 0 * x,
                                  u=(np.sin(x) * np.cos(y) * np.cos(z), -np.cos(x) * np.sin(y) * np.cos(z), 0.0 * z))
    fields = {}
    for sensor in ("strain", "gated_strain", "dilatation"):
        S, sl = _solver(orc, (32, 32, 32), (2 * np.pi,) * 3, tgv, sensor)
        fields[sensor] = (S.field(abi.CLES_FIELD_BETA_ART), S.field(abi.CLES_FIELD_MU_ART), sl)
    bs, ms, sl = fields["strain"]
    bg, mg, _ = fields["gated_strain"]
    bd, md, _ = fields["dilatation"]
    assert bd.max() < 1e-12 * bs.max()
    assert bg[sl].sum() < 1e-2 * bs[sl].sum()
    assert np.array_equal(md, ms) and np.array_equal(mg, ms)
    assert np.isfinite(bd).all() and np.isfinite(bg).all()

    ramp = lambda x, y, z: cl.Prim(rho=1.0 + 0 * x, p=1.0 + 0 * x,
                                   u=(0.5 * np.tanh((x - 0.5) / 0.02) + 0 * y, 0.0 * y, 0.0 * z))
    res = {}
    for sensor in ("strain", "gated_strain", "dilatation"):
        S, sl = _solver(orc, (64, 12, 12), (1.0, 0.2, 0.2), ramp, sensor)
        div = sum(S.field(abi.CLES_FIELD_GRAD_U0 + 4 * a) for a in range(3))
        res[sensor] = (S.field(abi.CLES_FIELD_BETA_ART)[sl], div[sl])
    bstrain = res["strain"][0]
    for sensor in ("gated_strain", "dilatation"):
        b, div = res[sensor]
        line_b, line_div = b[0, 0, :], div[0, 0, :]
        expanding = line_div > 0
        assert expanding.any()
        assert np.all(line_b[expanding] == 0.0)
        assert b.max() > 0.1 * bstrain.max()
    assert np.all(res["gated_strain"][0][0, 0, :] <= bstrain[0, 0, :] + 1e-300)


def test_unknown_beta_sensor_is_refused(orc):
    # test/runtests.jl:627-628
    with pytest.raises(ValueError, match="beta_sensor"):
        cl.solver_desc((16, 16, 16), (1.0, 1.0, 1.0), cl.PER3, orc.lele_d1_6(), orc.compact_filter(0.45),
                       art=cl.ArtParams(beta_sensor="bogus"))
