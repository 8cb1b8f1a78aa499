"""NASA-9 mixtures: the CEA reader, the species functions and the FP64 Newton
inversion, on the host module and the CPU oracle.

Golden values and tolerances follow test/runtests.jl:764-905.  The CEA
records come from tests/golden/nasa9_subset.json (generated from the
reference's data/thermo.inp by tests/golden/make_nasa9_subset.py); the
reader is exercised on a fixed-column file written here from those numbers.
"""
import json
import math
import pathlib

import numpy as np
import pytest

import compactles_b200 as cl
from compactles_b200 import abi
from compactles_b200 import nasa9 as n9

GOLD = json.loads((pathlib.Path(__file__).parent / "golden" / "nasa9_subset.json").read_text())


@pytest.fixture
def schemes(orc):
    return orc.lele_d1_6(), orc.compact_filter(0.45)


def _species(name):
    rec = next(s for s in GOLD["species"] if s["name"] == name)
    return n9.Nasa9Species(name, rec["R"], [n9.Nasa9Interval(iv["Tmin"], iv["Tmax"], tuple(iv["a"]), iv["b1"])
                                            for iv in rec["intervals"]])


def _sensible(sp, T_ref=298.15):
    return n9._reference(sp, "sensible", T_ref)


def _d16(x):
    return f"{x:16.9E}".replace("E", "D")


def _write_cea(path, species):
    """A thermo.inp-format file: comments, the thermo marker, product records,
    a zero-interval reactant record and the END markers."""
    L = ["! fixed-column NASA CEA records written by the test", "!", "thermo",
         "    200.000   1000.000   6000.000  20000.000   9/09/04"]
    for sp in species:
        M = 1000 * n9.R_UNIVERSAL / sp.R
        L.append(f"{sp.name:<16}  test record")
        hdr = f"{len(sp.intervals):2d} g 9/99 X   1.00    0.00    0.00    0.00    0.00"
        L.append(f"{hdr:<50}{0:2d}{M:13.7f}{0.0:15.3f}")
        for iv in sp.intervals:
            L.append(f"{iv.Tmin:11.3f}{iv.Tmax:11.3f}7 -2.0 -1.0  0.0  1.0  2.0  3.0  4.0  0.0{0.0:17.3f}")
            L.append("".join(_d16(v) for v in iv.a[:5]))
            L.append(_d16(iv.a[5]) + _d16(iv.a[6]) + " " * 16 + _d16(iv.b1) + _d16(0.0))
    L.append("END PRODUCTS")
    L.append(f"{'n-Butanol':<16}  reactant record without a fit")
    L.append(f"{' 0 g 5/23 C   4.00H  10.00O   1.00   0.00     0.00':<50}{0:2d}{74.1216:13.7f}{-251140.0:15.3f}")
    L.append("    298.150      0.0000  0.0  0.0  0.0  0.0  0.0  0.0  0.0  0.0            0.00")
    L.append("END REACTANTS")
    L.append("end")
    path.write_text("\n".join(L) + "\n")


def test_cea_reader_round_trip(tmp_path):
    names = [s["name"] for s in GOLD["species"]]
    sp = [_species(n) for n in names]
    f = tmp_path / "thermo.inp"
    _write_cea(f, sp)
    got = n9.read_nasa9(names, f, reference="formation")
    for a, b in zip(got, sp):
        assert a.name == b.name
        assert a.R == pytest.approx(b.R, rel=1e-12)
        assert len(a.intervals) == len(b.intervals)
        for x, y in zip(a.intervals, b.intervals):
            assert (x.Tmin, x.Tmax) == (y.Tmin, y.Tmax)
            assert np.allclose(x.a, y.a, rtol=1e-15, atol=0) and x.b1 == pytest.approx(y.b1, rel=1e-15)
    # order follows the request, one name gives one species
    assert [s.name for s in n9.read_nasa9(["CO2", "He"], f)] == ["CO2", "He"]
    assert n9.read_nasa9("Air", f).name == "Air"
    assert len(n9.read_nasa9("Jet-A(g)", f).intervals) == 2
    with pytest.raises(ValueError, match="reference must be"):
        n9.read_nasa9("CO2", f, reference="unknown")
    with pytest.raises(ValueError, match="T_ref must be positive"):
        n9.read_nasa9("CO2", f, T_ref=0.0)
    with pytest.raises(ValueError, match="no temperature intervals"):
        n9.read_nasa9("n-Butanol", f)
    with pytest.raises(ValueError, match="NASA CEA species not found"):
        n9.read_nasa9("not-a-CEA-species", f)


def test_cea_co2_golden_values(orc):
    # test/runtests.jl:843-881
    co2f = _species("CO2")
    co2 = _sensible(co2f)
    assert co2.R == pytest.approx(8.31446261815324 / 44.0095e-3, rel=1e-14)
    assert [(iv.Tmin, iv.Tmax) for iv in co2.intervals] == [(200.0, 1000.0), (1000.0, 6000.0), (6000.0, 20000.0)]
    sens = n9.Nasa9Mixture([co2])
    assert abs(sens.species_enthalpy(0, 298.15)) < 1e-6
    assert sens.species_cp(0, 300.0) == pytest.approx(845.7241586606974, rel=1e-13)
    for lo, hi in zip(co2.intervals[:-1], co2.intervals[1:]):
        Tj = lo.Tmax
        assert n9.cp_over_R(lo, Tj) == pytest.approx(n9.cp_over_R(hi, Tj), rel=5e-7)
        assert n9.h_over_R(lo, Tj) == pytest.approx(n9.h_over_R(hi, Tj), rel=5e-7)
    form = n9.Nasa9Mixture([co2f])
    assert abs(form.species_enthalpy(0, 298.15) * 44.0095e-3 - (-393510.0)) <= 5.0
    assert form.species_cp(0, 300.0) == sens.species_cp(0, 300.0)
    temps = (220.0, 300.0, 999.0, 1001.0, 1500.0, 5999.0, 6001.0, 10000.0)
    for mix in (sens, form):
        d = cl.solver_desc((8, 1, 1), (1.0, 1.0, 1.0), cl.PER3, orc.lele_d1_6(), orc.compact_filter(0.45), eos=mix)
        for T in temps:
            e = float(mix.species_energy(0, T))
            assert mix.mixture_temperature(e, [1.0]) == pytest.approx(T, rel=2e-13)
            assert orc.nasa9_temperature(d, e, [1.0]) == pytest.approx(T, rel=2e-13)
            # host module and oracle evaluate the same expressions
            assert orc.nasa9_cp(d, 0, T) == pytest.approx(float(mix.species_cp(0, T)), rel=1e-15)
            assert orc.nasa9_e(d, 0, T) == pytest.approx(e, rel=1e-14, abs=1e-9)
    Y = (0.3, 0.7)
    for ref in ("sensible", "formation"):
        he, c = _species("He"), _species("CO2")
        mix = n9.Nasa9Mixture([_sensible(he), _sensible(c)] if ref == "sensible" else [he, c])
        d = cl.solver_desc((8, 1, 1), (1.0, 1.0, 1.0), cl.PER3, orc.lele_d1_6(), orc.compact_filter(0.45), eos=mix)
        for T in (300.0, 1400.0, 7000.0):
            e = sum(Y[k] * float(mix.species_energy(k, T)) for k in range(2))
            assert mix.mixture_temperature(e, Y) == pytest.approx(T, rel=2e-13)
            assert orc.nasa9_temperature(d, e, Y) == pytest.approx(T, rel=2e-13)


def test_interval_validation():
    # the two loosest joins of the CEA table are accepted; a wrong coefficient is not
    for name in ("ALOCL", "SnCL2"):
        assert n9.Nasa9Mixture([_species(name)]).nspecies == 1
    good = n9.Nasa9Interval(200.0, 1000.0, (0.0, 0.0, 3.5, 0.0, 0.0, 0.0, 0.0), 0.0)
    bad = n9.Nasa9Interval(1000.0, 6000.0, (0.0, 0.0, 4.5, 0.0, 0.0, 0.0, 0.0), 0.0)
    with pytest.raises(ValueError):
        n9.Nasa9Species("broken", 287.0, [good, bad])


def _oracle_prims(orc, d, eos, prim_fn):
    S = orc.Solver(d)
    S.set_state(cl.initialize(d, prim_fn, eos=eos))
    S.max_rate()     # exchange_state! + primitives!
    return S


def test_constant_cp_reduces_to_ideal(orc, schemes):
    # test/runtests.jl:764-798
    g, R = 1.4, 1.0
    cp = g * R / (g - 1)
    ideal = cl.single_species(gamma=g, R=R)
    poly = n9.Nasa9Mixture([n9.nasa9_constant_cp("gas", R, cp)])
    d = cl.solver_desc((8, 1, 1), (1.0, 1.0, 1.0), cl.PER3, *schemes, eos=poly)
    for T in (0.3, 1.0, 7.5, 300.0):
        assert orc.nasa9_cp(d, 0, T) == pytest.approx(cp, rel=1e-14)
        assert orc.nasa9_h(d, 0, T) == pytest.approx(cp * T, rel=1e-14)
        assert orc.nasa9_e(d, 0, T) == pytest.approx((cp - R) * T, rel=1e-14)
    pr = cl.Prim(u=(0.3, -0.1, 0.2), p=0.8, T_ion=1.7)
    qi = cl.conserved_from_prim(ideal, pr)
    qp = cl.conserved_from_prim(poly, pr)
    assert np.allclose(qi, qp, rtol=1e-15, atol=0)
    I = (4 + 4, 4 + 3, 4 + 2)
    rhs = {}
    for eos in (ideal, poly):
        dd = cl.solver_desc((12, 12, 12), (2 * np.pi,) * 3, cl.PER3, *schemes, eos=eos)
        S = _oracle_prims(orc, dd, eos, lambda x, y, z: cl.Prim(u=(0.3 + 0.1 * np.sin(x), 0.0, 0.0 * z),
                                                              p=0.8 + 0.05 * np.cos(y), T_ion=1.7 + 0 * x))
        assert S.field(abi.CLES_FIELD_P)[I] == pytest.approx(0.8 + 0.05 * np.cos(2 * np.pi / 12 * 3), rel=1e-12)
        assert S.field(abi.CLES_FIELD_T)[I] == pytest.approx(1.7, rel=1e-12)
        assert S.field(abi.CLES_FIELD_C)[I] == pytest.approx(math.sqrt(g * R * 1.7), rel=1e-12)
        assert S.field(abi.CLES_FIELD_CP)[I] == pytest.approx(cp, rel=1e-12)
        rhs[type(eos).__name__] = (S.compute_rhs(), S.rhs_scales(cl.grid_spacing(dd)))
    (a, sc), (b, _) = rhs["IdealMixture"], rhs["Nasa9Mixture"]
    for c in range(a.shape[0]):
        assert np.abs(a[c] - b[c]).max() <= 1e-12 * max(sc[c], np.abs(a[c]).max())


def test_varying_cp_consistency(orc, schemes):
    # test/runtests.jl:800-841
    R = 287.0
    fake = n9.Nasa9Species.single("fake", R, (1.2e4, -50.0, 3.6, 6.0e-4, -1.0e-7, 1.0e-11, -4.0e-16), b1=-1.0e3)
    eos = n9.Nasa9Mixture([fake, n9.nasa9_constant_cp("inert", 200.0, 900.0)], T_guess=500.0)
    d = cl.solver_desc((12, 12, 12), (2 * np.pi,) * 3, cl.PER3, *schemes, eos=eos)
    for T in (250.0, 800.0, 2500.0):
        dl = 1e-4 * T
        dh = (orc.nasa9_h(d, 0, T + dl) - orc.nasa9_h(d, 0, T - dl)) / (2 * dl)
        assert dh == pytest.approx(orc.nasa9_cp(d, 0, T), rel=1e-7)
    assert orc.nasa9_cp(d, 0, 2500.0) / orc.nasa9_cp(d, 0, 300.0) > 1.2
    assert all(orc.nasa9_cp(d, 0, T) > R for T in np.arange(250.0, 2501.0, 50.0))
    for Y in ((1.0, 0.0), (0.5, 0.5), (0.2, 0.8)):
        for T in (250.0, 800.0, 2500.0):
            e = sum(Y[k] * orc.nasa9_e(d, k, T) for k in range(2))
            assert orc.nasa9_temperature(d, e, Y) == pytest.approx(T, rel=1e-12)
    S = _oracle_prims(orc, d, eos, lambda x, y, z: cl.Prim(Y=(0.35, 0.65), u=(120.0, 0.0, 0.0), p=2.5e5 + 0 * x,
                                                          T_ion=1400.0 + 0 * x))
    I = (4 + 4, 4 + 3, 4 + 2)
    assert S.field(abi.CLES_FIELD_P)[I] == pytest.approx(2.5e5, rel=1e-10)
    assert S.field(abi.CLES_FIELD_T)[I] == pytest.approx(1400.0, rel=1e-10)
    assert S.field(abi.CLES_FIELD_Y0 + 1)[I] == pytest.approx(0.65, rel=1e-12)
    rc, res = S.run(1e9, 3)
    assert rc == 0 and res.steps == 3
    assert np.all(np.isfinite(S.get_state()))
