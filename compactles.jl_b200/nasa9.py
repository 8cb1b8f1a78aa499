"""NASA-9 thermally perfect mixtures on the host side.

The counterpart of src/physics.jl:255-498 (Nasa9Interval, Nasa9Species,
Nasa9Mixture, the species cp / h / e functions and mixture_temperature) and
of src/nasa9_data.jl (read_nasa9, the fixed-column NASA CEA thermo.inp
reader).  The device evaluates the same polynomials inside the primitive
recovery (a bounded FP64 Newton per point) and in the species-enthalpy flux;
this module builds the descriptor tables, evaluates initial conditions and
reads CEA data.

Polynomials of one interval (T in kelvin):
    cp/R = a1 T^-2 + a2 T^-1 + a3 + a4 T + a5 T^2 + a6 T^3 + a7 T^4
    h/R  = -a1 T^-1 + a2 ln T + a3 T + a4 T^2/2 + a5 T^3/3 + a6 T^4/4 + a7 T^5/5 + b1
"""
import math
from dataclasses import dataclass, field
from typing import List, Sequence, Tuple

import numpy as np

R_UNIVERSAL = 8.31446261815324     # J/(mol K), src/nasa9_data.jl:19
CONTINUITY_RTOL = 2e-3             # src/physics.jl:320


@dataclass
class Nasa9Interval:
    """Nasa9Interval(Tmin, Tmax, a, b1) (src/physics.jl:291-296)."""
    Tmin: float
    Tmax: float
    a: Tuple[float, ...]
    b1: float = 0.0


def cp_over_R(iv, T):
    a = iv.a
    T2 = T * T
    return a[0] / T2 + a[1] / T + a[2] + a[3] * T + a[4] * T2 + a[5] * (T2 * T) + a[6] * (T2 * T2)


def h_over_R(iv, T):
    a = iv.a
    T2 = T * T
    return (-a[0] / T + a[1] * np.log(T) + a[2] * T + a[3] * T2 / 2 + a[4] * (T2 * T) / 3 + a[5] * (T2 * T2) / 4
            + a[6] * (T2 * T2 * T) / 5 + iv.b1)


def _validate(name, R, intervals):
    """_validate_nasa9_intervals (src/physics.jl:322-345)."""
    if not intervals:
        raise ValueError(f"NASA-9 species {name} has no intervals")
    if not R > 0:
        raise ValueError(f"NASA-9 species {name} has non-positive R")
    for iv in intervals:
        if not (iv.Tmin > 0 and iv.Tmin < iv.Tmax):
            raise ValueError(f"invalid NASA-9 interval for {name}")
    for lo, hi in zip(intervals[:-1], intervals[1:]):
        sT = max(abs(lo.Tmax), abs(hi.Tmin), 1.0)
        if not abs(lo.Tmax - hi.Tmin) <= 1e-10 * sT:
            raise ValueError(f"non-contiguous NASA-9 intervals for {name}")
        Tj = (lo.Tmax + hi.Tmin) / 2
        cl, ch = cp_over_R(lo, Tj), cp_over_R(hi, Tj)
        if not abs(cl - ch) <= CONTINUITY_RTOL * max(abs(cl), abs(ch), 1.0):
            raise ValueError(f"discontinuous NASA-9 cp for {name} at {Tj} K")
        hl, hh = h_over_R(lo, Tj), h_over_R(hi, Tj)
        if not abs(hl - hh) <= CONTINUITY_RTOL * max(abs(hl), abs(hh), Tj):
            raise ValueError(f"discontinuous NASA-9 h for {name} at {Tj} K")


@dataclass
class Nasa9Species:
    """Nasa9Species(name, R, intervals) (src/physics.jl:347-385)."""
    name: str
    R: float
    intervals: List[Nasa9Interval]

    def __post_init__(self):
        _validate(self.name, self.R, self.intervals)

    @staticmethod
    def single(name, R, a, b1=0.0, Tmin=200.0, Tmax=6000.0):
        """The keyword constructor with one interval."""
        return Nasa9Species(name, float(R), [Nasa9Interval(float(Tmin), float(Tmax), tuple(float(x) for x in a),
                                                           float(b1))])


def nasa9_constant_cp(name, R, cp):
    """nasa9_constant_cp(name, R, cp) (src/physics.jl:387-400): the calorically perfect limit."""
    return Nasa9Species.single(name, float(R), (0.0, 0.0, float(cp) / float(R), 0.0, 0.0, 0.0, 0.0), b1=0.0)


def _interval_index(sp, T):
    """_nasa9_interval: first interval with T <= Tmax, else the last (vectorised)."""
    T = np.asarray(T, dtype=np.float64)
    idx = np.full(T.shape, len(sp.intervals) - 1, dtype=np.int64)
    for i in range(len(sp.intervals) - 2, -1, -1):
        idx = np.where(T <= sp.intervals[i].Tmax, i, idx)
    return idx


def _piecewise(sp, T, fn):
    T = np.asarray(T, dtype=np.float64)
    idx = _interval_index(sp, T)
    out = np.zeros(T.shape)
    for i, iv in enumerate(sp.intervals):
        m = idx == i
        if np.any(m):
            out = np.where(m, fn(iv, np.where(m, T, 1.0)), out)
    return out if out.shape else float(out)


@dataclass
class Nasa9Mixture:
    """Nasa9Mixture(species; T_guess=300.0) (src/physics.jl:402-427)."""
    sp: Sequence[Nasa9Species]
    T_guess: float = 300.0

    @property
    def Rk(self):
        return [s.R for s in self.sp]

    @property
    def nspecies(self):
        return len(self.sp)

    def species_names(self):
        return [s.name for s in self.sp]

    def species_cp(self, k, T):
        s = self.sp[k]
        return s.R * _piecewise(s, T, cp_over_R)

    def species_enthalpy(self, k, T):
        s = self.sp[k]
        return s.R * _piecewise(s, T, h_over_R)

    def species_energy(self, k, T):
        return self.species_enthalpy(k, T) - self.sp[k].R * np.asarray(T, dtype=np.float64)

    def mixture_temperature(self, e, Y):
        """mixture_temperature(eos, e, Yat) (src/physics.jl:466-498), scalar."""
        n = self.nspecies
        e0 = sum(Y[k] * float(self.species_energy(k, self.T_guess)) for k in range(n))
        cv0 = sum(Y[k] * (float(self.species_cp(k, self.T_guess)) - self.sp[k].R) for k in range(n))
        if cv0 > 0:
            x = self.T_guess + (e - e0) / cv0
            T = 1e9 if x > 1e9 else (1e-3 if x < 1e-3 else x)
        else:
            T = self.T_guess
        for _ in range(30):
            f = -e
            cvm = 0.0
            for k in range(n):
                f += Y[k] * float(self.species_energy(k, T))
                cvm += Y[k] * (float(self.species_cp(k, T)) - self.sp[k].R)
            if not cvm > 0:
                break
            d = f / cvm
            T = max(T - d, 0.25 * T)
            if abs(d) <= 1e-14 * T:
                break
        return T


# ------------------------------------------------------------- CEA reader ----
def _field(line, first, last, context):
    """Columns first..last (1-based, inclusive) of a fixed-column record."""
    if len(line) < last:
        raise ValueError(f"short NASA CEA record while reading {context}")
    return line[first - 1:last]


def _float(field, context):
    value = field.strip().replace("D", "E").replace("d", "e")
    if not value:
        raise ValueError(f"empty NASA CEA field for {context}")
    try:
        return float(value)
    except ValueError:
        raise ValueError(f"invalid NASA CEA number '{value}' for {context}") from None


def _int(field, context):
    try:
        return int(field.strip())
    except ValueError:
        raise ValueError(f"invalid NASA CEA integer '{field.strip()}' for {context}") from None


def _record(lines, i, header, n_intervals, name, path):
    if n_intervals <= 0:
        raise ValueError(f"NASA CEA species {name} has no temperature intervals; it is a reactant-only record "
                         "carrying a heat of formation, not a fit")
    if _int(_field(header, 51, 52, name), name) != 0:
        raise ValueError(f"NASA CEA species {name} is not gaseous")
    molar_mass = _float(_field(header, 53, 65, name), name)
    if not molar_mass > 0:
        raise ValueError(f"non-positive molar mass for {name}")
    R = 1000 * R_UNIVERSAL / molar_mass
    intervals = []
    for j in range(n_intervals):
        b = i + 2 + 3 * j
        if b + 2 >= len(lines):
            raise ValueError(f"truncated NASA CEA intervals for {name} in {path}")
        bounds, c1, c2 = lines[b], lines[b + 1], lines[b + 2]
        Tmin = _float(_field(bounds, 1, 11, name), name)
        Tmax = _float(_field(bounds, 12, 22, name), name)
        a = tuple(_float(_field(c1 if f <= 5 else c2, 16 * (f if f <= 5 else f - 5) - 15,
                                16 * (f if f <= 5 else f - 5), name), name) for f in range(1, 8))
        b1 = _float(_field(c2, 49, 64, name), name)
        intervals.append(Nasa9Interval(Tmin, Tmax, a, b1))
    return Nasa9Species(name, R, intervals)


def _reference(sp, reference, T_ref):
    if reference == "formation":
        return sp
    iv = sp.intervals[int(_interval_index(sp, T_ref))]
    shift = -float(h_over_R(iv, T_ref))
    return Nasa9Species(sp.name, sp.R, [Nasa9Interval(x.Tmin, x.Tmax, x.a, x.b1 + shift) for x in sp.intervals])


def read_nasa9(names, path, reference="sensible", T_ref=298.15):
    """read_nasa9(names; path, reference=:sensible, T_ref=298.15) (src/nasa9_data.jl:104-186).

    Gas species from a NASA CEA thermo.inp file, in the requested order; R
    from each record's molar mass; reference "sensible" shifts every b1 so
    that h(T_ref) = 0, "formation" keeps the tabulated gauge.  One name
    returns one species."""
    single = isinstance(names, str)
    if single:
        names = [names]
    if reference not in ("sensible", "formation"):
        raise ValueError("reference must be :sensible or :formation")
    if not T_ref > 0:
        raise ValueError("T_ref must be positive")
    requested = [str(n) for n in names]
    if not requested:
        return []
    with open(path) as fh:
        lines = fh.read().splitlines()
    try:
        i = next(k for k, l in enumerate(lines) if l.strip() == "thermo") + 2
    except StopIteration:
        raise ValueError(f"NASA CEA thermo marker not found in {path}") from None
    wanted = set(requested)
    found = {}
    while i < len(lines):
        line = lines[i]
        st = line.strip()
        if st.lower() == "end":
            break
        if not st or st.startswith("!") or st in ("END PRODUCTS", "END REACTANTS"):
            i += 1
            continue
        name = _field(line, 1, 16, "species name").strip()
        if i + 1 >= len(lines):
            raise ValueError(f"truncated NASA CEA header for {name} in {path}")
        header = lines[i + 1]
        n_int = _int(_field(header, 1, 2, name), name)
        # first match wins: the gaseous fit precedes repeats of the name
        if name in wanted and name not in found:
            found[name] = _reference(_record(lines, i, header, n_int, name, path), reference, T_ref)
            if len(found) == len(wanted):
                break
        i += 3 if n_int == 0 else 2 + 3 * n_int
    absent = [n for n in dict.fromkeys(requested) if n not in found]
    if absent:
        raise ValueError("NASA CEA species not found: " + ", ".join(absent))
    out = [found[n] for n in requested]
    return out[0] if single else out


def fill_descriptor(desc, eos):
    """Write a Nasa9Mixture into a cles_solver_desc (eos, T_guess, R, tables)."""
    from . import abi
    if eos.nspecies > abi.CLES_MAX_SPECIES:
        raise ValueError("too many species")
    desc.eos = abi.CLES_EOS_NASA9
    desc.T_guess = float(eos.T_guess)
    for k, s in enumerate(eos.sp):
        if len(s.intervals) > abi.CLES_MAX_NASA9_INTERVALS:
            raise ValueError(f"species {s.name} has more than {abi.CLES_MAX_NASA9_INTERVALS} intervals")
        desc.R[k] = s.R
        desc.gamma[k] = 0.0
        desc.n_intervals[k] = len(s.intervals)
        for i, iv in enumerate(s.intervals):
            t = desc.nasa9[k][i]
            t.Tmin, t.Tmax, t.b1 = iv.Tmin, iv.Tmax, iv.b1
            for j in range(7):
                t.a[j] = iv.a[j]
