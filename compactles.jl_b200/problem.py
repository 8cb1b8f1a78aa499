"""Host-side frontend: the reference's Problem / Numerics / Prim vocabulary.

Mirrors src/problem.jl (Prim :41-57, conserved_from_prim :76-90, initialize!
:146-163, tanh_blend :172, Problem :243-252, Numerics :295-306, setup
:321-345), the IdealMixture EOS (src/physics.jl:104-126), Transport
(:589-593), ArtParams (src/artificial.jl:50-57) and StepControl
(src/stepcontrol.jl:116-136).  Pure Python/numpy: it builds the flat
cles_solver_desc descriptor and evaluates initial conditions on the host.
Initial-condition callables are evaluated vectorised: ic(x, y, z) receives
broadcastable numpy coordinate arrays and returns a Prim whose fields may be
arrays.
"""
import ctypes as C
from dataclasses import dataclass, field
from typing import Callable, Optional, Sequence, Tuple

import numpy as np

from . import abi
from .nasa9 import Nasa9Interval, Nasa9Mixture, Nasa9Species, fill_descriptor


# ------------------------------------------------------------------- EOS ----
@dataclass
class IdealSpecies:
    name: str
    R: float
    gamma: float


@dataclass
class IdealMixture:
    sp: Sequence[IdealSpecies]

    @property
    def Rk(self):
        return [s.R for s in self.sp]

    @property
    def cvk(self):
        return [s.R / (s.gamma - 1) for s in self.sp]

    @property
    def nspecies(self):
        return len(self.sp)


def single_species(gamma=1.4, R=1.0, name="gas"):
    """single_species(; gamma, R, name) (src/physics.jl:125-126)."""
    return IdealMixture([IdealSpecies(name, float(R), float(gamma))])


@dataclass
class Transport:
    mu0: float = 0.0
    Pr: float = 0.7
    Sc: float = 0.7


@dataclass
class ArtParams:
    enabled: bool = True
    C_mu: float = 0.002
    C_beta: float = 1.0
    C_kappa: float = 0.01
    C_D: float = 0.01
    beta_sensor: str = "strain"


@dataclass
class StepControl:
    predict: float = 0.0
    max_growth: float = 0.0
    landing_steps: int = 2
    dt_min: float = 0.0
    dt_min_ratio: float = 1e-8
    retries: int = 0
    cfl_backoff: float = 0.5
    savepoint_interval: int = 25

    def __post_init__(self):
        if self.landing_steps < 1:
            raise ValueError("StepControl: landing_steps must be >= 1 (1 is a hard clip onto the scheduled time)")

    def to_c(self):
        c = abi.cles_step_control()
        for k in ("predict", "max_growth", "landing_steps", "dt_min", "dt_min_ratio",
                  "retries", "cfl_backoff", "savepoint_interval"):
            setattr(c, k, getattr(self, k))
        return c


# -------------------------------------------------------------- boundaries --
class BoundaryCondition:
    code = None


class PeriodicBC(BoundaryCondition):
    code = abi.CLES_BC_PERIODIC


class SlipWallBC(BoundaryCondition):
    code = abi.CLES_BC_SLIPWALL


class DirichletBC(BoundaryCondition):
    """DirichletBC(fun) (src/problem.jl:174-207): the full state imposed on the
    face after each stage.  `state` is either a Prim with scalar fields
    (constant) or a function fun(x, y, z, t) -> Prim evaluated at the stage
    time on the face's node coordinates (numpy arrays)."""
    code = abi.CLES_BC_DIRICHLET

    def __init__(self, state):
        self.fun = state if callable(state) else None
        self.state = None if callable(state) else state


class NoSlipWallBC(BoundaryCondition):
    """NoSlipWallBC(; Twall=NaN) (src/boundary.jl:33-44): zero velocity on the
    wall plane; a finite Twall also sets the wall's internal energy."""
    code = abi.CLES_BC_NOSLIP_WALL

    def __init__(self, Twall=float("nan")):
        self.Twall = float(Twall)


class ExtrapolationBC(BoundaryCondition):
    """ExtrapolationBC() (src/boundary.jl:46-54): copy the adjacent interior plane."""
    code = abi.CLES_BC_EXTRAPOLATION


class NSCBCOutflowBC(BoundaryCondition):
    """NSCBCOutflowBC(; pinf, sigma=0.25, Lref=0.0, beta_t=-1.0) (src/nscbc.jl:33-57)."""
    code = abi.CLES_BC_NSCBC_OUTFLOW

    def __init__(self, pinf, sigma=0.25, Lref=0.0, beta_t=-1.0):
        self.pinf, self.sigma, self.Lref, self.beta_t = float(pinf), float(sigma), float(Lref), float(beta_t)


class NSCBCInflowBC(BoundaryCondition):
    """NSCBCInflowBC(; u, T_ion, Y=[1.0], eta_u=eta_T=eta_t=eta_Y=0.28, Lref=0.0)
    (src/nscbc.jl:178-218), constant targets."""
    code = abi.CLES_BC_NSCBC_INFLOW

    def __init__(self, u, T_ion, Y=(1.0,), eta_u=0.28, eta_T=0.28, eta_t=0.28, eta_Y=0.28, Lref=0.0, target=None):
        # target: optional fun(x, y, z, t) -> Prim overriding the constants per
        # node at the stage time; its Prim must carry T_ion and the full Y
        self.target = target
        self.u = tuple(float(v) for v in u)
        self.T_ion = float(T_ion)
        self.Y = tuple(float(v) for v in Y)
        self.eta_u, self.eta_T, self.eta_t, self.eta_Y = float(eta_u), float(eta_T), float(eta_t), float(eta_Y)
        self.Lref = float(Lref)


class AxisBC(BoundaryCondition):
    """AxisBC() (src/boundary.jl:53-63): regularized cylindrical axis at the low
    r face; half-offset r grid, parity mirror rows, antipodal pairing when
    theta is resolved."""
    code = abi.CLES_BC_AXIS


class OriginBC(BoundaryCondition):
    """OriginBC() (src/boundary.jl:65-73): regularized spherical origin at the low r face."""
    code = abi.CLES_BC_ORIGIN


class PoleBC(BoundaryCondition):
    """PoleBC() (src/boundary.jl:75-82): regularized spherical poles, at both theta faces."""
    code = abi.CLES_BC_POLE


_FOLD_CODES = (abi.CLES_BC_AXIS, abi.CLES_BC_ORIGIN, abi.CLES_BC_POLE)


class SwitchableBC(BoundaryCondition):
    """SwitchableBC(before, after) (src/boundary.jl:120-160): the face acts as
    `before` until Solver.switch_bc(dim, side), then as `after`."""

    def __init__(self, before, after):
        if before.code in _FOLD_CODES or after.code in _FOLD_CODES:
            raise ValueError("SwitchableBC cannot wrap a fold condition (AxisBC, OriginBC, PoleBC); "
                             "setup detects those by type")
        if (before.code == abi.CLES_BC_PERIODIC) != (after.code == abi.CLES_BC_PERIODIC):
            raise ValueError("SwitchableBC: both conditions must agree on periodicity")
        if isinstance(before, SwitchableBC) or isinstance(after, SwitchableBC):
            raise ValueError("SwitchableBC cannot wrap another SwitchableBC")
        self.before, self.after = before, after
        self.code = before.code


PER3 = tuple((PeriodicBC(), PeriodicBC()) for _ in range(3))


# ----------------------------------------------------------------- metrics --
class Metric:
    code = None


class CartesianMetric(Metric):
    """CartesianMetric() (src/metric.jl:24-29)."""
    code = abi.CLES_METRIC_CARTESIAN


class CylindricalMetric(Metric):
    """CylindricalMetric() (src/metric.jl:31-37): (r, theta, z), physical velocity components."""
    code = abi.CLES_METRIC_CYLINDRICAL


class SphericalMetric(Metric):
    """SphericalMetric() (src/metric.jl:39-45): (r, theta, phi), theta the polar angle."""
    code = abi.CLES_METRIC_SPHERICAL


@dataclass
class ConstantBodyForce:
    """ConstantBodyForce(acceleration=(0, -9.81, 0)) (src/sources.jl:5-30): adds
    rho g to the momenta and rho u . g to the total energy."""
    acceleration: Tuple[float, float, float] = (0.0, -9.81, 0.0)


@dataclass
class Stretch:
    """Stretch(x, dxdxi) (src/metric.jl:47-63): monotone map of the uniform
    computational coordinate xi in [0, 1]; both callables take numpy arrays."""
    x: Callable
    dxdxi: Callable


def sine_cluster(lo, hi, xic, a):
    """sine_cluster(lo, hi, xic, a) (src/metric.jl:65-78): spacing smallest at
    xi = xic, ratio (1+a)/(1-a)."""
    if not (0 <= a < 1):
        raise ValueError("sine_cluster: need 0 ≤ a < 1")
    lo, hi, xic, a = float(lo), float(hi), float(xic), float(a)
    L = hi - lo
    two_pi = 2 * np.pi
    return Stretch(lambda xi: lo + L * (xi - (a / two_pi) * (np.sin(two_pi * (xi - xic)) + np.sin(two_pi * xic))),
                   lambda xi: L * (1 - a * np.cos(two_pi * (xi - xic))))


def _fill_face(bc, eos, ncons, params, state):
    """Write one face condition's parameters and Dirichlet state; returns its code."""
    p = params
    p.Twall = float("nan")
    p.sigma, p.beta_t = 0.25, -1.0
    p.eta_u = p.eta_T = p.eta_t = p.eta_Y = 0.28
    if bc.code == abi.CLES_BC_DIRICHLET:
        if bc.state is not None:
            q = conserved_from_prim(eos, bc.state)
            for c in range(ncons):
                state[c] = float(np.asarray(q[c]))
    elif bc.code == abi.CLES_BC_NOSLIP_WALL:
        p.Twall = bc.Twall
    elif bc.code == abi.CLES_BC_NSCBC_OUTFLOW:
        p.pinf, p.sigma, p.Lref, p.beta_t = bc.pinf, bc.sigma, bc.Lref, bc.beta_t
    elif bc.code == abi.CLES_BC_NSCBC_INFLOW:
        if len(bc.Y) != eos.nspecies:
            raise ValueError(f"NSCBCInflowBC: target composition has {len(bc.Y)} entries; "
                             f"the EOS has {eos.nspecies} species")
        for j in range(3):
            p.u[j] = bc.u[j]
        p.T_ion = bc.T_ion
        for k, y in enumerate(bc.Y):
            p.Y[k] = y
        p.eta_u, p.eta_T, p.eta_t, p.eta_Y, p.Lref = bc.eta_u, bc.eta_T, bc.eta_t, bc.eta_Y, bc.Lref
    return bc.code


# ------------------------------------------------------------------- Prim ----
class Prim:
    """Prim(; u, p, T_ion, rho, Y): exactly two of p, rho, T_ion."""

    def __init__(self, u=(0.0, 0.0, 0.0), p=None, T_ion=None, rho=None, Y=(1.0,)):
        given = [v is not None for v in (p, T_ion, rho)]
        if sum(given) != 2:
            raise ValueError("Prim: specify exactly two of p, rho, and T_ion; the EOS derives the third")
        self.u = tuple(u)
        self.p, self.T_ion, self.rho = p, T_ion, rho
        self.Y = tuple(Y)
        tot = sum(np.asarray(y, dtype=np.float64) for y in self.Y)
        if np.any(np.abs(tot - 1) >= 1e-10):
            raise ValueError("Prim: mass fractions must sum to 1")


def conserved_from_prim(eos, pr):
    """conserved_from_prim(::NavierStokes1T, ::IdealMixture, pr) (src/problem.jl:76-90)
    and (::Nasa9Mixture) (src/problem.jl:105-120), vectorised over
    array-valued Prim fields; returns a list of n_cons arrays."""
    N = len(pr.Y)
    if N != eos.nspecies:
        raise ValueError(f"Prim carries {N} mass fractions; EOS has {eos.nspecies} species")
    if isinstance(eos, Nasa9Mixture):
        Rm = 0.0
        for k in range(N):
            Rm = Rm + pr.Y[k] * eos.Rk[k]
        rho = pr.p / (Rm * pr.T_ion) if pr.rho is None else pr.rho
        T = pr.p / (rho * Rm) if pr.T_ion is None else pr.T_ion
        e = 0.0
        for k in range(N):
            e = e + pr.Y[k] * eos.species_energy(k, T)
        u = pr.u
        ke = 0.5 * (u[0] ** 2 + u[1] ** 2 + u[2] ** 2)
        out = [rho * pr.Y[k] for k in range(N)]
        out += [rho * u[0], rho * u[1], rho * u[2], rho * (e + ke)]
        return out
    Rk, cvk = eos.Rk, eos.cvk
    Rm = 0.0
    cvm = 0.0
    for k in range(N):
        Rm = Rm + pr.Y[k] * Rk[k]
        cvm = cvm + pr.Y[k] * cvk[k]
    rho = pr.p / (Rm * pr.T_ion) if pr.rho is None else pr.rho
    T = pr.p / (rho * Rm) if pr.T_ion is None else pr.T_ion
    u = pr.u
    ke = 0.5 * (u[0] ** 2 + u[1] ** 2 + u[2] ** 2)
    out = [rho * pr.Y[k] for k in range(N)]
    out += [rho * u[0], rho * u[1], rho * u[2], rho * (cvm * T + ke)]
    return out


def tanh_blend(x, x0, delta):
    """tanh_blend(x, x0, delta) (src/problem.jl:172)."""
    return 0.5 * (1 + np.tanh((x - x0) / delta))


# ---------------------------------------------------------- Problem/Numerics --
@dataclass
class Problem:
    domain: Tuple[Tuple[float, float], Tuple[float, float], Tuple[float, float]]
    bcs: tuple
    ic: Callable
    name: str = "problem"
    eos: IdealMixture = field(default_factory=single_species)
    transport: Transport = field(default_factory=Transport)
    metric: Metric = field(default_factory=CartesianMetric)
    sources: tuple = ()


@dataclass
class Numerics:
    n_global: Tuple[int, int, int]
    deriv: Optional[object] = None       # cles_scheme; None = lele_d1_6()
    filt: Optional[object] = None        # cles_scheme; None = compact_filter(0.45)
    art: ArtParams = field(default_factory=ArtParams)
    cfl: float = 0.5
    control: StepControl = field(default_factory=StepControl)
    filter_interval: int = 1
    n_halo: int = 4
    precision: str = "fp64"              # "fp64" (drop-in) or "mixed"
    stretch: tuple = (None, None, None)  # Stretch or None per dimension


_BETA = {"strain": abi.CLES_BETA_STRAIN, "gated_strain": abi.CLES_BETA_GATED_STRAIN,
         "dilatation": abi.CLES_BETA_DILATATION}


def solver_desc(n_global, L_domain, bcs, deriv, filt, eos=None, transport=None, art=None,
                origin=(0.0, 0.0, 0.0), cfl=0.5, filter_interval=1, control=None,
                n_halo=4, precision="fp64", metric=None, stretch=(None, None, None), sources=()):
    """The flat descriptor for Solver(; n_global, L_domain, bcs, ...) (src/rhs.jl:122-135).

    A Stretch on dimension d is sampled at the nodes xi_i = i / (n - 1)
    (src/metric.jl:99-106); the samples live as long as the descriptor."""
    eos = eos or single_species()
    transport = transport or Transport()
    art = art or ArtParams()
    control = control or StepControl()
    if art.beta_sensor not in _BETA:
        raise ValueError(f"art.beta_sensor must be :strain, :gated_strain or :dilatation, got :{art.beta_sensor}")
    d = abi.cles_solver_desc()
    ncons = eos.nspecies + 4
    face_fns = []
    for k in range(3):
        d.n_global[k] = int(n_global[k])
        d.L[k] = float(L_domain[k])
        d.origin[k] = float(origin[k])
        lo, hi = bcs[k]
        if (lo.code == abi.CLES_BC_PERIODIC) != (hi.code == abi.CLES_BC_PERIODIC):
            raise ValueError(f"dimension {k + 1} mixes periodic and non-periodic conditions")
        if n_global[k] == 1 and lo.code != abi.CLES_BC_PERIODIC:
            raise ValueError(f"collapsed dimension {k + 1} must use (PeriodicBC(), PeriodicBC())")
        for s, bc in enumerate((lo, hi)):
            if isinstance(bc, SwitchableBC):
                d.bc[k][s] = _fill_face(bc.before, eos, ncons, d.bc_params[k][s], d.bc_state[k][s])
                d.bc_switchable[k][s] = 1
                d.bc_after[k][s] = _fill_face(bc.after, eos, ncons, d.bc_after_params[k][s], d.bc_after_state[k][s])
                faces = ((0, bc.before), (1, bc.after))
            else:
                d.bc[k][s] = _fill_face(bc, eos, ncons, d.bc_params[k][s], d.bc_state[k][s])
                faces = ((0, bc),)
            for which, b in faces:
                fn = getattr(b, "fun", None) if b.code == abi.CLES_BC_DIRICHLET else getattr(b, "target", None)
                if fn is not None:
                    face_fns.append((k, s, which, b.code, fn))
    if eos.nspecies > abi.CLES_MAX_SPECIES:
        raise ValueError("too many species")
    d.n_species = eos.nspecies
    if isinstance(eos, Nasa9Mixture):
        fill_descriptor(d, eos)
    else:
        d.eos = abi.CLES_EOS_IDEAL
        d.T_guess = 300.0
        for k, s in enumerate(eos.sp):
            d.R[k] = s.R
            d.gamma[k] = s.gamma
    d.mu0, d.Pr, d.Sc = transport.mu0, transport.Pr, transport.Sc
    d.art_enabled = int(art.enabled)
    d.C_mu, d.C_beta, d.C_kappa, d.C_D = art.C_mu, art.C_beta, art.C_kappa, art.C_D
    d.beta_sensor = _BETA[art.beta_sensor]
    d.deriv = deriv
    d.filt = filt
    d.cfl = float(cfl)
    d.filter_interval = int(filter_interval)
    d.control = control.to_c()
    d.n_halo = int(n_halo)
    d.precision = abi.CLES_PREC_MIXED if precision == "mixed" else abi.CLES_PREC_FP64
    d.metric = (metric or CartesianMetric()).code
    if len(sources) > abi.CLES_MAX_BODY_FORCES:
        raise ValueError(f"at most {abi.CLES_MAX_BODY_FORCES} sources")
    for f, src in enumerate(sources):
        if not isinstance(src, ConstantBodyForce):
            raise ValueError("sources: ConstantBodyForce only")
        for a in range(3):
            d.body_force[f][a] = float(src.acceleration[a])
    d.n_body_forces = len(sources)
    keep = []
    for k in range(3):
        st = stretch[k]
        if st is None:
            continue
        n = int(n_global[k])
        if n < 2:
            raise ValueError(f"dimension {k + 1}: a stretched dimension must be resolved")
        xi = np.arange(n, dtype=np.float64) * (1.0 / (n - 1))
        xs = np.ascontiguousarray(np.broadcast_to(np.asarray(st.x(xi), dtype=np.float64), (n,)))
        ms = np.ascontiguousarray(np.broadcast_to(np.asarray(st.dxdxi(xi), dtype=np.float64), (n,)))
        keep += [xs, ms]
        d.stretch_x[k] = xs.ctypes.data_as(C.POINTER(C.c_double))
        d.stretch_dxdxi[k] = ms.ctypes.data_as(C.POINTER(C.c_double))
    d._stretch_keep = keep
    d._face_fns = face_fns
    d._eos = eos
    return d


def face_callbacks(desc):
    """ctypes callbacks (cles_face_fn) for the function-valued faces of a
    descriptor built by solver_desc: [(dim, side, which, callback)].  A
    Dirichlet face writes conserved_from_prim of fun(x, y, z, t); an NSCBC
    inflow face writes the target velocity, temperature and composition.
    An exception inside a function fills its face with NaN and is kept in
    `errors` (the run then fails as non-finite)."""
    out, errors = [], []
    eos = getattr(desc, "_eos", None) or eos_from_desc(desc)
    for k, s, which, code, fn in getattr(desc, "_face_fns", []):
        def cb(user, dim, side, t, npts, x1, x2, x3, o, fn=fn, code=code):
            n = int(npts)
            X = [np.ctypeslib.as_array(x, shape=(n,)) for x in (x1, x2, x3)]
            dst = np.ctypeslib.as_array(o, shape=((eos.nspecies + 4), n))
            try:
                pr = fn(X[0], X[1], X[2], float(t))
                if code == abi.CLES_BC_DIRICHLET:
                    vals = conserved_from_prim(eos, pr)
                else:
                    if pr.T_ion is None:
                        raise ValueError("NSCBCInflowBC target must specify T_ion")
                    if len(pr.Y) != eos.nspecies:
                        raise ValueError("NSCBCInflowBC target must carry the full composition")
                    vals = list(pr.u) + [pr.T_ion] + list(pr.Y)
                for c, v in enumerate(vals):
                    dst[c, :] = np.broadcast_to(np.asarray(v, dtype=np.float64), (n,))
            except Exception as e:   # noqa: BLE001 - reported through `errors`
                errors.append(e)
                dst[...] = np.nan
        out.append((k, s, which, abi.FACE_FN(cb)))
    return out, errors


def _folds(desc):
    """(fold at the low end, fold at the high end) per dimension (src/rhs.jl:149-197)."""
    lo0 = desc.bc[0][0] in (abi.CLES_BC_AXIS, abi.CLES_BC_ORIGIN)
    poles = desc.bc[1][0] == abi.CLES_BC_POLE and desc.bc[1][1] == abi.CLES_BC_POLE
    return (lo0, poles, False), (False, poles, False)


def stretched(desc, k):
    return bool(desc.stretch_x[k])


def grid_spacing(desc):
    """h per dimension (src/rhs.jl:191-204): 1 collapsed, 1/(N-1) stretched,
    L/N with folds at both ends, L/(N-1/2) with a fold at the low end, L/N
    periodic, L/(N-1) closed."""
    flo, fhi = _folds(desc)
    h = []
    for k in range(3):
        n = desc.n_global[k]
        if n == 1:
            h.append(1.0)
        elif stretched(desc, k):
            h.append(1.0 / (n - 1))
        elif flo[k] and fhi[k]:
            h.append(desc.L[k] / n)
        elif flo[k]:
            h.append(desc.L[k] / (n - 0.5))
        elif desc.bc[k][0] == abi.CLES_BC_PERIODIC:
            h.append(desc.L[k] / n)
        else:
            h.append(desc.L[k] / (n - 1))
    return tuple(h)


def coords(desc):
    """Interior node coordinates per dimension (global_xcoord, src/rhs.jl:331-335):
    origin + half-cell fold shift + i h, or the stretch map at the nodes."""
    h = grid_spacing(desc)
    flo, _ = _folds(desc)
    out = []
    for k in range(3):
        n = desc.n_global[k]
        if stretched(desc, k):
            out.append(np.array(desc.stretch_x[k][:n], dtype=np.float64))
            continue
        shift = h[k] / 2 if flo[k] else 0.0
        out.append((desc.origin[k] + shift) + np.arange(n) * h[k])
    return tuple(out)


def state_shape(desc, layout=abi.CLES_LAYOUT_PADDED):
    ncons = desc.n_species + 4
    sh = []
    for k in (2, 1, 0):
        n = desc.n_global[k]
        pad = desc.n_halo if (n > 1 and layout == abi.CLES_LAYOUT_PADDED) else 0
        sh.append(n + 2 * pad)
    return (ncons,) + tuple(sh)


def interior_slices(desc):
    sl = []
    for k in (2, 1, 0):
        n = desc.n_global[k]
        pad = desc.n_halo if n > 1 else 0
        sl.append(slice(pad, pad + n))
    return tuple(sl)


def eos_from_desc(desc):
    """The equation of state a descriptor carries."""
    if desc.eos == abi.CLES_EOS_NASA9:
        sp = []
        for k in range(desc.n_species):
            ivs = [Nasa9Interval(t.Tmin, t.Tmax, tuple(t.a[j] for j in range(7)), t.b1)
                   for t in list(desc.nasa9[k])[:desc.n_intervals[k]]]
            sp.append(Nasa9Species(f"species_{k}", desc.R[k], ivs))
        return Nasa9Mixture(sp, T_guess=desc.T_guess)
    return IdealMixture([IdealSpecies(f"species_{k}", desc.R[k], desc.gamma[k]) for k in range(desc.n_species)])


def initialize(desc, ic, eos=None, layout=abi.CLES_LAYOUT_PADDED, Q=None):
    """initialize!(solver, Q, ic) (src/problem.jl:146-163): evaluate ic at the
    interior nodes and write the conserved state; halos are left as they are
    (zero for a fresh array)."""
    eos = eos or eos_from_desc(desc)
    if Q is None:
        Q = np.zeros(state_shape(desc, layout))
    x, y, z = coords(desc)
    X = x[None, None, :]
    Y = y[None, :, None]
    Z = z[:, None, None]
    pr = ic(X, Y, Z)
    q = conserved_from_prim(eos, pr)
    shape = (desc.n_global[2], desc.n_global[1], desc.n_global[0])
    sl = interior_slices(desc) if layout == abi.CLES_LAYOUT_PADDED else (slice(None),) * 3
    for c, qc in enumerate(q):
        Q[(c,) + sl] = np.broadcast_to(np.asarray(qc, dtype=np.float64), shape)
    return Q


def problem_desc(prob, num, deriv, filt):
    """Split setup(prob, num) (src/problem.jl:321-345) into the descriptor."""
    origin = tuple(prob.domain[k][0] for k in range(3))
    L = tuple(prob.domain[k][1] - prob.domain[k][0] for k in range(3))
    if not all(v > 0 for v in L):
        raise ValueError("domain extents must be positive")
    return solver_desc(num.n_global, L, prob.bcs, deriv, filt, eos=prob.eos,
                       transport=prob.transport, art=num.art, origin=origin, cfl=num.cfl,
                       filter_interval=num.filter_interval, control=num.control,
                       n_halo=num.n_halo, precision=num.precision, metric=prob.metric,
                       stretch=num.stretch, sources=prob.sources)


# ------------------------------------------------------------- test cases ----
def taylor_green_problem(p0=71.43):
    """The README quick-start Taylor-Green vortex on [0, 2pi]^3 (README.md:31-39)."""
    two_pi = 2 * np.pi
    return Problem(domain=((0.0, two_pi), (0.0, two_pi), (0.0, two_pi)), bcs=PER3,
                   ic=lambda x, y, z: Prim(u=(np.sin(x) * np.cos(y), -np.cos(x) * np.sin(y), 0.0 * z),
                                           p=p0 + 0.0 * x, rho=1.0 + 0.0 * x),
                   name="taylor_green")
