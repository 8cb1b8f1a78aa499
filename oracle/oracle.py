"""ctypes wrapper of the CPU FP64 oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline / reference arm, always as the checker or the timed
CPU baseline, never as the product path.

Arrays are numpy float64 in the reference's padded layout: a scalar field has
shape (nz+2h, ny+2h, nx+2h) (C order, so x is fastest, as in Julia's
column-major (nx+2h, ny+2h, nz+2h)); a conserved state has the component as
the leading (slowest) axis.
"""
import ctypes as C
import importlib.util
import os
import pathlib
import subprocess

import numpy as np

_HERE = pathlib.Path(__file__).resolve().parent
_ROOT = _HERE.parent


def _load_abi():
    import sys
    # share the struct classes with an already-loaded package so descriptors
    # built by its host code can be passed here unchanged
    if "compactles_b200.abi" in sys.modules:
        return sys.modules["compactles_b200.abi"]
    path = _ROOT / "compactles.jl_b200" / "abi.py"
    spec = importlib.util.spec_from_file_location("_cles_abi_for_oracle", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


abi = _load_abi()
_DP = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")


def build():
    """Compile liboracle.so (make in oracle/)."""
    subprocess.run(["make", "-s", "-C", str(_HERE)], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        so = _HERE / "liboracle.so"
        if not so.exists():
            build()
        L = C.CDLL(str(so))
        L.orc_last_error.restype = C.c_char_p
        L.orc_set_threads.argtypes = [C.c_int]
        for nm in ("orc_scheme_lele_d1_6", "orc_scheme_pade_d1_4", "orc_scheme_lele_d1_10"):
            getattr(L, nm).argtypes = [C.POINTER(abi.cles_scheme)]
        L.orc_scheme_compact_filter.argtypes = [C.c_double, C.POINTER(abi.cles_scheme)]
        L.orc_plan_create.restype = C.c_void_p
        L.orc_plan_create.argtypes = [C.POINTER(abi.cles_grid), C.POINTER(abi.cles_scheme), C.c_int, C.c_double, C.c_int]
        L.orc_plan_destroy.argtypes = [C.c_void_p]
        L.orc_apply_along.argtypes = [C.c_void_p, _DP, _DP]
        L.orc_exchange_halos.argtypes = [C.POINTER(abi.cles_grid), _DP]
        L.orc_exchange_dim.argtypes = [C.POINTER(abi.cles_grid), _DP, C.c_int]
        L.orc_solver_create.restype = C.c_void_p
        L.orc_solver_create.argtypes = [C.POINTER(abi.cles_solver_desc)]
        L.orc_solver_split.argtypes = [C.c_void_p, C.c_int, C.c_int]
        L.orc_band_solve.argtypes = [C.c_int, C.c_int, _DP, _DP]
        L.orc_volume_integral.argtypes = [C.c_void_p, _DP]
        L.orc_volume_integral.restype = C.c_double
        L.orc_solver_destroy.argtypes = [C.c_void_p]
        L.orc_field_size.restype = C.c_int64
        L.orc_field_size.argtypes = [C.c_void_p]
        for nm in ("orc_set_state", "orc_get_state", "orc_get_rhs"):
            getattr(L, nm).argtypes = [C.c_void_p, _DP]
        L.orc_apply_bcs.argtypes = [C.c_void_p]
        L.orc_compute_rhs.argtypes = [C.c_void_p, C.c_int]
        L.orc_max_rate.argtypes = [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.orc_step.argtypes = [C.c_void_p, C.c_double, C.c_int]
        L.orc_filter_state.argtypes = [C.c_void_p]
        L.orc_run.argtypes = [C.c_void_p, C.c_double, C.c_int64, C.POINTER(abi.cles_run_result)]
        for nm in ("orc_nasa9_cp", "orc_nasa9_h", "orc_nasa9_e"):
            getattr(L, nm).restype = C.c_double
            getattr(L, nm).argtypes = [C.POINTER(abi.cles_solver_desc), C.c_int, C.c_double]
        L.orc_nasa9_temperature.restype = C.c_double
        L.orc_nasa9_temperature.argtypes = [C.POINTER(abi.cles_solver_desc), C.c_double, _DP]
        L.orc_switch_bc.argtypes = [C.c_void_p, C.c_int, C.c_int]
        L.orc_kinetic_energy.restype = C.c_double
        L.orc_kinetic_energy.argtypes = [C.c_void_p]
        L.orc_dissipation_rate.restype = C.c_double
        L.orc_dissipation_rate.argtypes = [C.c_void_p]
        L.orc_get_clock.argtypes = [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int64), C.POINTER(C.c_double)]
        L.orc_set_clock.argtypes = [C.c_void_p, C.c_double, C.c_int64, C.c_double]
        L.orc_get_field.argtypes = [C.c_void_p, C.c_int, _DP]
        L.orc_get_flux.argtypes = [C.c_void_p, C.c_int, C.c_int, _DP]
        L.orc_check_step.argtypes = [C.POINTER(abi.cles_step_control), C.c_double, C.c_double, C.c_double]
        L.orc_get_geometry.argtypes = [C.c_void_p, C.c_int, _DP]
        L.orc_grid_spacing.argtypes = [C.c_void_p, _DP, _DP, _DP]
        L.orc_solver_deriv.argtypes = [C.c_void_p, _DP, _DP, C.c_int, C.c_int, C.c_int]
        L.orc_solver_filter.argtypes = [C.c_void_p, _DP, _DP, C.c_int, C.c_int]
        L.orc_solver_set_face_fn.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, abi.FACE_FN, C.c_void_p]
        _lib = L
    return _lib


def set_threads(n):
    return lib().orc_set_threads(int(n))


def _err():
    return lib().orc_last_error().decode()


# ---------------------------------------------------------------- schemes --
def lele_d1_6():
    s = abi.cles_scheme()
    lib().orc_scheme_lele_d1_6(C.byref(s))
    return s


def pade_d1_4():
    s = abi.cles_scheme()
    lib().orc_scheme_pade_d1_4(C.byref(s))
    return s


def compact_filter(alphaf=0.45):
    s = abi.cles_scheme()
    lib().orc_scheme_compact_filter(float(alphaf), C.byref(s))
    return s


def lele_d1_10():
    s = abi.cles_scheme()
    lib().orc_scheme_lele_d1_10(C.byref(s))
    return s


# ------------------------------------------------------------------- grids --
def grid(n_global, periodic, n_halo=4):
    g = abi.cles_grid()
    for d in range(3):
        g.n_global[d] = int(n_global[d])
        g.periodic[d] = int(bool(periodic[d]))
    g.n_halo = int(n_halo)
    return g


def padded_shape(g):
    nh = [g.n_halo if g.n_global[d] > 1 else 0 for d in range(3)]
    return tuple(g.n_global[d] + 2 * nh[d] for d in (2, 1, 0))


def interior(g, f):
    """Interior view (nz, ny, nx) of a padded field or (..., nz, ny, nx) state."""
    nh = [g.n_halo if g.n_global[d] > 1 else 0 for d in range(3)]
    sl = tuple(slice(nh[d], nh[d] + g.n_global[d]) for d in (2, 1, 0))
    return f[(Ellipsis,) + sl]


def exchange_halos(g, f):
    lib().orc_exchange_halos(C.byref(g), f)
    return f


def exchange_dim(g, f, dim):
    lib().orc_exchange_dim(C.byref(g), f, int(dim))
    return f


class Plan:
    """plan_direction(decomp, scheme, dim, h) with P emulated ranks along dim."""

    def __init__(self, g, scheme, dim, h, P=1):
        self.g = g
        self.scheme = scheme
        self.h = h
        self.ptr = lib().orc_plan_create(C.byref(g), C.byref(scheme), int(dim), float(h), int(P))
        if not self.ptr:
            raise ValueError(_err())
        self.dim = dim

    def apply(self, f, out=None):
        """apply_along!(out, plan, f, decomp); f needs current halos."""
        if out is None:
            out = np.zeros_like(f)
        lib().orc_apply_along(self.ptr, np.ascontiguousarray(f), out)
        return out

    def __del__(self):
        try:
            if getattr(self, "ptr", None):
                lib().orc_plan_destroy(self.ptr)
                self.ptr = None
        except Exception:
            pass


def band_solve(A, b, q):
    """BandFactor(Ab, q) + solve_col! on the dense n x n banded matrix A."""
    n = A.shape[0]
    Ab = np.zeros((n, 2 * q + 1))
    for i in range(n):
        for t in range(-q, q + 1):
            if 0 <= i + t < n:
                Ab[i, q + t] = A[i, i + t]
    x = np.ascontiguousarray(b, dtype=np.float64).copy()
    if lib().orc_band_solve(int(q), int(n), np.ascontiguousarray(Ab), x):
        raise ValueError(_err())
    return x


class Solver:
    """The oracle Solver; state arrays in the padded layout."""

    def __init__(self, desc):
        self.desc = desc
        self.ptr = lib().orc_solver_create(C.byref(desc))
        if not self.ptr:
            raise ValueError(_err())
        self.g = grid(desc.n_global, [desc.bc[d][0] == abi.CLES_BC_PERIODIC for d in range(3)], desc.n_halo)
        self.n_cons = desc.n_species + 4
        self.field_shape = padded_shape(self.g)
        self.state_shape = (self.n_cons,) + self.field_shape
        # function-valued faces, through the package's callback builder when present
        self._face_cbs, self.face_errors = [], []
        if getattr(desc, "_face_fns", None):
            import sys
            self._face_cbs, self.face_errors = sys.modules["compactles_b200"].problem.face_callbacks(desc)
        for k, s, which, cb in self._face_cbs:
            if lib().orc_solver_set_face_fn(self.ptr, k, s, which, cb, None):
                raise ValueError(_err())

    def __del__(self):
        try:
            if getattr(self, "ptr", None):
                lib().orc_solver_destroy(self.ptr)
                self.ptr = None
        except Exception:
            pass

    def set_state(self, Q):
        Q = np.ascontiguousarray(Q, dtype=np.float64)
        assert Q.shape == self.state_shape, (Q.shape, self.state_shape)
        lib().orc_set_state(self.ptr, Q)

    def get_state(self):
        Q = np.zeros(self.state_shape)
        lib().orc_get_state(self.ptr, Q)
        return Q

    def get_rhs(self):
        dQ = np.zeros(self.state_shape)
        lib().orc_get_rhs(self.ptr, dQ)
        return dQ

    def apply_bcs(self):
        lib().orc_apply_bcs(self.ptr)

    def compute_rhs(self, primitives_current=False):
        lib().orc_compute_rhs(self.ptr, int(primitives_current))
        return self.get_rhs()

    def max_rate(self):
        r, m = C.c_double(), C.c_double()
        lib().orc_max_rate(self.ptr, C.byref(r), C.byref(m))
        return r.value, m.value

    def step(self, dt, prepared=False):
        lib().orc_step(self.ptr, float(dt), int(prepared))

    def filter_state(self):
        lib().orc_filter_state(self.ptr)

    def run(self, tfinal, nmax=2**62):
        res = abi.cles_run_result()
        rc = lib().orc_run(self.ptr, float(tfinal), int(nmax), C.byref(res))
        return rc, res

    def volume_integral(self, f):
        """volume_integral(solver, f) of a padded field (src/diagnostics.jl:41-80)."""
        f = np.ascontiguousarray(f, dtype=np.float64)
        if f.shape != self.field_shape:
            raise ValueError(f"field shape {f.shape} is not the solver's {self.field_shape}")
        return float(lib().orc_volume_integral(self.ptr, f))

    def split(self, dim, P):
        """Emulate P ranks along dim (1-based) in every compact application along it."""
        if lib().orc_solver_split(self.ptr, int(dim), int(P)):
            raise ValueError(_err())
        return self

    def switch_bc(self, dim, side):
        """switch!(::SwitchableBC) on face (dim 1..3, side 1 low / 2 high)."""
        if lib().orc_switch_bc(self.ptr, int(dim) - 1, int(side) - 1):
            raise ValueError(_err())

    def field(self, which):
        out = np.zeros(self.field_shape)
        rc = lib().orc_get_field(self.ptr, int(which), out)
        if rc:
            raise ValueError(_err())
        return out

    def flux(self, d, c):
        """flux[d][c] (0-based) of the last compute_rhs, padded."""
        out = np.zeros(self.field_shape)
        if lib().orc_get_flux(self.ptr, int(d), int(c), out):
            raise ValueError(_err())
        return out

    def rhs_scales(self, h):
        """Per conserved component, max over dims and points of |F_dc| / h_d: the size of
        the directional flux-divergence terms whose sum is the RHS."""
        sl = interior(self.g, np.zeros(self.field_shape))
        out = []
        for c in range(self.n_cons):
            m = 0.0
            for d in range(3):
                if self.desc.n_global[d] > 1:
                    m = max(m, float(np.abs(interior(self.g, self.flux(d, c))).max()) / h[d])
            out.append(m)
        return out

    def clock(self):
        t, s, c = C.c_double(), C.c_int64(), C.c_double()
        lib().orc_get_clock(self.ptr, C.byref(t), C.byref(s), C.byref(c))
        return t.value, s.value, c.value

    def set_clock(self, t, step, cfl):
        lib().orc_set_clock(self.ptr, float(t), int(step), float(cfl))

    def kinetic_energy(self):
        return lib().orc_kinetic_energy(self.ptr)

    GEOMETRY = {"inv_J": 0, "A1": 1, "A2": 2, "A3": 3, "inv_h1": 4, "inv_h2": 5, "inv_h3": 6,
                "inv_r": 7, "cot_over_r": 8}

    def geometry(self, name):
        """A geometry array of init_geometry! (src/metric.jl:109-150), padded."""
        out = np.zeros(self.field_shape)
        if lib().orc_get_geometry(self.ptr, self.GEOMETRY[name], out):
            raise ValueError(_err())
        return out

    def spacing(self):
        """(h, coord_shift, origin) per dimension (src/rhs.jl:191-205, :286)."""
        h, sh, o = np.zeros(3), np.zeros(3), np.zeros(3)
        lib().orc_grid_spacing(self.ptr, h, sh, o)
        return h, sh, o

    def deriv(self, f, d, sig=1, scale=True):
        """deriv_along!(out, f, solver, d, sig) (+ _scale_grad!) on a padded field, d 1-based."""
        f = np.array(f, dtype=np.float64, order="C")
        out = np.zeros_like(f)
        if lib().orc_solver_deriv(self.ptr, f, out, int(d) - 1, int(sig), int(bool(scale))):
            raise ValueError(_err())
        return out

    def filt(self, f, d, sig=1):
        """filt_along!(out, f, solver, d, sig) on a padded field, d 1-based."""
        f = np.array(f, dtype=np.float64, order="C")
        out = np.zeros_like(f)
        if lib().orc_solver_filter(self.ptr, f, out, int(d) - 1, int(sig)):
            raise ValueError(_err())
        return out

    def dissipation_rate(self):
        return lib().orc_dissipation_rate(self.ptr)


def check_step(control, dt, rho_min, dt_seen):
    return abi.FAIL_NAMES[lib().orc_check_step(C.byref(control), float(dt), float(rho_min), float(dt_seen))]


def default_threads():
    return os.cpu_count() or 1


def nasa9_cp(desc, k, T):
    """species_cp of a NASA-9 descriptor (src/physics.jl:437-441)."""
    return lib().orc_nasa9_cp(C.byref(desc), int(k), float(T))


def nasa9_h(desc, k, T):
    """species_enthalpy (src/physics.jl:443-447)."""
    return lib().orc_nasa9_h(C.byref(desc), int(k), float(T))


def nasa9_e(desc, k, T):
    """species_energy (src/physics.jl:449-451)."""
    return lib().orc_nasa9_e(C.byref(desc), int(k), float(T))


def nasa9_temperature(desc, e, Y):
    """mixture_temperature (src/physics.jl:466-498)."""
    return lib().orc_nasa9_temperature(C.byref(desc), float(e), np.ascontiguousarray(Y, dtype=np.float64))
