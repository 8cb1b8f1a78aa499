"""ctypes mirror of include/cles.h: constants and descriptor structs.

This module has no dependencies beyond ctypes so that any ctypes client of a
library built on cles.h can load it by path.
"""
import ctypes as C

CLES_OK = 0
CLES_EINVAL = 1
CLES_ENOMEM = 2
CLES_ENUMERIC = 3
CLES_ETIMEOUT = 4
CLES_ECUDA = 5
CLES_EFAILURE = 6
CLES_EXCHANGE = 7

CLES_MAX_Q = 2
CLES_MAX_M = 4
CLES_MAX_NC = 4
CLES_MAX_CLO_LEN = 8
CLES_MAX_SPECIES = 8
CLES_MAX_BODY_FORCES = 4

CLES_F64 = 0
CLES_F32 = 1
CLES_LAYOUT_PADDED = 0
CLES_LAYOUT_INTERIOR = 1

CLES_BC_PERIODIC = 0
CLES_BC_SLIPWALL = 1
CLES_BC_DIRICHLET = 2

CLES_BETA_STRAIN = 0
CLES_BETA_GATED_STRAIN = 1
CLES_BETA_DILATATION = 2

CLES_PREC_FP64 = 0
CLES_PREC_MIXED = 1

CLES_FAIL_NONE = 0
CLES_FAIL_NONFINITE = 1
CLES_FAIL_NEGATIVE_DENSITY = 2
CLES_FAIL_PLANCK = 3
CLES_FAIL_DT_MIN = 4
CLES_FAIL_DT_COLLAPSE = 5
FAIL_NAMES = {
    CLES_FAIL_NONE: None,
    CLES_FAIL_NONFINITE: "nonfinite",
    CLES_FAIL_NEGATIVE_DENSITY: "negative_density",
    CLES_FAIL_PLANCK: "planck",
    CLES_FAIL_DT_MIN: "dt_min",
    CLES_FAIL_DT_COLLAPSE: "dt_collapse",
}

CLES_FIELD_RHO = 0
CLES_FIELD_U = 1
CLES_FIELD_V = 2
CLES_FIELD_W = 3
CLES_FIELD_P = 4
CLES_FIELD_T = 5
CLES_FIELD_C = 6
CLES_FIELD_CP = 7
CLES_FIELD_MU_ART = 8
CLES_FIELD_BETA_ART = 9
CLES_FIELD_KAPPA_ART = 10
CLES_FIELD_SENSOR = 11
CLES_FIELD_Y0 = 16
CLES_FIELD_D_ART0 = 32
CLES_FIELD_GRAD_U0 = 48


class cles_scheme(C.Structure):
    _fields_ = [
        ("name", C.c_char * 48),
        ("q", C.c_int),
        ("lhs", C.c_double * CLES_MAX_Q),
        ("a0", C.c_double),
        ("M", C.c_int),
        ("coeffs", C.c_double * CLES_MAX_M),
        ("symmetric", C.c_int),
        ("nc", C.c_int),
        ("clo_lhs", (C.c_double * (2 * CLES_MAX_Q + 1)) * CLES_MAX_NC),
        ("clo_len", C.c_int * CLES_MAX_NC),
        ("clo_rhs", (C.c_double * CLES_MAX_CLO_LEN) * CLES_MAX_NC),
    ]


class cles_grid(C.Structure):
    _fields_ = [
        ("n_global", C.c_int * 3),
        ("periodic", C.c_int * 3),
        ("n_halo", C.c_int),
    ]


class cles_split_desc(C.Structure):
    _fields_ = [
        ("n_local", C.c_int * 3),
        ("n_halo", C.c_int),
        ("dim", C.c_int),
        ("n_global", C.c_int),
        ("ranks", C.c_int),
        ("rank", C.c_int),
        ("periodic", C.c_int),
    ]


class cles_split_info(C.Structure):
    _fields_ = [
        ("halo_elems", C.c_int64),
        ("iface_elems", C.c_int64),
        ("field_elems", C.c_int64),
        ("prev", C.c_int),
        ("next", C.c_int),
        ("ranks", C.c_int),
        ("q", C.c_int),
        ("M", C.c_int),
    ]


class cles_step_control(C.Structure):
    _fields_ = [
        ("predict", C.c_double),
        ("max_growth", C.c_double),
        ("landing_steps", C.c_int),
        ("dt_min", C.c_double),
        ("dt_min_ratio", C.c_double),
        ("retries", C.c_int),
        ("cfl_backoff", C.c_double),
        ("savepoint_interval", C.c_int),
    ]


CLES_EOS_IDEAL = 0
CLES_EOS_NASA9 = 1
CLES_MAX_NASA9_INTERVALS = 4


class cles_nasa9_interval(C.Structure):
    _fields_ = [
        ("Tmin", C.c_double),
        ("Tmax", C.c_double),
        ("a", C.c_double * 7),
        ("b1", C.c_double),
    ]


CLES_BC_NOSLIP_WALL = 3
CLES_BC_EXTRAPOLATION = 4
CLES_BC_NSCBC_OUTFLOW = 5
CLES_BC_NSCBC_INFLOW = 6
CLES_BC_AXIS = 7
CLES_BC_ORIGIN = 8
CLES_BC_POLE = 9

# ---- decomposition (cles_decomp / cles_exchange) ----
CLES_REDUCE_MAX = 0
CLES_REDUCE_SUM = 1


class cles_decomp(C.Structure):
    _fields_ = [("dims", C.c_int * 3), ("coords", C.c_int * 3), ("rank", C.c_int)]


# halo(user, dim, prev, next, send_lo, send_hi, recv_lo, recv_hi, bytes, stream)
HALO_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                      C.c_void_p, C.c_int64, C.c_void_p)
# gather(user, dim, local, all, bytes, stream)
GATHER_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p)
# allreduce(user, op, vals, count)
ALLREDUCE_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int, C.POINTER(C.c_double), C.c_int)


class cles_exchange(C.Structure):
    _fields_ = [("user", C.c_void_p), ("halo", HALO_FN), ("gather", GATHER_FN), ("allreduce", ALLREDUCE_FN)]


# cles_face_fn: (user, dim, side, t, npts, x1, x2, x3, out)
FACE_FN = C.CFUNCTYPE(None, C.c_void_p, C.c_int, C.c_int, C.c_double, C.c_int64, C.POINTER(C.c_double),
                      C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double))

CLES_METRIC_CARTESIAN = 0
CLES_METRIC_CYLINDRICAL = 1
CLES_METRIC_SPHERICAL = 2


class cles_bc_params(C.Structure):
    _fields_ = [
        ("Twall", C.c_double),
        ("pinf", C.c_double),
        ("sigma", C.c_double),
        ("Lref", C.c_double),
        ("beta_t", C.c_double),
        ("u", C.c_double * 3),
        ("T_ion", C.c_double),
        ("Y", C.c_double * CLES_MAX_SPECIES),
        ("eta_u", C.c_double),
        ("eta_T", C.c_double),
        ("eta_t", C.c_double),
        ("eta_Y", C.c_double),
    ]


class cles_solver_desc(C.Structure):
    _fields_ = [
        ("n_global", C.c_int * 3),
        ("L", C.c_double * 3),
        ("origin", C.c_double * 3),
        ("bc", (C.c_int * 2) * 3),
        ("bc_state", ((C.c_double * (CLES_MAX_SPECIES + 4)) * 2) * 3),
        ("bc_params", (cles_bc_params * 2) * 3),
        ("bc_switchable", (C.c_int * 2) * 3),
        ("bc_after", (C.c_int * 2) * 3),
        ("bc_after_params", (cles_bc_params * 2) * 3),
        ("bc_after_state", ((C.c_double * (CLES_MAX_SPECIES + 4)) * 2) * 3),
        ("n_species", C.c_int),
        ("R", C.c_double * CLES_MAX_SPECIES),
        ("gamma", C.c_double * CLES_MAX_SPECIES),
        ("mu0", C.c_double),
        ("Pr", C.c_double),
        ("Sc", C.c_double),
        ("art_enabled", C.c_int),
        ("C_mu", C.c_double),
        ("C_beta", C.c_double),
        ("C_kappa", C.c_double),
        ("C_D", C.c_double),
        ("beta_sensor", C.c_int),
        ("deriv", cles_scheme),
        ("filt", cles_scheme),
        ("cfl", C.c_double),
        ("filter_interval", C.c_int),
        ("control", cles_step_control),
        ("n_halo", C.c_int),
        ("precision", C.c_int),
        ("eos", C.c_int),
        ("T_guess", C.c_double),
        ("n_intervals", C.c_int * CLES_MAX_SPECIES),
        ("nasa9", (cles_nasa9_interval * CLES_MAX_NASA9_INTERVALS) * CLES_MAX_SPECIES),
        ("metric", C.c_int),
        ("stretch_x", C.POINTER(C.c_double) * 3),
        ("stretch_dxdxi", C.POINTER(C.c_double) * 3),
        ("n_body_forces", C.c_int),
        ("body_force", (C.c_double * 3) * CLES_MAX_BODY_FORCES),
    ]


class cles_solver_info(C.Structure):
    _fields_ = [
        ("n_local", C.c_int * 3),
        ("active", C.c_int * 3),
        ("h", C.c_double * 3),
        ("n_cons", C.c_int),
        ("n_species", C.c_int),
        ("cells", C.c_int64),
        ("padded_cells", C.c_int64),
        ("device_bytes", C.c_size_t),
    ]


class cles_run_result(C.Structure):
    _fields_ = [
        ("steps", C.c_int64),
        ("t", C.c_double),
        ("last_dt", C.c_double),
        ("cfl", C.c_double),
        ("failure", C.c_int),
        ("retries_used", C.c_int),
    ]


def step_control_default():
    """StepControl() defaults (src/stepcontrol.jl:116-125)."""
    c = cles_step_control()
    c.predict = 0.0
    c.max_growth = 0.0
    c.landing_steps = 2
    c.dt_min = 0.0
    c.dt_min_ratio = 1e-8
    c.retries = 0
    c.cfl_backoff = 0.5
    c.savepoint_interval = 25
    return c


class cles_profile_entry(C.Structure):
    _fields_ = [
        ("name", C.c_char * 32),
        ("launches", C.c_int64),
        ("total_ms", C.c_double),
        ("bytes", C.c_double),
    ]


CLES_REQ_QUEUED = 0
CLES_REQ_RUNNING = 1
CLES_REQ_DONE = 2
CLES_REQ_FAILED = 3
CLES_REQ_CANCELLED = 4
REQ_STATES = {0: "queued", 1: "running", 2: "done", 3: "failed", 4: "cancelled"}


class cles_batch_tuning(C.Structure):
    _fields_ = [
        ("op", C.c_int),
        ("dim", C.c_int),
        ("threads", C.c_int),
        ("smem", C.c_int64),
        ("ctas", C.c_int),
        ("tuned_ms", C.c_double),
    ]


class cles_batch_stats(C.Structure):
    _fields_ = [
        ("members", C.c_int),
        ("active", C.c_int),
        ("compositions", C.c_int),
        ("steps", C.c_int64),
        ("launches_per_step", C.c_int),
        ("cells_total", C.c_int64),
        ("n_roles", C.c_int),
        ("tuning", cles_batch_tuning * 9),
    ]


class cles_request_status(C.Structure):
    _fields_ = [
        ("state", C.c_int),
        ("failure", C.c_int),
        ("steps", C.c_int64),
        ("t", C.c_double),
        ("submit_s", C.c_double),
        ("admit_s", C.c_double),
        ("done_s", C.c_double),
        ("device_bytes", C.c_size_t),
    ]
