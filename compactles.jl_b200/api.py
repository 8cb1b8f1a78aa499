"""ctypes host mirror of the reference's operator interface over libcles.so.

Names follow CompactLES.jl: plan_direction / apply_along (src/operators.jl),
Solver / compute_rhs / step / max_rate / filter_state / run
(src/rhs.jl, src/timestep.jl), check_step / SolverFailure
(src/stepcontrol.jl).  Every compute call goes through the CUDA library; if
libcles.so is missing or no B200 is visible these raise, there is no CPU
fallback.
"""
import ctypes as C
import os
import pathlib
import subprocess

import numpy as np

from . import abi
from .problem import face_callbacks, grid_spacing, state_shape

_HERE = pathlib.Path(__file__).resolve().parent
LIB_PATH = _HERE / "libcles.so"

_lib = None


class ClesError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"[cles status {code}] {msg}")
        self.code = code


class SolverFailure(RuntimeError):
    """Raised by run when step control rejects a step (src/stepcontrol.jl:145-152)."""

    def __init__(self, reason, result):
        super().__init__(f"SolverFailure(:{reason}) at t = {result.t}, cfl = {result.cfl}")
        self.reason = reason
        self.result = result


def build(jobs=8):
    """Compile libcles.so in place (nvcc, sm_100a)."""
    subprocess.run(["make", "-s", "-j", str(jobs), "-C", str(_HERE / "csrc")], check=True)


def lib():
    """The loaded libcles.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ClesError(abi.CLES_ECUDA, f"{LIB_PATH} is missing: build it with compactles_b200.api.build()")
        L = C.CDLL(str(LIB_PATH))
        vp = C.c_void_p
        dp = C.POINTER(C.c_double)
        L.cles_last_error.restype = C.c_char_p
        L.cles_kernel_launches.restype = C.c_int64
        for nm in ("cles_scheme_lele_d1_6", "cles_scheme_pade_d1_4", "cles_scheme_lele_d1_10"):
            getattr(L, nm).argtypes = [C.POINTER(abi.cles_scheme)]
        L.cles_scheme_compact_filter.argtypes = [C.c_double, C.POINTER(abi.cles_scheme)]
        L.cles_ctx_create.argtypes = [C.c_int, vp, C.c_size_t, C.POINTER(vp)]
        L.cles_ctx_destroy.argtypes = [vp]
        L.cles_ctx_set_stream.argtypes = [vp, vp]
        L.cles_selftest_bounded_wait.argtypes = [vp, C.c_int64]
        L.cles_plan_create.argtypes = [vp, C.POINTER(abi.cles_grid), C.POINTER(abi.cles_scheme), C.c_int, C.c_double,
                                       C.c_int, C.c_int, C.POINTER(vp)]
        L.cles_plan_destroy.argtypes = [vp]
        L.cles_apply_along.argtypes = [vp, vp, vp]
        L.cles_apply_along_batch.argtypes = [vp, vp, vp, C.c_int, C.c_int64]
        L.cles_apply_along_host.argtypes = [vp, vp, vp]
        L.cles_split_plan_create.argtypes = [vp, C.POINTER(abi.cles_split_desc), C.POINTER(abi.cles_scheme),
                                             C.c_double, C.c_int, C.POINTER(vp)]
        L.cles_split_plan_destroy.argtypes = [vp]
        L.cles_split_plan_info.argtypes = [vp, C.POINTER(abi.cles_split_info)]
        L.cles_split_halo_pack.argtypes = [vp, vp, vp, vp, C.c_int, C.c_int64]
        L.cles_split_halo_unpack.argtypes = [vp, vp, vp, vp, C.c_int, C.c_int64]
        L.cles_split_apply_begin.argtypes = [vp, vp, vp, vp, C.c_int, C.c_int64]
        L.cles_split_apply_end.argtypes = [vp, vp, vp, C.c_int, C.c_int64]
        L.cles_solver_switch_bc.argtypes = [vp, C.c_int, C.c_int]
        L.cles_solver_set_face_fn.argtypes = [vp, C.c_int, C.c_int, C.c_int, abi.FACE_FN, vp]
        L.cles_solver_bc_switched.argtypes = [vp, C.c_int, C.c_int, C.POINTER(C.c_int)]
        L.cles_checkpoint_save.argtypes = [vp, C.c_char_p]
        L.cles_checkpoint_load.argtypes = [vp, C.c_char_p]
        L.cles_step_control_default.argtypes = [C.POINTER(abi.cles_step_control)]
        L.cles_step_control_default.restype = None
        L.cles_solver_desc_default.argtypes = [C.POINTER(abi.cles_solver_desc)]
        L.cles_solver_desc_default.restype = None
        L.cles_solver_create.argtypes = [vp, C.POINTER(abi.cles_solver_desc), C.POINTER(vp)]
        L.cles_solver_create_decomposed.argtypes = [vp, C.POINTER(abi.cles_solver_desc), C.POINTER(abi.cles_decomp),
                                                    C.POINTER(abi.cles_exchange), C.POINTER(vp)]
        L.cles_local_group_create.argtypes = [C.POINTER(C.c_int), C.c_double, C.POINTER(vp)]
        L.cles_local_group_destroy.argtypes = [vp]
        L.cles_local_group_destroy.restype = None
        L.cles_local_group_exchange.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(abi.cles_exchange)]
        L.cles_local_group_abort.argtypes = [vp]
        L.cles_local_group_abort.restype = None
        L.cles_solver_destroy.argtypes = [vp]
        L.cles_solver_info_get.argtypes = [vp, C.POINTER(abi.cles_solver_info)]
        L.cles_set_state.argtypes = [vp, vp, C.c_int]
        L.cles_get_state.argtypes = [vp, vp, C.c_int]
        L.cles_state_device.argtypes = [vp, C.POINTER(dp)]
        L.cles_apply_bcs.argtypes = [vp]
        L.cles_max_rate.argtypes = [vp, dp, dp]
        L.cles_compute_rhs.argtypes = [vp, C.c_int]
        L.cles_get_rhs.argtypes = [vp, vp, C.c_int]
        L.cles_step.argtypes = [vp, C.c_double, C.c_int]
        L.cles_filter_state.argtypes = [vp]
        L.cles_get_field.argtypes = [vp, C.c_int, vp, C.c_int]
        L.cles_get_clock.argtypes = [vp, dp, C.POINTER(C.c_int64), dp]
        L.cles_set_clock.argtypes = [vp, C.c_double, C.c_int64, C.c_double]
        L.cles_check_step.argtypes = [C.POINTER(abi.cles_step_control), C.c_double, C.c_double, C.c_double, C.c_int64,
                                      C.c_double, C.c_double, C.POINTER(C.c_int)]
        L.cles_run.argtypes = [vp, C.c_double, C.c_int64, C.POINTER(abi.cles_run_result)]
        L.cles_step_host.argtypes = [vp, vp, C.c_int, C.c_double, C.POINTER(abi.cles_run_result)]
        L.cles_profile_enable.argtypes = [C.c_int]
        L.cles_profile_read.argtypes = [C.POINTER(abi.cles_profile_entry), C.c_int, C.POINTER(C.c_int)]
        L.cles_max_rate_static.argtypes = [vp, vp, C.c_int64, C.c_int, dp, dp, dp, C.c_double, C.c_double,
                                           C.c_double, vp, vp]
        L.cles_run_graph.argtypes = [vp, C.c_double, C.c_int64, C.POINTER(abi.cles_run_result)]
        L.cles_server_create.argtypes = [C.c_int, C.c_size_t, C.c_int, C.POINTER(vp)]
        L.cles_server_destroy.argtypes = [vp]
        L.cles_server_submit.argtypes = [vp, C.POINTER(abi.cles_solver_desc), vp, C.c_int, C.c_double, C.c_int64,
                                         C.POINTER(C.c_int64)]
        L.cles_server_tick.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.cles_server_status.argtypes = [vp, C.c_int64, C.POINTER(abi.cles_request_status)]
        L.cles_server_fetch.argtypes = [vp, C.c_int64, vp]
        L.cles_server_cancel.argtypes = [vp, C.c_int64]
        L.cles_server_set_batching.argtypes = [vp, C.c_int, C.c_int]
        L.cles_batch_create.argtypes = [vp, C.POINTER(abi.cles_solver_desc), C.POINTER(vp)]
        L.cles_batch_destroy.argtypes = [vp]
        L.cles_batch_destroy.restype = None
        L.cles_batch_add.argtypes = [vp, C.POINTER(abi.cles_solver_desc), vp, C.c_int, C.c_double, C.c_int64,
                                     C.POINTER(C.c_int64)]
        L.cles_batch_step.argtypes = [vp, C.POINTER(C.c_int)]
        L.cles_batch_run.argtypes = [vp, C.c_int64, C.POINTER(C.c_int)]
        L.cles_batch_status.argtypes = [vp, C.c_int64, C.POINTER(abi.cles_request_status)]
        L.cles_batch_fetch.argtypes = [vp, C.c_int64, vp]
        L.cles_batch_cancel.argtypes = [vp, C.c_int64]
        L.cles_batch_stats_get.argtypes = [vp, C.POINTER(abi.cles_batch_stats)]
        L.cles_batch_set_strategy.argtypes = [vp, C.c_int]
        L.cles_kinetic_energy.argtypes = [vp, dp]
        L.cles_dissipation_rate.argtypes = [vp, dp]
        _lib = L
    return _lib


def _check(rc):
    if rc != abi.CLES_OK:
        raise ClesError(rc, lib().cles_last_error().decode())


def kernel_launches():
    return int(lib().cles_kernel_launches())


def profile_enable(on=True):
    """Bracket every compact-operator launch with CUDA events from now on (clears records)."""
    _check(lib().cles_profile_enable(int(on)))


def profile_read():
    """{name: (launches, total_ms, algorithmic_bytes)} per direction since profile_enable."""
    arr = (abi.cles_profile_entry * 8)()
    n = C.c_int()
    _check(lib().cles_profile_read(arr, 8, C.byref(n)))
    return {arr[i].name.decode(): (arr[i].launches, arr[i].total_ms, arr[i].bytes) for i in range(n.value)}


# ---------------------------------------------------------------- schemes ----
def lele_d1_6():
    s = abi.cles_scheme()
    _check(lib().cles_scheme_lele_d1_6(C.byref(s)))
    return s


def pade_d1_4():
    s = abi.cles_scheme()
    _check(lib().cles_scheme_pade_d1_4(C.byref(s)))
    return s


def compact_filter(alphaf=0.45):
    s = abi.cles_scheme()
    _check(lib().cles_scheme_compact_filter(float(alphaf), C.byref(s)))
    return s


def lele_d1_10():
    s = abi.cles_scheme()
    _check(lib().cles_scheme_lele_d1_10(C.byref(s)))
    return s


def check_step(control, dt, rho_min, dt_seen, step=0, t=0.0, cfl=0.5):
    """check_step (src/stepcontrol.jl:184-204) -> None or the failure reason."""
    r = C.c_int()
    _check(lib().cles_check_step(C.byref(control), float(dt), float(rho_min), float(dt_seen), int(step), float(t),
                                 float(cfl), C.byref(r)))
    return abi.FAIL_NAMES[r.value]


# ---------------------------------------------------------------- context ----
class Context:
    """Device + stream every call is ordered on (cles_ctx)."""

    def __init__(self, device=0, stream=None, hbm_budget=0):
        self.ptr = C.c_void_p()
        _check(lib().cles_ctx_create(int(device), C.c_void_p(stream or 0), int(hbm_budget), C.byref(self.ptr)))
        self.device = device

    def set_stream(self, stream):
        _check(lib().cles_ctx_set_stream(self.ptr, C.c_void_p(stream or 0)))

    def __del__(self):
        try:
            if self.ptr:
                lib().cles_ctx_destroy(self.ptr)
                self.ptr = None
        except Exception:
            pass


_default_ctx = None


def default_context():
    global _default_ctx
    if _default_ctx is None:
        _default_ctx = Context(int(os.environ.get("CLES_DEVICE", "0")))
    return _default_ctx


def grid(n_global, periodic, n_halo=4):
    g = abi.cles_grid()
    for d in range(3):
        g.n_global[d] = int(n_global[d])
        g.periodic[d] = int(bool(periodic[d]))
    g.n_halo = int(n_halo)
    return g


class DirPlan:
    """plan_direction(decomp, scheme, dim, h) (src/operators.jl:44-101, src/operators_banded.jl:29-125)."""

    def __init__(self, g, scheme, dim, h, dtype="f64", layout="padded", ctx=None):
        self.ctx = ctx or default_context()
        self.g = g
        self.dim = dim
        self.dtype = abi.CLES_F64 if dtype in ("f64", np.float64) else abi.CLES_F32
        self.layout = abi.CLES_LAYOUT_PADDED if layout == "padded" else abi.CLES_LAYOUT_INTERIOR
        self.ptr = C.c_void_p()
        _check(lib().cles_plan_create(self.ctx.ptr, C.byref(g), C.byref(scheme), int(dim), float(h), self.dtype,
                                      self.layout, C.byref(self.ptr)))

    def shape(self):
        sh = []
        for k in (2, 1, 0):
            n = self.g.n_global[k]
            pad = self.g.n_halo if (n > 1 and self.layout == abi.CLES_LAYOUT_PADDED) else 0
            sh.append(n + 2 * pad)
        return tuple(sh)

    def __del__(self):
        try:
            if self.ptr:
                lib().cles_plan_destroy(self.ptr)
                self.ptr = None
        except Exception:
            pass


plan_direction = DirPlan


def apply_along(out, plan, f):
    """apply_along!(out, plan, f) (src/operators.jl:199-215).

    numpy arrays: host path (copies through the plan's device buffers);
    torch CUDA tensors: device path on the context's stream.  Writes the
    interior of `out`."""
    if hasattr(f, "data_ptr") and getattr(f, "is_cuda", False):
        _check(lib().cles_apply_along(plan.ptr, C.c_void_p(f.data_ptr()), C.c_void_p(out.data_ptr())))
        return out
    want = np.float64 if plan.dtype == abi.CLES_F64 else np.float32
    if f.dtype != want or out.dtype != want or not f.flags.c_contiguous or not out.flags.c_contiguous:
        raise TypeError("apply_along host path needs C-contiguous arrays of the plan's dtype")
    if f.shape != plan.shape() or out.shape != plan.shape():
        raise ValueError(f"field shape {f.shape} does not match the plan's {plan.shape()}")
    _check(lib().cles_apply_along_host(plan.ptr, f.ctypes.data_as(C.c_void_p), out.ctypes.data_as(C.c_void_p)))
    return out


# ----------------------------------------------------------------- solver ----
class Solver:
    """Device-resident Solver (src/rhs.jl:17-72) built from a cles_solver_desc.

    With `decomp` (a decomp.Decomp or an abi.cles_decomp) and `exchange` (an
    object whose `.struct` is an abi.cles_exchange, e.g. decomp.LocalGroup's
    or decomp.TorchExchange's), the solver is one rank of a decomposed grid:
    `desc` describes the global problem and states, fields and checkpoints are
    this rank's block."""

    def __init__(self, desc, ctx=None, decomp=None, exchange=None):
        self.ctx = ctx or default_context()
        self.desc = desc
        self.ptr = C.c_void_p()
        if decomp is None:
            _check(lib().cles_solver_create(self.ctx.ptr, C.byref(desc), C.byref(self.ptr)))
        else:
            if exchange is None:
                raise ValueError("a decomposed solver needs an exchange")
            dc = decomp.struct() if hasattr(decomp, "struct") else decomp
            self._exchange = exchange   # the callbacks must outlive the solver
            _check(lib().cles_solver_create_decomposed(self.ctx.ptr, C.byref(desc), C.byref(dc),
                                                       C.byref(exchange.struct), C.byref(self.ptr)))
        self.n_cons = desc.n_species + 4
        self.h = grid_spacing(desc)
        inf = self.info()
        self.n_local = tuple(int(v) for v in inf.n_local)
        # DirichletBC(fun) / NSCBCInflowBC(target=fun) faces, called back at the stage times
        self._face_cbs, self.face_errors = face_callbacks(desc)
        for k, s, which, cb in self._face_cbs:
            _check(lib().cles_solver_set_face_fn(self.ptr, k, s, which, cb, None))

    def __del__(self):
        try:
            if self.ptr:
                lib().cles_solver_destroy(self.ptr)
                self.ptr = None
        except Exception:
            pass

    def info(self):
        i = abi.cles_solver_info()
        _check(lib().cles_solver_info_get(self.ptr, C.byref(i)))
        return i

    def state_shape(self, layout=abi.CLES_LAYOUT_PADDED):
        """Host state shape (component, z, y, x) of this solver's block."""
        sh = []
        for k in (2, 1, 0):
            n = self.n_local[k]
            pad = self.desc.n_halo if (self.desc.n_global[k] > 1 and layout == abi.CLES_LAYOUT_PADDED) else 0
            sh.append(n + 2 * pad)
        return (self.n_cons,) + tuple(sh)

    def _arr(self, layout, ncomp=None):
        sh = self.state_shape(layout)
        if ncomp is not None:
            sh = (ncomp,) + sh[1:]
        return np.zeros(sh)

    @staticmethod
    def _layout(layout):
        return abi.CLES_LAYOUT_PADDED if layout == "padded" else abi.CLES_LAYOUT_INTERIOR

    def set_state(self, Q, layout="padded"):
        Q = np.ascontiguousarray(Q, dtype=np.float64)
        lay = self._layout(layout)
        if Q.shape != self.state_shape(lay):
            raise ValueError(f"state shape {Q.shape} != {self.state_shape(lay)}")
        _check(lib().cles_set_state(self.ptr, Q.ctypes.data_as(C.c_void_p), lay))

    def get_state(self, layout="padded"):
        lay = self._layout(layout)
        Q = self._arr(lay)
        _check(lib().cles_get_state(self.ptr, Q.ctypes.data_as(C.c_void_p), lay))
        return Q

    def apply_bcs(self):
        _check(lib().cles_apply_bcs(self.ptr))

    def max_rate(self):
        r, m = C.c_double(), C.c_double()
        _check(lib().cles_max_rate(self.ptr, C.byref(r), C.byref(m)))
        return r.value, m.value

    def compute_rhs(self, primitives_current=False, layout="padded"):
        _check(lib().cles_compute_rhs(self.ptr, int(primitives_current)))
        lay = self._layout(layout)
        dQ = self._arr(lay)
        _check(lib().cles_get_rhs(self.ptr, dQ.ctypes.data_as(C.c_void_p), lay))
        return dQ

    def step(self, dt, prepared=False):
        _check(lib().cles_step(self.ptr, float(dt), int(prepared)))

    def filter_state(self):
        _check(lib().cles_filter_state(self.ptr))

    def field(self, which, layout="padded"):
        lay = self._layout(layout)
        out = self._arr(lay, ncomp=1)[0]
        _check(lib().cles_get_field(self.ptr, int(which), out.ctypes.data_as(C.c_void_p), lay))
        return out

    def clock(self):
        t, s, c = C.c_double(), C.c_int64(), C.c_double()
        _check(lib().cles_get_clock(self.ptr, C.byref(t), C.byref(s), C.byref(c)))
        return t.value, s.value, c.value

    def set_clock(self, t, step, cfl):
        _check(lib().cles_set_clock(self.ptr, float(t), int(step), float(cfl)))

    def switch_bc(self, dim, side):
        """switch!(bc) for the SwitchableBC on face (dim 1..3, side 1 low / 2 high)
        (src/boundary.jl:150-160); idempotent."""
        _check(lib().cles_solver_switch_bc(self.ptr, int(dim) - 1, int(side) - 1))

    def switched(self, dim, side):
        out = C.c_int()
        _check(lib().cles_solver_bc_switched(self.ptr, int(dim) - 1, int(side) - 1, C.byref(out)))
        return bool(out.value)

    def save_checkpoint(self, prefix):
        """save_checkpoint(solver, Q, prefix) (src/io.jl:8-41): writes prefix.rNNNN.ckpt
        (NNNN: the decomposition's rank, 0000 on one rank)."""
        _check(lib().cles_checkpoint_save(self.ptr, str(prefix).encode()))
        return str(prefix)

    def load_checkpoint(self, prefix):
        """load_checkpoint!(solver, Q, prefix) (src/io.jl:43-72)."""
        _check(lib().cles_checkpoint_load(self.ptr, str(prefix).encode()))

    @property
    def t(self):
        return self.clock()[0]

    @property
    def steps(self):
        return self.clock()[1]

    def run(self, tfinal, nmax=2 ** 62, raise_on_failure=True):
        """run!(solver, Q; tfinal, nmax) without callbacks (src/timestep.jl:277-405)."""
        res = abi.cles_run_result()
        rc = lib().cles_run(self.ptr, float(tfinal), int(nmax), C.byref(res))
        if rc == abi.CLES_EFAILURE:
            if raise_on_failure:
                raise SolverFailure(abi.FAIL_NAMES[res.failure], res)
            return res
        _check(rc)
        return res

    def run_graph(self, tfinal, nmax=2 ** 62, raise_on_failure=True):
        """run! with every step as one CUDA-graph launch (device-side dt and floors)."""
        res = abi.cles_run_result()
        rc = lib().cles_run_graph(self.ptr, float(tfinal), int(nmax), C.byref(res))
        if rc == abi.CLES_EFAILURE:
            if raise_on_failure:
                raise SolverFailure(abi.FAIL_NAMES[res.failure], res)
            return res
        _check(rc)
        return res

    def step_host(self, Q, tfinal, layout="padded"):
        """One run! iteration on a host state array, updated in place."""
        res = abi.cles_run_result()
        rc = lib().cles_step_host(self.ptr, Q.ctypes.data_as(C.c_void_p), self._layout(layout), float(tfinal),
                                  C.byref(res))
        if rc not in (abi.CLES_OK, abi.CLES_EFAILURE):
            _check(rc)
        return res

    def kinetic_energy(self):
        v = C.c_double()
        _check(lib().cles_kinetic_energy(self.ptr, C.byref(v)))
        return v.value

    def dissipation_rate(self):
        v = C.c_double()
        _check(lib().cles_dissipation_rate(self.ptr, C.byref(v)))
        return v.value


def setup(prob, num, ctx=None):
    """setup(prob, num) -> (solver, Q) (src/problem.jl:321-345); Q is the padded host state,
    already uploaded to the device solver."""
    from .problem import initialize, problem_desc
    deriv = num.deriv if num.deriv is not None else lele_d1_6()
    filt = num.filt if num.filt is not None else compact_filter(0.45)
    desc = problem_desc(prob, num, deriv, filt)
    s = Solver(desc, ctx=ctx)
    Q = initialize(desc, prob.ic, eos=prob.eos)
    s.set_state(Q)
    return s, Q


class Server:
    """Continuous-batching server of independent solves on one device (cles_server_*)."""

    def __init__(self, device=0, hbm_budget=0, max_active=64, batching=False, batch_members=0):
        self.ptr = C.c_void_p()
        _check(lib().cles_server_create(int(device), int(hbm_budget), int(max_active), C.byref(self.ptr)))
        self._layout = {}
        if batching:
            _check(lib().cles_server_set_batching(self.ptr, 1, int(batch_members)))

    def __del__(self):
        try:
            if self.ptr:
                lib().cles_server_destroy(self.ptr)
                self.ptr = None
        except Exception:
            pass

    def submit(self, desc, Q0, tfinal, nmax=2 ** 62, layout="padded"):
        Q0 = np.ascontiguousarray(Q0, dtype=np.float64)
        lay = abi.CLES_LAYOUT_PADDED if layout == "padded" else abi.CLES_LAYOUT_INTERIOR
        rid = C.c_int64()
        _check(lib().cles_server_submit(self.ptr, C.byref(desc), Q0.ctypes.data_as(C.c_void_p), lay, float(tfinal),
                                        int(nmax), C.byref(rid)))
        self._layout[rid.value] = Q0.shape
        return rid.value

    def tick(self):
        r, q = C.c_int(), C.c_int()
        _check(lib().cles_server_tick(self.ptr, C.byref(r), C.byref(q)))
        return r.value, q.value

    def status(self, rid):
        st = abi.cles_request_status()
        _check(lib().cles_server_status(self.ptr, int(rid), C.byref(st)))
        return {"state": abi.REQ_STATES[st.state], "failure": abi.FAIL_NAMES.get(st.failure), "steps": st.steps,
                "t": st.t, "submit_s": st.submit_s, "admit_s": st.admit_s, "done_s": st.done_s,
                "device_bytes": st.device_bytes}

    def fetch(self, rid):
        out = np.zeros(self._layout[rid])
        _check(lib().cles_server_fetch(self.ptr, int(rid), out.ctypes.data_as(C.c_void_p)))
        del self._layout[rid]
        return out

    def cancel(self, rid):
        _check(lib().cles_server_cancel(self.ptr, int(rid)))

    def drain(self, max_ticks=10 ** 8):
        """Tick until nothing is running or queued."""
        for _ in range(max_ticks):
            r, q = self.tick()
            if r == 0 and q == 0:
                return
        raise ClesError(abi.CLES_ETIMEOUT, "server did not drain")


class Batch:
    """Many solves of one physics class advanced together (cles_batch_*): one
    arena, one captured CUDA graph per composition, O(stages) launches per step
    whatever the number of members.  `cls` is a solver descriptor of the class
    (grid extents, domain and boundary states are per member)."""

    STRATEGIES = {"auto": 0, "batched": 1, "per_member": 2}

    def __init__(self, cls, ctx=None, strategy="auto"):
        self.ctx = ctx or default_context()
        self.ptr = C.c_void_p()
        _check(lib().cles_batch_create(self.ctx.ptr, C.byref(cls), C.byref(self.ptr)))
        self._shape = {}
        if strategy != "auto":
            self.set_strategy(strategy)

    def set_strategy(self, strategy):
        """How line solves launch: "batched", "per_member" or "auto" (the autotuner picks per operator)."""
        _check(lib().cles_batch_set_strategy(self.ptr, self.STRATEGIES[strategy]))

    def __del__(self):
        try:
            if self.ptr:
                lib().cles_batch_destroy(self.ptr)
                self.ptr = None
        except Exception:
            pass

    def add(self, desc, Q0, tfinal, nmax=2 ** 62, layout="padded"):
        Q0 = np.ascontiguousarray(Q0, dtype=np.float64)
        lay = abi.CLES_LAYOUT_PADDED if layout == "padded" else abi.CLES_LAYOUT_INTERIOR
        mid = C.c_int64()
        _check(lib().cles_batch_add(self.ptr, C.byref(desc), Q0.ctypes.data_as(C.c_void_p), lay, float(tfinal),
                                    int(nmax), C.byref(mid)))
        self._shape[mid.value] = Q0.shape
        return mid.value

    def step(self):
        n = C.c_int()
        _check(lib().cles_batch_step(self.ptr, C.byref(n)))
        return n.value

    def run(self, max_steps=2 ** 62):
        n = C.c_int()
        _check(lib().cles_batch_run(self.ptr, int(max_steps), C.byref(n)))
        return n.value

    def status(self, mid):
        st = abi.cles_request_status()
        _check(lib().cles_batch_status(self.ptr, int(mid), C.byref(st)))
        return {"state": abi.REQ_STATES[st.state], "failure": abi.FAIL_NAMES.get(st.failure), "steps": st.steps,
                "t": st.t, "admit_s": st.admit_s, "done_s": st.done_s, "device_bytes": st.device_bytes}

    def fetch(self, mid):
        out = np.zeros(self._shape[mid])
        _check(lib().cles_batch_fetch(self.ptr, int(mid), out.ctypes.data_as(C.c_void_p)))
        return out

    def cancel(self, mid):
        _check(lib().cles_batch_cancel(self.ptr, int(mid)))

    def stats(self):
        st = abi.cles_batch_stats()
        _check(lib().cles_batch_stats_get(self.ptr, C.byref(st)))
        ops = ("deriv", "filter", "filter_state")
        return {"members": st.members, "active": st.active, "compositions": st.compositions, "steps": st.steps,
                "launches_per_step": st.launches_per_step, "cells_total": st.cells_total,
                "tuning": [{"op": ops[t.op], "dim": t.dim, "threads": t.threads, "smem": t.smem, "ctas": t.ctas,
                            "tuned_ms": t.tuned_ms} for t in st.tuning[:st.n_roles]]}
