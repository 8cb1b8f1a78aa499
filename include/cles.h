/*
 * cles.h — C ABI of the B200 implementation of CompactLES.jl's RHS-and-step
 * hot path (compact derivatives/filters as batched line solves, Cook
 * artificial properties, flux/RHS assembly, LSRK(5,4) with the CFL rate
 * reduction).
 *
 * Every entry point is `extern "C"`, takes plain pointers and sizes, returns an
 * int status (CLES_OK on success) and never lets an exception cross the ABI.
 * The text of the last failure on the calling thread is cles_last_error().
 *
 * Citations name the reference function each entry point replaces, as
 * path:line inside the CompactLES.jl source tree.
 *
 * Layouts.  A "padded" field is the reference's own storage
 * (src/decomposition.jl:129-134): Float64, x fastest, extent n_local[d] +
 * 2*n_halo on every active dimension and 1 on a collapsed one; a conserved
 * state appends the component index as the slowest dimension.  An
 * "interior" field drops the halos (extent n_local[d]).  On one rank halos
 * are never read by this library: periodic lines wrap by index, closed lines
 * use closure rows, exactly the values the reference would read from current
 * halos.  The split-line entry points (cles_split_*) read the halo planes
 * beyond a rank interface, which cles_split_halo_unpack fills.
 *
 * Ownership.  The library allocates and frees its own device memory (plans,
 * solver state, scratch).  Caller buffers (host or device) are never freed or
 * retained past the call.  Calls on one solver/plan must be serialised by the
 * caller (the reference's operators are likewise called from serial sections
 * only, src/tridiag.jl:133-135); work is ordered on the stream given at
 * creation.
 */
#ifndef CLES_H
#define CLES_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ----------------------------------------------------- */
#define CLES_OK        0
#define CLES_EINVAL    1   /* bad descriptor; same checks as plan_direction (src/operators.jl:50-53) */
#define CLES_ENOMEM    2   /* device allocation failed or HBM budget exceeded */
#define CLES_ENUMERIC  3   /* non-finite / non-positive density seen by a kernel */
#define CLES_ETIMEOUT  4   /* a bounded device wait expired */
#define CLES_ECUDA     5   /* a CUDA runtime call failed */
#define CLES_EFAILURE  6   /* run! raised SolverFailure (src/stepcontrol.jl:145-152) */
#define CLES_EXCHANGE  7   /* a decomposed solver's exchange callback failed */

/* ---- fixed maxima of the descriptors ----------------------------------- */
#define CLES_MAX_Q        2   /* LHS half-bandwidth (1 tridiagonal, 2 pentadiagonal) */
#define CLES_MAX_M        4   /* interior RHS half-width (<= n_halo of the reference) */
#define CLES_MAX_NC       4   /* closure rows per edge */
#define CLES_MAX_CLO_LEN  8   /* closure RHS stencil length */
#define CLES_MAX_SPECIES  8
#define CLES_MAX_BODY_FORCES 4   /* ConstantBodyForce sources per solver */

/* element types */
#define CLES_F64  0
#define CLES_F32  1

/* field layouts */
#define CLES_LAYOUT_PADDED    0
#define CLES_LAYOUT_INTERIOR  1

/* boundary conditions (src/boundary.jl) */
#define CLES_BC_PERIODIC   0   /* PeriodicBC */
#define CLES_BC_SLIPWALL   1   /* SlipWallBC, enforce! at src/boundary.jl:232-243 */
#define CLES_BC_DIRICHLET  2   /* DirichletBC: bc_state, or a function of (x, t) via cles_solver_set_face_fn (src/problem.jl:174-207) */
#define CLES_BC_NOSLIP_WALL     3   /* NoSlipWallBC(Twall), enforce! at src/boundary.jl:245-265 */
#define CLES_BC_EXTRAPOLATION   4   /* ExtrapolationBC, enforce! at src/boundary.jl:267-278 */
#define CLES_BC_NSCBC_OUTFLOW   5   /* NSCBCOutflowBC, correct_rhs! at src/nscbc.jl:59-157 */
#define CLES_BC_NSCBC_INFLOW    6   /* NSCBCInflowBC (constant targets), correct_rhs! at src/nscbc.jl:220-307 */
/* Coordinate-singularity folds (src/boundary.jl:53-82, src/folds.jl): no state
 * enforcement; a half-offset grid, mirror rows and the antipodal pairing. */
#define CLES_BC_AXIS            7   /* AxisBC: low r face of a CylindricalMetric grid */
#define CLES_BC_ORIGIN          8   /* OriginBC: low r face of a SphericalMetric grid */
#define CLES_BC_POLE            9   /* PoleBC: both theta faces of a SphericalMetric grid */

/* Orthogonal metrics (src/metric.jl:20-45) */
#define CLES_METRIC_CARTESIAN    0   /* (x, y, z) */
#define CLES_METRIC_CYLINDRICAL  1   /* (r, theta, z), scale factors (1, r, 1) */
#define CLES_METRIC_SPHERICAL    2   /* (r, theta, phi), theta polar, scale factors (1, r, r sin theta) */

/* Parameters of one face condition (unused fields are ignored). */
typedef struct cles_bc_params {
    double Twall;                       /* NoSlipWallBC: NaN = adiabatic, finite = isothermal */
    double pinf, sigma, Lref, beta_t;   /* NSCBCOutflowBC (sigma 0.25, Lref <= 0 -> domain length, beta_t < 0 -> local Mach) */
    double u[3], T_ion;                 /* NSCBCInflowBC targets */
    double Y[CLES_MAX_SPECIES];         /* NSCBCInflowBC target composition (n_species entries) */
    double eta_u, eta_T, eta_t, eta_Y;  /* NSCBCInflowBC relaxation (0.28 each); Lref above */
} cles_bc_params;

/* beta sensors (src/artificial.jl:50-57) */
#define CLES_BETA_STRAIN        0
#define CLES_BETA_GATED_STRAIN  1
#define CLES_BETA_DILATATION    2

/* precision modes */
#define CLES_PREC_FP64   0   /* plain drop-in: everything FP64 */
#define CLES_PREC_MIXED  1   /* FP32 fields and line solves, FP64 RK state and reductions */

/* SolverFailure reasons (src/stepcontrol.jl:145-204) */
#define CLES_FAIL_NONE              0
#define CLES_FAIL_NONFINITE         1
#define CLES_FAIL_NEGATIVE_DENSITY  2
#define CLES_FAIL_PLANCK            3
#define CLES_FAIL_DT_MIN            4
#define CLES_FAIL_DT_COLLAPSE       5

/* ---- scheme descriptor ------------------------------------------------
 * One struct covers both CompactScheme (src/kernels.jl:28-50, q = 1) and
 * BandedCompactScheme (src/kernels_banded.jl:19-39, q >= 1):
 *   sum_s lhs[s-1] (g_{i-s} + g_{i+s}) + g_i = a0 f_i + sum_m coeffs[m-1] (f_{i+m} ± f_{i-m})
 * with '+' and a0 for symmetric (filter) schemes, '-' for derivatives.
 * Closure row j (0-based from the low edge) carries its full centred LHS band
 * clo_lhs[j][0..2q] (diagonal at index q) and an RHS stencil on f[0..clo_len-1]
 * counted inward from the edge; high-edge rows are mirrored by the planner
 * exactly as plan_direction does (src/operators.jl:77-83,
 * src/operators_banded.jl:91-98). */
typedef struct cles_scheme {
    char   name[48];
    int    q;
    double lhs[CLES_MAX_Q];
    double a0;
    int    M;
    double coeffs[CLES_MAX_M];
    int    symmetric;
    int    nc;
    double clo_lhs[CLES_MAX_NC][2 * CLES_MAX_Q + 1];
    int    clo_len[CLES_MAX_NC];
    double clo_rhs[CLES_MAX_NC][CLES_MAX_CLO_LEN];
} cles_scheme;

/* Scheme presets; replace lele_d1_6 / pade_d1_4 / compact_filter
 * (src/kernels.jl:61-111) and lele_d1_10 (src/kernels_banded.jl:54-64). */
int cles_scheme_lele_d1_6(cles_scheme* out);
int cles_scheme_pade_d1_4(cles_scheme* out);
int cles_scheme_compact_filter(double alphaf, cles_scheme* out);
int cles_scheme_lele_d1_10(cles_scheme* out);

/* ---- grid (the single-rank Decomp, src/decomposition.jl:80-122) -------- */
typedef struct cles_grid {
    int n_global[3];
    int periodic[3];   /* per dimension; a collapsed dimension (n == 1) is inactive */
    int n_halo;        /* halo width of padded fields on active dimensions (reference default 4) */
} cles_grid;

/* ---- library context ---------------------------------------------------- */
typedef struct cles_ctx    cles_ctx;
typedef struct cles_plan   cles_plan;
typedef struct cles_solver cles_solver;

/* Device selection and the stream every call of this context is ordered on
 * (NULL = the legacy default stream).  hbm_budget_bytes = 0 means no budget. */
int  cles_ctx_create(int device, void* stream, size_t hbm_budget_bytes, cles_ctx** out);
void cles_ctx_destroy(cles_ctx* ctx);
int  cles_ctx_set_stream(cles_ctx* ctx, void* stream);
/* Text of the last failure on this thread ("" if none). */
const char* cles_last_error(void);
/* Number of kernels this library has launched so far in this process. */
int64_t cles_kernel_launches(void);

/* Self-test of the bounded device wait (no counterpart in the reference).
 * Every mbarrier wait in the compact-operator kernels gives up after 2 s,
 * records the expiry in a device counter and returns; the next call that
 * reads the counter (cles_max_rate, and so every run! step) returns
 * CLES_ETIMEOUT and clears it.  This call runs that expiry path on purpose:
 * one CTA waits limit_ns (1e3 .. 2e9) on an mbarrier that nothing completes
 * (no copy is issued, so nothing is in flight when it gives up), then the
 * counter is read on the context's stream.  Returns CLES_ETIMEOUT when the
 * path works; the context stays usable. */
int  cles_selftest_bounded_wait(cles_ctx* ctx, int64_t limit_ns);

/* ---- directional plans ---------------------------------------------------
 * cles_plan_create replaces plan_direction(decomp, scheme, dim, h)
 * (src/operators.jl:44-101, src/operators_banded.jl:29-125): LHS assembly
 * with closures, coupling blocks, 1/h prescale, factorisation.  dim is
 * 1-based like the reference.  dtype CLES_F64 / CLES_F32, layout
 * CLES_LAYOUT_PADDED / CLES_LAYOUT_INTERIOR.  Returns CLES_EINVAL for the
 * reference's plan-time errors (extent below max(2nc+1, 2M+1, 2q+1), M > n_halo). */
int  cles_plan_create(cles_ctx* ctx, const cles_grid* grid, const cles_scheme* scheme,
                      int dim, double h, int dtype, int layout, cles_plan** out);
void cles_plan_destroy(cles_plan* plan);

/* cles_apply_along replaces apply_along!(out, plan, f, decomp)
 * (src/operators.jl:199-215): fill -> batched line solve (+ reduced interface
 * solve for periodic lines) -> scatter into the interior of out.  f and out
 * are DEVICE pointers in the plan's layout/dtype; out may equal f. */
int  cles_apply_along(cles_plan* plan, const void* f_dev, void* out_dev);
/* Same, over `count` fields spaced `field_stride` elements apart (one launch). */
int  cles_apply_along_batch(cles_plan* plan, const void* f_dev, void* out_dev,
                            int count, int64_t field_stride);
/* Same as cles_apply_along with HOST buffers (copies in and out through
 * plan-owned device memory).  Float64 padded or interior per the plan. */
int  cles_apply_along_host(cles_plan* plan, const void* f_host, void* out_host);

/* ---- lines split across ranks -------------------------------------------
 * The reference's decomposed operator: plan_direction on a Decomp with P > 1
 * ranks along `dim` (src/operators.jl:44-101, src/tridiag.jl:85-123,
 * src/banded.jl:108-169) and apply_along! over it (src/operators.jl:199-215,
 * src/tridiag.jl:136-170, src/banded.jl:177-214), one process per GPU.  The
 * library does the arithmetic; the caller moves the data between ranks at
 * the two points the reference calls MPI: the halo Sendrecv!
 * (src/halo.jl:143-194) and the Allgather! of the interface values
 * (src/tridiag.jl:148).  One application on rank r:
 *   cles_split_halo_pack(f -> send_lo, send_hi)
 *   send send_hi to rank `next` and send_lo to rank `prev`; receive recv_lo
 *     from `prev` (its send_hi) and recv_hi from `next` (its send_lo)
 *   cles_split_halo_unpack(recv_lo, recv_hi -> halo of f)
 *   cles_split_apply_begin(f -> out, iface)
 *   all-gather iface from every rank along dim, in rank order -> iface_all
 *   cles_split_apply_end(iface_all -> out)
 * Plan creation needs no exchange: every rank rebuilds every rank's local
 * factorisation (the reference all-gathers the spike end values instead).
 * Fields are padded (n_halo >= the scheme's M on every active dimension);
 * only the halo planes beyond this rank's open ends are read.  Folds are not
 * supported on a split dimension. */
typedef struct cles_split_plan cles_split_plan;
typedef struct cles_split_desc {
    int n_local[3];   /* this rank's interior extents (Decomp n_local) */
    int n_halo;       /* halo width of the padded fields */
    int dim;          /* split dimension, 1-based */
    int n_global;     /* global extent along dim */
    int ranks;        /* ranks along dim */
    int rank;         /* this rank's coordinate along dim, 0-based */
    int periodic;     /* the global line wraps */
} cles_split_desc;
typedef struct cles_split_info {
    int64_t halo_elems;   /* elements per field of each of send_lo/send_hi/recv_lo/recv_hi: M x lines */
    int64_t iface_elems;  /* elements per field of iface: 2q x lines (iface_all holds ranks x count x this) */
    int64_t field_elems;  /* elements of one padded field */
    int prev, next;       /* neighbouring rank coordinates along dim, -1 for none */
    int ranks, q, M;
} cles_split_info;
int  cles_split_plan_create(cles_ctx* ctx, const cles_split_desc* desc, const cles_scheme* scheme, double h,
                            int dtype, cles_split_plan** out);
void cles_split_plan_destroy(cles_split_plan* plan);
int  cles_split_plan_info(const cles_split_plan* plan, cles_split_info* out);
/* Buffers are DEVICE pointers; `count` fields spaced field_stride elements
 * apart (the padded field size for count = 1); halo and iface buffers hold
 * `count` consecutive blocks of the per-field sizes in cles_split_info.
 * Buffers of an end without a neighbour are neither read nor written (pass
 * NULL). */
int  cles_split_halo_pack(cles_split_plan* plan, const void* f_dev, void* send_lo, void* send_hi, int count,
                          int64_t field_stride);
int  cles_split_halo_unpack(cles_split_plan* plan, const void* recv_lo, const void* recv_hi, void* f_dev, int count,
                            int64_t field_stride);
/* Local solve: out = this rank's rows of the line solved with its own
 * factorisation (the halo of f beyond an open end must be current), iface =
 * each line's first and last q values of that solution.  out may equal f. */
int  cles_split_apply_begin(cles_split_plan* plan, const void* f_dev, void* out_dev, void* iface, int count,
                            int64_t field_stride);
/* Correction from every rank's iface (iface_all, rank-major): out becomes the
 * interior of apply_along!(out, plan, f, decomp). */
int  cles_split_apply_end(cles_split_plan* plan, const void* iface_all, void* out_dev, int count,
                          int64_t field_stride);

/* ---- solver -------------------------------------------------------------- */

/* StepControl (src/stepcontrol.jl:116-136). */
typedef struct cles_step_control {
    double predict;
    double max_growth;
    int    landing_steps;
    double dt_min;
    double dt_min_ratio;
    int    retries;
    double cfl_backoff;
    int    savepoint_interval;
} cles_step_control;
void cles_step_control_default(cles_step_control* out);

/* The Solver's scalar configuration (src/rhs.jl:122-135, src/problem.jl:243-306).
 * Orthogonal metric, optional stretching and coordinate folds; no sources. */
/* Equation of state of the mixture. */
#define CLES_EOS_IDEAL 0   /* IdealMixture: R[k], gamma[k] (src/physics.jl:87-120) */
#define CLES_EOS_NASA9 1   /* Nasa9Mixture: R[k] and the NASA-9 intervals (src/physics.jl:402-427) */
#define CLES_MAX_NASA9_INTERVALS 4

/* One NASA-9 interval (Nasa9Interval, src/physics.jl:291-296):
 *   cp/R = a1 T^-2 + a2 T^-1 + a3 + a4 T + a5 T^2 + a6 T^3 + a7 T^4
 *   h/R  = -a1 T^-1 + a2 ln T + a3 T + a4 T^2/2 + a5 T^3/3 + a6 T^4/4 + a7 T^5/5 + b1 */
typedef struct cles_nasa9_interval {
    double Tmin, Tmax;
    double a[7];
    double b1;
} cles_nasa9_interval;

typedef struct cles_solver_desc {
    int    n_global[3];
    double L[3];                 /* domain extents */
    double origin[3];            /* low corner */
    int    bc[3][2];             /* CLES_BC_* per (dim, side) */
    /* conserved state imposed on a CLES_BC_DIRICHLET face without a face function */
    double bc_state[3][2][CLES_MAX_SPECIES + 4];
    cles_bc_params bc_params[3][2];
    /* SwitchableBC(before, after) (src/boundary.jl:120-177): a face with
     * bc_switchable set behaves as bc/bc_params/bc_state until
     * cles_solver_switch_bc, then as bc_after/bc_after_params/bc_after_state.
     * Both conditions must agree on periodicity. */
    int    bc_switchable[3][2];
    int    bc_after[3][2];
    cles_bc_params bc_after_params[3][2];
    double bc_after_state[3][2][CLES_MAX_SPECIES + 4];
    int    n_species;            /* IdealMixture species count */
    double R[CLES_MAX_SPECIES];  /* specific gas constants */
    double gamma[CLES_MAX_SPECIES];
    double mu0, Pr, Sc;          /* Transport (src/physics.jl:589-593) */
    int    art_enabled;          /* ArtParams (src/artificial.jl:50-57) */
    double C_mu, C_beta, C_kappa, C_D;
    int    beta_sensor;
    cles_scheme deriv;
    cles_scheme filt;
    double cfl;
    int    filter_interval;
    cles_step_control control;
    int    n_halo;               /* halo width of padded host arrays (layout only) */
    int    precision;            /* CLES_PREC_FP64 / CLES_PREC_MIXED */
    /* CLES_EOS_NASA9: temperature from internal energy by the bounded FP64
     * Newton of mixture_temperature (src/physics.jl:466-498) in every
     * precision mode; gamma[] is unused. */
    int    eos;                  /* CLES_EOS_IDEAL (default) or CLES_EOS_NASA9 */
    double T_guess;              /* Newton seed reference temperature (default 300 K) */
    int    n_intervals[CLES_MAX_SPECIES];
    cles_nasa9_interval nasa9[CLES_MAX_SPECIES][CLES_MAX_NASA9_INTERVALS];
    /* Geometry (src/rhs.jl:122-311, src/metric.jl).  metric = CLES_METRIC_*.
     * A Stretch (src/metric.jl:47-68) on dimension d is given by its mapping
     * sampled at the n_global[d] nodes xi_i = i / (n_global[d] - 1), i = 0..n-1:
     * stretch_x[d][i] = x(xi_i) and stretch_dxdxi[d][i] = dx/dxi(xi_i) (host
     * arrays, read at create time only; NULL = uniform).  A stretched dimension
     * must be non-periodic and not folded; its origin is ignored.  Fold faces
     * (CLES_BC_AXIS / _ORIGIN / _POLE) select the half-offset grids and the
     * parity plans of the reference; their validation is the reference's
     * (src/rhs.jl:143-189). */
    int    metric;
    const double* stretch_x[3];
    const double* stretch_dxdxi[3];
    /* Problem.sources (src/sources.jl): n_body_forces ConstantBodyForce
     * accelerations, applied in order after the boundary corrections. */
    int    n_body_forces;
    double body_force[CLES_MAX_BODY_FORCES][3];
} cles_solver_desc;

/* Defaults of Problem()/Numerics() for a grid: single_species(1.4, R=1),
 * Transport(), ArtParams(), lele_d1_6, compact_filter(0.45), cfl 0.5,
 * filter_interval 1, periodic everywhere, domain [0, L). */
void cles_solver_desc_default(cles_solver_desc* out);

typedef struct cles_solver_info {
    int     n_local[3];
    int     active[3];
    double  h[3];
    int     n_cons;
    int     n_species;
    int64_t cells;
    int64_t padded_cells;
    size_t  device_bytes;
} cles_solver_info;

/* Replaces Solver(...) + plan_direction per active dim (src/rhs.jl:122-311). */
int  cles_solver_create(cles_ctx* ctx, const cles_solver_desc* desc, cles_solver** out);
void cles_solver_destroy(cles_solver* s);
int  cles_solver_info_get(const cles_solver* s, cles_solver_info* out);

/* ---- one rank of a decomposed grid (Decomp, src/decomposition.jl:80-140) --
 * The process grid splits each active dimension d into dims[d] pieces by
 * local_range (src/decomposition.jl:73-78); this rank owns the block at
 * `coords`.  `rank` is its number in the communicator (checkpoint file
 * names, src/io.jl:8).  Collapsed dimensions are not split. */
typedef struct cles_decomp {
    int dims[3];
    int coords[3];
    int rank;
} cles_decomp;

enum { CLES_REDUCE_MAX = 0, CLES_REDUCE_SUM = 1 };

/* The three points where the reference calls MPI, as host callbacks (one
 * process per GPU: NCCL through torch.distributed, or MPI.jl from Julia).
 * Each returns 0 on success; a non-zero return fails the solver call with
 * CLES_EXCHANGE.  Every rank makes the same calls in the same order.
 *
 * halo: Sendrecv! with both neighbours along dimension `dim` (0-based,
 *   src/halo.jl:143-194): recv_lo <- the previous rank's send_hi, recv_hi <-
 *   the next rank's send_lo.  prev / next are the neighbours' coordinates
 *   along dim (-1 at a closed end; equal to this rank's coordinate when it is
 *   its own periodic neighbour).  `bytes` per buffer.
 * gather: Allgather! over the ranks along dim in coordinate order
 *   (src/tridiag.jl:148, src/banded.jl:190): `all` receives dims[dim] blocks
 *   of `bytes`, block r from the rank at coordinate r.
 * allreduce: Allreduce! over every rank of `count` host doubles in place
 *   (CLES_REDUCE_MAX: max_rate, src/timestep.jl:173; CLES_REDUCE_SUM: the
 *   volume integrals of the diagnostics).
 *
 * Buffers of halo and gather are device memory.  On entry the sends are
 * complete in the order of `stream` (the solver's stream); on return the
 * receives must be complete in that order (NCCL on `stream`, or a stream
 * synchronisation around host-driven copies). */
typedef struct cles_exchange {
    void* user;
    int (*halo)(void* user, int dim, int prev, int next, const void* send_lo, const void* send_hi, void* recv_lo,
                void* recv_hi, int64_t bytes, void* stream);
    int (*gather)(void* user, int dim, const void* local, void* all, int64_t bytes, void* stream);
    int (*allreduce)(void* user, int op, double* vals, int count);
} cles_exchange;

/* Replaces Solver(...) on a Decomp with several ranks: `desc` describes the
 * GLOBAL problem (n_global, L, faces); the solver holds this rank's block.
 * Compact applications along a split dimension run the P > 1 line solve
 * (local solve with open ends, interface gather, reduced solve, correction:
 * src/tridiag.jl:136-170, src/banded.jl:177-214), delta4_sum! reads the
 * exchanged planes beyond each rank interface, boundary conditions act only
 * on the faces this rank owns (at_lo_edge / at_hi_edge), and max_rate
 * reduces (rate, -rho_min) with max over every rank.  States, fields and
 * checkpoints are this rank's block (n_local of cles_solver_info).
 * Supported: uniform Cartesian grids (no metric, stretching or folds), no
 * characteristic (NSCBC) faces on a split dimension; host-stepped run!
 * (cles_run_graph refuses a decomposed solver).  `ex` is copied. */
int  cles_solver_create_decomposed(cles_ctx* ctx, const cles_solver_desc* desc, const cles_decomp* decomp,
                                   const cles_exchange* ex, cles_solver** out);

/* An in-process exchange among the prod(dims) ranks of one process, one host
 * thread per rank (several GPUs driven from one process, or several ranks on
 * one GPU for a decomposition test).  Each call records a "sends ready" event
 * on the caller's stream, meets the other ranks at a host barrier, makes its
 * stream wait on its peers' ready events and copies from their buffers with
 * cudaMemcpyAsync, records a "copied" event, meets them again and makes its
 * stream wait on the copied events of the ranks that read its buffers.  The
 * host does not wait for the device, and no kernel waits on another rank
 * (stream-event dependencies only).  A barrier that is not met within
 * `timeout_s` seconds (or after cles_local_group_abort) fails the call. */
typedef struct cles_local_group cles_local_group;
int  cles_local_group_create(const int dims[3], double timeout_s, cles_local_group** out);
void cles_local_group_destroy(cles_local_group* g);
/* The exchange of the rank at `coords` (valid while the group lives). */
int  cles_local_group_exchange(cles_local_group* g, const int coords[3], cles_exchange* out);
/* Fail every pending and future barrier of the group (a rank that stopped). */
void cles_local_group_abort(cles_local_group* g);

/* Conserved state in and out (host arrays, layout CLES_LAYOUT_PADDED or
 * _INTERIOR, Float64, component slowest).  Output writes the interior only. */
int  cles_set_state(cles_solver* s, const double* Q_host, int layout);
int  cles_get_state(cles_solver* s, double* Q_host, int layout);
/* Device pointer of the resident conserved state (interior layout, Float64,
 * component stride = cells). */
int  cles_state_device(cles_solver* s, double** Q_dev);

/* Replaces apply_bcs!(solver, Q) (src/boundary.jl:280-286). */
int  cles_apply_bcs(cles_solver* s);
/* Replaces max_rate(solver, Q) (src/timestep.jl:125-175): refreshes the
 * primitives from the resident state and returns (rate, min density). */
int  cles_max_rate(cles_solver* s, double* rate, double* rho_min);
/* Replaces compute_rhs!(solver, Q, dQ, primitives_current) (src/rhs.jl:624-694);
 * dQ stays on the device (read it with cles_get_rhs). */
int  cles_compute_rhs(cles_solver* s, int primitives_current);
int  cles_get_rhs(cles_solver* s, double* dQ_host, int layout);
/* Replaces step!(solver, Q, dQ, du, dt, prepared) (src/timestep.jl:72-99). */
int  cles_step(cles_solver* s, double dt, int prepared);
/* Replaces filter_state!(solver, Q) (src/timestep.jl:414-426). */
int  cles_filter_state(cles_solver* s);

/* Named solver fields for diagnostics and parity checks (interior, Float64). */
#define CLES_FIELD_RHO        0
#define CLES_FIELD_U          1
#define CLES_FIELD_V          2
#define CLES_FIELD_W          3
#define CLES_FIELD_P          4
#define CLES_FIELD_T          5
#define CLES_FIELD_C          6
#define CLES_FIELD_CP         7
#define CLES_FIELD_MU_ART     8
#define CLES_FIELD_BETA_ART   9
#define CLES_FIELD_KAPPA_ART 10
#define CLES_FIELD_SENSOR    11
#define CLES_FIELD_Y0        16   /* + species index */
#define CLES_FIELD_D_ART0    32   /* + species index */
#define CLES_FIELD_GRAD_U0   48   /* + 3*(d-1) + (j-1): d/dx_d of u_j */
int  cles_get_field(cles_solver* s, int which, double* host, int layout);

/* Clock of the solver (solver.t, solver.step, solver.cfl). */
int  cles_get_clock(const cles_solver* s, double* t, int64_t* step, double* cfl);
int  cles_set_clock(cles_solver* s, double t, int64_t step, double cfl);

/* Checkpoint / restart in the reference's raw binary format.
 * cles_checkpoint_save replaces save_checkpoint(solver, Q, prefix)
 * (src/io.jl:8-41): it writes `prefix.r0000.ckpt` (one rank: n_local =
 * n_global, coords = 0), little-endian: UInt64 magic 0x434c4553434b5054,
 * Int64 n_cons, Int64 n_global[3], Int64 n_local[3], Int64 coords[3],
 * Float64 t, Int64 step, then the interior of Q as Float64 in Julia order
 * (x fastest, conserved component slowest), straight from the device state.
 * cles_checkpoint_load replaces load_checkpoint!(solver, Q, prefix)
 * (src/io.jl:43-72): it checks the magic, the conserved layout, the global
 * grid, the decomposition and the rank layout (CLES_EINVAL with the
 * reference's message on a mismatch) and restores the state, t and step. */
/* switch!(bc::SwitchableBC) (src/boundary.jl:150-160) on face (dim 0..2, side
 * 0 low / 1 high): from now on the face acts as its `after` condition
 * (idempotent; CLES_EINVAL if the face is not switchable). */
int  cles_solver_switch_bc(cles_solver* s, int dim, int side);

/* Face conditions given as functions of position and time: DirichletBC(fun)
 * (src/problem.jl:180-207) and NSCBCInflowBC(target = fun) (src/nscbc.jl:
 * 178-307).  The library calls fn on the host at the RK stage time at which
 * the reference evaluates them (each apply_bcs! for a Dirichlet face, each
 * correct_rhs! for an inflow face), for the npts nodes of face (dim 0..2,
 * side 0 low / 1 high) in plane order (the lower-numbered transverse
 * dimension fastest), with their physical coordinates x1, x2, x3.  fn fills
 *   a CLES_BC_DIRICHLET face:     out[c * npts + p] = conserved component c;
 *   a CLES_BC_NSCBC_INFLOW face:  out[a * npts + p], a = 0..2 target velocity,
 *                                 3 target temperature, 4 + k target Y_k.
 * which = 0 sets the face's condition, 1 the `after` condition of a
 * SwitchableBC; fn = NULL returns to the descriptor's constants.  A solver
 * with a face function does not run in graph mode (CLES_EINVAL). */
typedef void (*cles_face_fn)(void* user, int dim, int side, double t, int64_t npts, const double* x1,
                             const double* x2, const double* x3, double* out);
int  cles_solver_set_face_fn(cles_solver* s, int dim, int side, int which, cles_face_fn fn, void* user);
int  cles_solver_bc_switched(const cles_solver* s, int dim, int side, int* switched);

int  cles_checkpoint_save(cles_solver* s, const char* prefix);
int  cles_checkpoint_load(cles_solver* s, const char* prefix);

/* check_step(control, dt, rho_min, dt_seen, step, t, cfl)
 * (src/stepcontrol.jl:184-204); *reason = CLES_FAIL_* (CLES_FAIL_NONE = accepted). */
int  cles_check_step(const cles_step_control* control, double dt, double rho_min,
                     double dt_seen, int64_t step, double t, double cfl, int* reason);

typedef struct cles_run_result {
    int64_t steps;        /* steps completed by this call */
    double  t;            /* solver.t after the call */
    double  last_dt;
    double  cfl;          /* solver.cfl after any retries */
    int     failure;      /* CLES_FAIL_* that ended the run, or CLES_FAIL_NONE */
    int     retries_used;
} cles_run_result;

/* Replaces run!(solver, Q; tfinal, nmax, control) without callbacks
 * (src/timestep.jl:277-405): bcs -> max_rate -> dt/check_step (+ rollback and
 * CFL backoff) -> step!(prepared) -> filter_state! every filter_interval steps.
 * Returns CLES_EFAILURE when a SolverFailure is raised. */
int  cles_run(cles_solver* s, double tfinal, int64_t nmax, cles_run_result* out);

/* Host-buffer drop-in of one run! iteration, the unit the end-to-end
 * benchmark times: copy Q_host (padded or interior, pinned or pageable) to
 * the device, do one step of cles_run, copy the state back to Q_host. */
int  cles_step_host(cles_solver* s, double* Q_host, int layout, double tfinal,
                    cles_run_result* out);

/* Allocation-free CFL rate reduction (no counterpart in the reference).
 * For callers that cannot call cudaMalloc -- code inside a host framework
 * that owns every device allocation, a plugin barred from allocating after
 * start-up, or a process held to a fixed HBM budget.  For an ideal mixture on
 * a uniform Cartesian grid it computes what cles_max_rate computes for an
 * FP64 solver (the rate max of src/timestep.jl:125-175 and the minimum
 * mixture density; identical values) from caller-owned device arrays,
 * keeping its per-block partials in a library-owned static device array
 * instead of allocating.  It has no per-node 1/h (stretched or curvilinear
 * grids), no curvature_rate term and no NASA-9 thermodynamics, and it works
 * on FP64 primitives where a mixed-precision solver rounds them to FP32: for
 * those solvers call cles_max_rate.  Arguments:
 *   Q_dev      conserved state, interior layout, component slowest (n_species+4 fields of `cells`)
 *   art_dev    mu*, beta*, kappa*, D*_1..D*_Ns (3+n_species fields of `cells`)
 *   inv_h      1/h per dimension, 0 for a collapsed one
 *   result_dev two doubles written on the device: rate, rho_min
 * At most CLES_STATIC_MAX_CELLS cells per call (larger grids: CLES_EINVAL).
 * All calls on a device share the static array, so calls that overlap on the
 * GPU race; order them on one stream.  The first call on a device resolves the
 * array's address (cudaGetSymbolAddress) and should come before any stream
 * capture; after a cudaDeviceReset the next call resolves it again (the
 * cached address is keyed by the context's unique id), so that call is a
 * first call too.  Work is queued on `stream` (NULL = legacy default stream),
 * which must belong to the current device (CLES_EINVAL otherwise). */
#define CLES_STATIC_MAX_CELLS 33554432LL
int  cles_max_rate_static(const double* Q_dev, const double* art_dev, int64_t cells, int n_species,
                          const double* R, const double* gamma, const double* inv_h, double mu0, double Pr,
                          double Sc, double* result_dev, void* stream);

/* Measurement hook (no counterpart in the reference): while enabled, every
 * compact-operator launch is bracketed by CUDA events on its stream and its
 * algorithmic bytes (input read once, output written once, plus the output
 * read for accumulating stores) are recorded.  Enabling clears the records;
 * cles_profile_read synchronises and returns one entry per direction
 * ("compact_x", "compact_y", "compact_z"). */
typedef struct cles_profile_entry {
    char    name[32];
    int64_t launches;
    double  total_ms;
    double  bytes;
} cles_profile_entry;
int  cles_profile_enable(int on);
int  cles_profile_read(cles_profile_entry* out, int max_entries, int* n_entries);

/* run! in graph mode (no counterpart in the reference): every step is one
 * CUDA-graph launch with the timestep, the check_step floors and the clock on
 * the device, so no host round trip happens inside a step.  Same results as
 * cles_run for the same state (bitwise in FP64); rate prediction, growth
 * capping and rollback retries are not available in this mode (CLES_EINVAL). */
int  cles_run_graph(cles_solver* s, double tfinal, int64_t nmax, cles_run_result* out);

/* ---- serving: continuous batching of independent solves -----------------
 * No counterpart in the reference (one problem per process there).  A server
 * owns one device.  Requests (a solver descriptor, an initial state and an
 * end time) are queued; every cles_server_tick admits queued requests in
 * arrival order while the active count and the HBM budget allow, advances
 * every running request by one run! step (one graph launch each, on its own
 * stream, so the steps of different requests overlap on the device), and
 * retires finished or failed ones, freeing their memory for the queue.  Each
 * request's arithmetic is independent of the others, so its result is the
 * same alone and in any mix.  Requests with rollback retries are stepped on
 * the host instead of by graph. */
typedef struct cles_server cles_server;
#define CLES_REQ_QUEUED    0
#define CLES_REQ_RUNNING   1
#define CLES_REQ_DONE      2
#define CLES_REQ_FAILED    3
#define CLES_REQ_CANCELLED 4
typedef struct cles_request_status {
    int     state;          /* CLES_REQ_* */
    int     failure;        /* CLES_FAIL_* when failed */
    int64_t steps;
    double  t;
    double  submit_s;       /* seconds since server creation */
    double  admit_s;        /* -1 while queued */
    double  done_s;         /* -1 until finished */
    size_t  device_bytes;   /* admission estimate */
} cles_request_status;
int  cles_server_create(int device, size_t hbm_budget_bytes, int max_active, cles_server** out);
void cles_server_destroy(cles_server* s);
int  cles_server_submit(cles_server* s, const cles_solver_desc* desc, const double* Q0_host, int layout,
                        double tfinal, int64_t nmax, int64_t* id);
int  cles_server_tick(cles_server* s, int* n_running, int* n_queued);
int  cles_server_status(cles_server* s, int64_t id, cles_request_status* out);
/* Final state of a finished request (same layout as submitted); releases it. */
int  cles_server_fetch(cles_server* s, int64_t id, double* Q_host);
int  cles_server_cancel(cles_server* s, int64_t id);
/* Batching (off by default): while on, an admitted request that the batch
 * path supports (see cles_batch_create) joins a batch of its physics class
 * instead of getting its own solver; every tick advances each batch by one
 * captured step, whatever its member count.  max_members > 0 caps the
 * members of one batch: a class then spreads over several batches, each on
 * its own stream, stepped concurrently.  Batched results equal the same
 * request run alone through a batch, bitwise, and the one-grid solver's to
 * rounding (different line-solve kernels). */
int  cles_server_set_batching(cles_server* s, int on, int max_members);

/* ---- batches: many solves of one physics class advanced together --------
 * No counterpart in the reference (one problem per process there).  A batch
 * holds independent solves ("members") that share everything in the solver
 * descriptor except the grid extents (n_global, with the same dimensions
 * active), the domain (L, origin) and the boundary states: species, transport,
 * artificial-property parameters, schemes, cfl, filter_interval, step-control
 * floors, precision and the kind of every face.  Supported: ideal mixtures on
 * uniform Cartesian grids with periodic, slip-wall, no-slip-wall,
 * extrapolation and constant Dirichlet faces, stepped as run! in graph mode
 * (no rate prediction, growth cap or rollback).  cles_batch_create takes the
 * class from `cls` (its grid fields are ignored apart from which dimensions
 * are active); CLES_EINVAL names the first differing field of a member.
 *
 * Every member's fields live in one device arena, so one step of the whole
 * batch is a fixed number of kernel launches -- per-cell kernels over every
 * member's cells at once, line solves, stencils, boundary planes and
 * reductions from per-grid descriptor tables -- captured once as a CUDA
 * graph per batch composition.  Each member keeps its own dt, clock, end
 * time and SolverFailure checks.  The composition changes when members are
 * added, finish, fail or are cancelled; the next step then rebuilds the arena
 * and tables and re-captures the graph.  A project-written autotuner times
 * the thread count (lines per CTA, x-tile depth) of every batched line-solve
 * launch the first time a launch shape is built and keeps the fastest.  A
 * member's arithmetic does not depend on the other members, so its results
 * are the same alone and in any mix. */
typedef struct cles_batch cles_batch;
typedef struct cles_batch_tuning {
    int     op;          /* 0 derivative, 1 filter of derived fields, 2 filter_state! of Q */
    int     dim;         /* 1-based direction */
    int     threads;     /* chosen threads per CTA of the batched kernel; 0 = per-member kernels */
    int64_t smem;        /* dynamic shared memory per CTA */
    int     ctas;        /* CTAs per field (per-member kernels: the member count) */
    double  tuned_ms;    /* the winner's time per launch (one field) when it was tuned here, else 0 */
} cles_batch_tuning;
typedef struct cles_batch_stats {
    int     members;           /* added so far */
    int     active;            /* not yet finished, failed or cancelled */
    int     compositions;      /* arena rebuilds / graph captures */
    int64_t steps;             /* batch steps (graph launches) */
    int     launches_per_step; /* kernels in one captured step */
    int64_t cells_total;       /* arena cells of the current composition (with alignment padding) */
    int     n_roles;
    cles_batch_tuning tuning[9];
} cles_batch_stats;
int  cles_batch_create(cles_ctx* ctx, const cles_solver_desc* cls, cles_batch** out);
void cles_batch_destroy(cles_batch* b);
/* Adds a member with its initial state (host, padded or interior layout);
 * it joins the batch at the next step. */
int  cles_batch_add(cles_batch* b, const cles_solver_desc* desc, const double* Q0_host, int layout, double tfinal,
                    int64_t nmax, int64_t* id);
/* One run! step of every running member; *n_active = members still running. */
int  cles_batch_step(cles_batch* b, int* n_active);
/* Steps until no member is running or max_steps batch steps were taken. */
int  cles_batch_run(cles_batch* b, int64_t max_steps, int* n_active);
int  cles_batch_status(cles_batch* b, int64_t id, cles_request_status* out);
/* A member's current (or final) state, in the layout it was added with. */
int  cles_batch_fetch(cles_batch* b, int64_t id, double* Q_host);
int  cles_batch_cancel(cles_batch* b, int64_t id);
int  cles_batch_stats_get(const cles_batch* b, cles_batch_stats* out);
/* How the line solves of a batch step are launched.  CLES_BATCH_BATCHED: one
 * batched kernel per operator and direction over every member (a fixed
 * number of launches per step).  CLES_BATCH_PER_MEMBER: every member's
 * one-grid kernel (the tile, warp or generic kernel the solver would pick),
 * spread over eight streams inside the captured step; members whose last
 * divergence cannot apply the RK update get one batched RK pass.
 * CLES_BATCH_AUTO (default): the autotuner times both for every operator and
 * direction and keeps the faster.  Results of the two forms agree to
 * rounding; with a fixed form a member's results do not depend on the other
 * members.  Takes effect at the next step. */
#define CLES_BATCH_AUTO        0
#define CLES_BATCH_BATCHED     1
#define CLES_BATCH_PER_MEMBER  2
int  cles_batch_set_strategy(cles_batch* b, int strategy);

/* Volume-averaged kinetic energy ∫½ρ|u|²dV / V and dissipation rate
 * (src/diagnostics.jl:354-378, bench/tgv_energy.jl:175-184) of the resident
 * state. */
int  cles_kinetic_energy(cles_solver* s, double* ke);
int  cles_dissipation_rate(cles_solver* s, double* eps);

#ifdef __cplusplus
}
#endif
#endif /* CLES_H */
