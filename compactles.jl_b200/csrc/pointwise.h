// Pointwise kernels of the RHS and the integrator.
#pragma once

#include "cles_internal.h"

namespace cles {

// Slots of the primitive block (one interior field each, component stride = cells).
// T and the mass fractions are adjacent so their gradients are one batched launch.
enum { P_RHO = 0, P_U = 1, P_V = 2, P_W = 3, P_P = 4, P_C = 5, P_CP = 6, P_T = 7, P_Y0 = 8 };
// Slots of the artificial-property block.
enum { A_MU = 0, A_BETA = 1, A_KAPPA = 2, A_D0 = 3 };

struct PhysConst {
    double Rk[CLES_MAX_SPECIES];
    double cvk[CLES_MAX_SPECIES];
    double cpk[CLES_MAX_SPECIES];
    // Nasa9Mixture (eos == CLES_EOS_NASA9): piecewise cp/R polynomials, and the
    // species energy and cv at T_guess that seed the Newton solve
    int eos;
    double T_guess;
    double e_ref[CLES_MAX_SPECIES], cv_ref[CLES_MAX_SPECIES];
    int nint[CLES_MAX_SPECIES];
    double Tmax[CLES_MAX_SPECIES][CLES_MAX_NASA9_INTERVALS];
    double a[CLES_MAX_SPECIES][CLES_MAX_NASA9_INTERVALS][7];
    double b1[CLES_MAX_SPECIES][CLES_MAX_NASA9_INTERVALS];
};

// Host evaluation of the NASA-9 species functions (the same expressions as
// the device), used for the Newton seed constants and by validation.
double nasa9_cp_over_R(const cles_nasa9_interval& iv, double T);
double nasa9_h_over_R(const cles_nasa9_interval& iv, double T);
// Fill the NASA-9 part of a PhysConst from a descriptor; throws on a bad table
// (the checks of Nasa9Species, src/physics.jl:322-345).
void nasa9_setup(PhysConst& pc, const cles_solver_desc& d);
// e_k(T) of a NASA-9 descriptor on the host (species_energy)
double nasa9_species_energy(const cles_solver_desc& d, int k, double T);

struct Grid3 {
    int n[3];
    int active[3];
    int periodic[3];
};

struct Weights3 {
    double w[3];
};

// Neighbours of a decomposed grid for delta4_sum!: along a split dimension d
// the two planes beyond an open end (a rank interface) come from lo[d] /
// hi[d], laid out [field][plane][line] (plane 0 nearest the low end, line the
// other two indices with the lower dimension fastest).  Elements of the
// field's type.
struct Halo4 {
    const void* lo[3];
    const void* hi[3];
    int open_lo[3], open_hi[3];
};

// State of one enforced face condition: the Dirichlet state, or the wall
// energy of an isothermal no-slip wall, rho e = (sum_k Q_k ew_k) * Twall for an
// ideal mixture (ew_k = cv_k) or sum_k Q_k e_k(Twall) for NASA-9 (ew_k = e_k(Twall)).
struct BcState {
    double q[CLES_MAX_SPECIES + 4];
    double ew[CLES_MAX_SPECIES];
    double Twall;
    int iso;          // isothermal no-slip wall
    int ew_times_T;   // ideal-mixture form of the wall energy
};

// One characteristic (NSCBC) face, parameters resolved on the host.
struct NscbcParams {
    int kind;         // CLES_BC_NSCBC_OUTFLOW or CLES_BC_NSCBC_INFLOW
    int act[3];       // active dimensions
    double Lref;      // > 0
    double pinf, sigma, beta_t;
    double u[3], T, Y[CLES_MAX_SPECIES], eta_u, eta_T, eta_t, eta_Y;
};

// Orthogonal-metric geometry (src/metric.jl:109-150) as per-dimension node
// tables; the per-point factors J, A_d, 1/h_d, 1/r are recomputed where they
// are used instead of being streamed from HBM.
struct Geom {
    int metric;          // CLES_METRIC_*
    int n[3];
    const double* x[3];  // physical node coordinate per dimension (n[d] values)
    const double* m[3];  // mapping Jacobian dx/dxi per dimension (1 when unstretched)
    const double* sn;    // sin(theta) at the theta nodes (spherical)
    const double* cs;    // cos(theta) at the theta nodes (spherical)
    const double* cotr;  // cot(theta)/r per cell after the GCL correction, or null (analytic)
};

// On-rank antipodal pairing of a folded dimension (src/folds.jl:128-155):
// shift pdim by half its extent, reverse revdim (-1 = none); sd is the
// dimension whose lower half holds the canonical slots.
struct PairParams {
    int n[3];
    int pdim, revdim, sd;
};

// ConstantBodyForce sources (src/sources.jl:20-82), applied in order.
struct BodyForces {
    int n;
    double g[CLES_MAX_BODY_FORCES][3];
};

template <typename F>
struct Pointwise {
    // esens: also write the kappa*-sensor input (internal energy) into slot P_Y0 + Ns
    static void primitives(const double* Q, F* prim, int64_t cells, int Ns, const PhysConst& pc, cudaStream_t st,
                           int esens = 0);
    // delta4_sum! of one (f1 == nullptr) or two fields in one tiled pass
    static void delta4_tiled(const F* f0, const F* f1, F* o0, F* o1, const Grid3& g, const double w0[3],
                             const double w1[3], cudaStream_t st);
    // the same on a rank's block of a decomposed grid: g.periodic is 0 along
    // split dimensions, whose open ends read the exchanged planes of h
    static void delta4_halo(const F* f0, const F* f1, F* o0, F* o1, const Grid3& g, const double w0[3],
                            const double w1[3], const Halo4& h, cudaStream_t st);
    static void art_coef(const F* s_strain, const F* s_energy, const F* prim, const F* g, F* art, int64_t cells,
                         double C_mu, double C_beta, double C_kappa, int gate, cudaStream_t st);
    static void strain(const F* g, F* out, int64_t cells, cudaStream_t st);
    static void delta4(const F* f, F* out, const Grid3& g, const double wd[3], cudaStream_t st);
    static void mu_beta(const F* sensor, const F* prim, const F* g, F* art, int64_t cells, double C_mu, double C_beta,
                        int gate, cudaStream_t st);
    static void dilatation(const F* g, F* div, F* sw, int64_t cells, cudaStream_t st);
    static void beta_dilatation(const F* sensor, const F* prim, const F* sw, F* art, int64_t cells, double C_beta,
                                cudaStream_t st);
    static void energy(const double* Q, const F* prim, F* out, int64_t cells, int Ns, cudaStream_t st);
    static void kappa(const F* sensor, const F* prim, F* art, int64_t cells, double C_kappa, cudaStream_t st);
    static void dart(const F* sensor, const F* prim, F* art, int64_t cells, double C_D, int sp, cudaStream_t st);
    static void fluxes(const double* Q, const F* prim, const F* g, const F* gty, const F* art, F* flux, int64_t cells,
                       int Ns, const PhysConst& pc, double mu0, double Pr, double Sc, cudaStream_t st);
    static void lsrk(double* Q, double* du, const F* dQ, int64_t n, double A, double B, double dt, cudaStream_t st,
                     const double* dtp = nullptr);
    static void rate(const double* Q, const F* prim, const F* art, double* part, double* out, int64_t cells, int Ns,
                     const double idx[3], const int act[3], double mu0, double Pr, double Sc, cudaStream_t st);
    static void kinetic(const double* Q, double* part, double* out, int64_t cells, int Ns, cudaStream_t st);
    // G: geometry of a curvilinear / stretched grid (null = unit Jacobian);
    // foldmask bit 2d + side marks a folded edge (quadrature weight 1)
    static void dissipation(const F* prim, const F* g, const F* art, double* part, double* out, const Grid3& gr,
                            double mu0, cudaStream_t st, const Geom* G = nullptr, unsigned foldmask = 0u);
    static void convert(const double* a, F* b, int64_t n, cudaStream_t st);
    static void to_double(const F* a, double* b, int64_t n, cudaStream_t st);
    // correct_rhs! of an NSCBC face (src/nscbc.jl:59-307) on the plane of
    // (d, side): dpd = dp/dx_d, dpt0/dpt1 = dp along the two transverse dims
    // (outflow, unread when inactive), drd = drho/dx_d (inflow); gty holds
    // [dT, dY_k] per dimension (ngty fields each).
    static void nscbc(F* dQ, const F* prim, const F* g, const F* gty, int ngty, const F* dpd, const F* dpt0,
                      const F* dpt1, const F* drd, const Grid3& gr, int d, int side, int Ns, const PhysConst& pc,
                      const NscbcParams& bp, cudaStream_t st, const double* tgt = nullptr,
                      const Geom* G = nullptr);
    // add_sources! (src/sources.jl:42-82): dQ += rho g on the momenta and
    // Q_m . g on the energy, per body force in order
    static void body_forces(F* dQ, const double* Q, int64_t cells, int Ns, const BodyForces& bf, cudaStream_t st);
    // fluxes with each direction's flux multiplied by its area factor A_d
    // (the A_d F_d product of src/rhs.jl:670-675), for curvilinear / stretched grids
    static void fluxes_geo(const double* Q, const F* prim, const F* g, const F* gty, const F* art, F* flux,
                           int64_t cells, int Ns, const PhysConst& pc, double mu0, double Pr, double Sc,
                           const Geom& G, cudaStream_t st);
};

// Curvilinear / stretched-grid passes (geometry.cu).
template <typename F>
struct MetricOps {
    // velocity gradients: 1/h_d scaling of the coordinate derivatives (zero on
    // collapsed dims) plus the curvature terms (src/rhs.jl:596-604, src/metric.jl:177-221)
    static void metric_grad(F* g, const F* prim, const Geom& G, const Grid3& gr, cudaStream_t st);
    // 1/h_d scaling of `count` gradient fields per active dim ([d][count] layout)
    static void scale_grad(F* f, int count, const Geom& G, const Grid3& gr, cudaStream_t st);
    // dQ_c = -sum_d inv_J D_d(A_d F_dc) from the per-direction derivatives in
    // fd ([d][ncons] layout), then the momentum sources (src/rhs.jl:650-687)
    static void metric_div(F* dQ, const F* fd, int ncons, int Ns, const F* prim, const F* g, const F* art,
                           double mu0, const Geom& G, const Grid3& gr, cudaStream_t st);
    // max_rate with the inverse physical spacing 1/(h_d h) and the curvature rate
    static void rate_geo(const double* Q, const F* prim, const F* art, double* part, double* out, int Ns,
                         const double h[3], double mu0, double Pr, double Sc, const Geom& G, const Grid3& gr,
                         cudaStream_t st);
};

// Folded-dimension butterflies (src/folds.jl:162-262) on `count` interior
// fields of element type T spaced fs apart: w <- (e, o) combination of f;
// out (even result on the canonical half, odd result on the partner half)
// <- (Re + Ro, sig (Re - Ro)) in place.
template <typename T>
void pair_forward(const T* f, T* w, int count, int64_t fs, const PairParams& pp, int sig, cudaStream_t st);
template <typename T>
void pair_backward(T* out, int count, int64_t fs, const PairParams& pp, int sig, cudaStream_t st);

#ifdef __CUDACC__
// init_geometry! (src/metric.jl:109-140) at interior cell (i, j, k): the same
// products and quotients in the same order, with no contraction.
struct GeoPoint {
    double inv_J, A[3], inv_h[3], inv_r, cotr;
};
__device__ __forceinline__ double geo_max(double x, double y) {
    if (x != x) return x;
    return y > x ? y : x;
}
__device__ __forceinline__ GeoPoint geo_point(const Geom& G, int i, int j, int k, int64_t I) {
    const double tiny = 1e-300;
    const double x1 = G.x[0][i];
    double h1 = 1.0, h2 = 1.0, h3 = 1.0;
    if (G.metric != CLES_METRIC_CARTESIAN) h2 = x1;
    if (G.metric == CLES_METRIC_SPHERICAL) h3 = __dmul_rn(x1, G.sn[j]);
    h1 = geo_max(__dmul_rn(h1, G.m[0][i]), tiny);
    h2 = geo_max(__dmul_rn(h2, G.m[1][j]), tiny);
    h3 = geo_max(__dmul_rn(h3, G.m[2][k]), tiny);
    const double J = __dmul_rn(__dmul_rn(h1, h2), h3);
    GeoPoint p;
    p.inv_J = 1.0 / J;
    p.A[0] = J / h1;
    p.A[1] = J / h2;
    p.A[2] = J / h3;
    p.inv_h[0] = 1.0 / h1;
    p.inv_h[1] = 1.0 / h2;
    p.inv_h[2] = 1.0 / h3;
    p.inv_r = 1.0 / geo_max(x1, tiny);
    p.cotr = 0.0;
    if (G.metric == CLES_METRIC_SPHERICAL)
        p.cotr = G.cotr ? G.cotr[I] : G.cs[j] / geo_max(__dmul_rn(x1, G.sn[j]), tiny);
    return p;
}
__device__ __forceinline__ void cell_ijk(int64_t I, const int n[3], int& i, int& j, int& k) {
    i = (int)(I % n[0]);
    const int64_t r = I / n[0];
    j = (int)(r % n[1]);
    k = (int)(r / n[1]);
}
#endif

// A_d over the interior (double), and cot(theta)/r = inv_J * dA (GCL, src/metric.jl:154-170)
void geo_area(double* out, int d, const Geom& G, cudaStream_t st);
void geo_gcl(double* cotr, const double* dA, const Geom& G, cudaStream_t st);
// k_rate_final of pointwise.cu: reduce nb (rate, rho_min) partials
void rate_final(const double* part, int nb, double* out, cudaStream_t st);

// qface: per-node conserved state ([c][plane]) of a DirichletBC(fun) face, else null
void bc_plane(double* Q, const Grid3& g, int d, int side, int Ns, int kind, const BcState& s, cudaStream_t st,
              const double* qface = nullptr);
// Interior of one padded field (extents n + 2 pad, x fastest) into the interior layout.
void gather_interior(const double* padded, double* interior, const int n[3], const int pad[3], cudaStream_t st);

// Device clock of the graph-mode run loop: slots of a double[16] buffer.
enum { DC_T = 0, DC_DT = 1, DC_RATE = 2, DC_RHO_MIN = 3, DC_FAILURE = 4, DC_STEP = 5, DC_DT_SEEN = 6, DC_DONE = 7 };
struct ClockConst {
    double cfl, tfinal, nmax, dt_min, dt_min_ratio;
};
void clock_before(double* clk, const double* rate_rmin, const ClockConst& c, cudaStream_t st);
void clock_after(double* clk, const ClockConst& c, cudaStream_t st);
int64_t rate_partials(int64_t cells);

// ---- many grids advanced together (batch.cpp) ------------------------------
// The fields of every grid of a batch live in shared arena blocks: field f of
// grid g starts at element f * cells_total + off.  Per-cell kernels run over
// all cells_total elements at once; the kernels below take tables of grids,
// tiles, faces and cell chunks.
struct BatchGrid {
    Grid3 g;
    int64_t off;      // element offset of the grid's cell (0, 0, 0) in every block
    int64_t cells;
    double h[3];      // grid spacing (1 on a collapsed dimension)
    double* clk;      // graph-mode clock (DC_* slots) of this grid
    ClockConst cc;
};
// cells of one delta4_sum! tile (x, y, z)
constexpr int kD4X = 32, kD4Y = 16, kD4Z = 32;
struct BatchTile { int grid, x0, y0, z0; };     // one delta4 tile (kD4X x kD4Y x kD4Z cells)
struct BatchFace { int grid, d, side, kind; BcState st; };
struct BatchChunk { int grid; int64_t c0; };    // cells [c0, c0 + kBatchChunk) of a grid
constexpr int kBatchChunk = 2048;

template <typename F>
struct BatchOps {
    // primitives / fluxes of an ideal mixture whose species constants are per
    // member: mc[24 m ..] = R_k, cv_k, cp_k (8 each) of member m = tmap[cell / 64]
    static void primitives(const double* Q, F* prim, int64_t cells_total, int Ns, const PhysConst& pc, int esens,
                           const double* mc, const int* tmap, cudaStream_t st);
    static void fluxes(const double* Q, const F* prim, const F* g, const F* gty, const F* art, F* flux,
                       int64_t cells_total, int Ns, const PhysConst& pc, double mu0, double Pr, double Sc,
                       const double* mc, const int* tmap, cudaStream_t st);
    // delta4_sum! of one (f1 == nullptr) or two fields of every grid; field k
    // is weighted by h_d^pk per dimension
    static void delta4(const F* f0, const F* f1, F* o0, F* o1, int p0, int p1, const BatchGrid* grids,
                       const BatchTile* tiles, int ntiles, int64_t cells_total, cudaStream_t st);
    // max_rate of every grid (per-chunk partials, then one block per grid
    // reduces them) followed by the graph-mode clock_before of that grid;
    // chunk_first[g] .. chunk_first[g + 1] are grid g's chunks
    // LSRK update (src/timestep.jl:86-95) of the members with need[m] != 0,
    // each with the dt of its clock
    static void lsrk(double* Q, double* du, const F* dQ, int64_t cells_total, int ncons, const int* tmap,
                     const BatchGrid* grids, const int* need, double A, double B, cudaStream_t st);
    static void rate_clock(const double* Q, const F* prim, const F* art, const BatchGrid* grids, int G,
                           const BatchChunk* chunks, int nchunks, const int* chunk_first, double* part,
                           int64_t cells_total, int Ns, double mu0, double Pr, double Sc, cudaStream_t st);
};
// enforce! on the listed faces (one block per face)
void batch_bc(double* Q, const BatchGrid* grids, const BatchFace* faces, int nfaces, int64_t cells_total, int Ns,
              cudaStream_t st);
// clock_after of every grid
void batch_clock_after(const BatchGrid* grids, int G, cudaStream_t st);

}  // namespace cles
