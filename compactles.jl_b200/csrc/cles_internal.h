// Internal declarations shared by the host runtime and the CUDA kernels.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/cles.h"

namespace cles {

// ---------------------------------------------------------------- errors ----
struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};
void set_last_error(const std::string& s);
#define CLES_CUDA(call)                                                                         \
    do {                                                                                        \
        cudaError_t e_ = (call);                                                                \
        if (e_ != cudaSuccess)                                                                  \
            throw ::cles::Error(CLES_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)
void count_launch(int n = 1);
int64_t launch_count();   // kernels launched by this library so far
// CUDA-event bracketing of compact launches (cles_profile_enable)
bool profiling();
int prof_begin(cudaStream_t st, int family, double bytes);
void prof_end(int rec, cudaStream_t st);
void check_launch(const char* what);

// ------------------------------------------------------------ field views ----
// A batch of scalar fields of one grid: element (i, j, k) of field b sits at
// base + b*comp_stride + i + j*sy + k*sz (elements).  `base` points at
// interior element (0, 0, 0).
struct FieldView {
    void* base;
    int64_t comp_stride;
    int64_t sy, sz;
};

// ------------------------------------------------------------ compact plans ---
constexpr int kMaxSeg = 32;        // points per thread (register tile)
constexpr int kMaxClo = CLES_MAX_NC;
constexpr int kMaxCloLen = CLES_MAX_CLO_LEN;

// Kernel parameters of one directional compact operator (passed by value).
struct CompactParams {
    int n;               // line length
    int dim;             // 0, 1, 2
    int nx, ny, nz;      // interior extents of the grid
    int S;               // segments per line
    int seg_base, seg_rem;  // segment s: length seg_base + (s < seg_rem), local_range split
    int LB;              // lines per CTA
    int q, M;
    int symmetric;
    int periodic;
    int lo_closed, hi_closed;
    // an open end is a rank interface of a split line: interior rows whose
    // stencil reads the caller's halo, couplings beyond the end left to the
    // rank-level spikes
    int lo_open, hi_open;
    int nc;
    int hasred;
    double a0;
    double ci[CLES_MAX_M];
    int clo_len[kMaxClo];
    double clo[kMaxClo][kMaxCloLen];
    double chi[kMaxClo][kMaxCloLen];
    // offsets (elements) into the coefficient table
    int64_t off_f0, off_f1, off_f2, off_f3, off_f4;  // q=1: l, dinv, c ; q=2: L1, L2, U1, U2, Uinv0
    int64_t off_V, off_W;                              // V[s][t][i], W[s][t][i]
    int64_t off_G;                                     // reduced inverse, (2qS) x (2qS) row-major
    // Closed tridiagonal lines: the interface system is solved by parallel
    // cyclic reduction with precomputed 2x2 blocks instead of the dense inverse.
    // Level l (distance 2^l), segment s: alpha[4], gamma[4] at off_pcr + (l*S + s)*8,
    // then the final 2x2 inverse of segment s at off_pcr + (pcr_levels*S + s)*8.
    int pcr, pcr_levels;
    int64_t off_pcr;
    int64_t lines;
};

// Warp-per-line form for periodic tridiagonal x lines of n = 32 * XP points
// (XP = 2, 4, 6, 8, 12, 16: n = 64, 128, 192, 256, 384, 512):
// lane s owns the XP contiguous points [s*XP, (s+1)*XP).  Every lane segment
// is the same Toeplitz block, so the local factorisation, the spikes and the
// parallel-cyclic-reduction matrices of the 32-segment interface system are
// line- and lane-independent and travel as kernel parameters.
constexpr int kMaxXP = 16;
struct WarpLineParams {
    int XP;                                   // points per lane: 2, 4, 6, 8, 12 or 16
    double l[kMaxXP], dinv[kMaxXP], c[kMaxXP];  // segment Thomas factors
    double v[kMaxXP], w[kMaxXP];              // spikes: couplings to the previous tail / next head
    double alpha[4][4], gamma[4][4];          // PCR steps at distances 1, 2, 4, 8 (2x2, row-major)
    double alpha_f[4], binv_f[4];             // pairing at distance 16, then the 2x2 solve
    float lf[kMaxXP], dinvf[kMaxXP], cf[kMaxXP], vf[kMaxXP], wf[kMaxXP];
    float alphaf[4][4], gammaf[4][4], alpha_ff[4], binv_ff[4];
};

// TMA-pipelined form for periodic tridiagonal y/z lines with equal segments
// (n = S * m, m <= 32, n <= 256): every segment has the same factorisation and
// spikes, which travel as kernel parameters; the reduced inverse stays in the
// table (copied to shared memory once per persistent CTA).
struct TileLineParams {
    int m;
    double l[kMaxSeg], dinv[kMaxSeg], c[kMaxSeg], v[kMaxSeg], w[kMaxSeg];
    float lf[kMaxSeg], dinvf[kMaxSeg], cf[kMaxSeg], vf[kMaxSeg], wf[kMaxSeg];
};

// Host-side plan: parameters plus the coefficient tables on the device.
// General tile form (closed lines, or the pentadiagonal C10): with equal
// segments only three segment classes exist -- the first (closure rows, no
// left spike), the interior ones (all alike) and the last -- so their
// factorisations and spikes travel as kernel parameters with static indices.
// f: q = 1 -> l, dinv, c; q = 2 -> L1, L2, U1, U2, 1/U0 (same as the table).
struct TileGenParams {
    double f[3][5][kMaxSeg];
    double v[3][2][kMaxSeg], w[3][2][kMaxSeg];
    float ff[3][5][kMaxSeg];
    float vf[3][2][kMaxSeg], wf[3][2][kMaxSeg];
};

struct SigPlan;
struct CompactPlan {
    bool has_tl = false;
    TileLineParams TL;
    bool has_tg = false;   // y/z lines fit the general tile kernel (closures, q = 2)
    TileGenParams TG;
    bool has_xw = false;
    WarpLineParams XW;
    CompactParams P;
    int dtype = CLES_F64;
    double* tab64 = nullptr;
    float* tab32 = nullptr;
    size_t tab_elems = 0;
    // few long closed x lines: the line is cut into pieces solved side by side
    std::unique_ptr<SigPlan> sig;
    ~CompactPlan();
};

// Few long closed x lines (1-D problems, very thin 2-D grids) split into P
// pieces inside the GPU: the reference's P > 1 line solve (src/tridiag.jl:
// 136-170, src/banded.jl:177-214) with the pieces of one line in place of
// ranks and global memory in place of the exchange.  Pieces of one class
// share a local plan: the first (closed low end, open high end), the P - 2
// middle ones (both ends open, equal lengths) and the last.  One launch
// solves every piece with its halo read from the neighbouring pieces and
// writes its heads and tails; a second forms the reduced system's unknowns
// beside each piece from the dense inverse G and corrects:
// x = y - V z_prev - W z_next.
constexpr int kSigFields = 12;   // fields per pass (larger counts run in passes)
struct SigPlan {
    int P = 0, q = 1;
    int len[3] = {0, 0, 0};        // piece length of the first, middle and last class
    int64_t lines = 0;             // lines of the whole plan
    CompactPlan cls[3];            // local plans of the classes (forced equal S and LB)
    int dtype = CLES_F64;
    void* tab = nullptr;           // class c: V [q][len_c], W [q][len_c]; then G (2qP)^2; plan dtype
    int64_t off_V[3] = {0, 0, 0}, off_W[3] = {0, 0, 0}, off_G = 0;
    void* loc = nullptr;           // local solutions: kSigFields x lines x n
    void* iface[3] = {nullptr, nullptr, nullptr};   // heads / tails: kSigFields x 2q x lines of the class
    ~SigPlan();
};

// Builds the plan of `scheme` along `dim` (0-based) of a grid with interior
// extents n3[3]; periodic says whether the line wraps.  lo_fold / hi_fold set
// a coordinate-singularity fold at that end of a closed line: the antipodal
// parity (+1 / -1) of the field the plan is applied to, 0 for a closure.
// lo_open / hi_open make that end of a non-periodic line a rank interface.
// pow2_seg_max > 0 (batched plans): S is the fewest power-of-two segments of
// at most pow2_seg_max (8, 16 or 32) points.
// force_S / force_LB > 0 fix the segments per line and the lines per CTA (the
// classes of a SigPlan, which share one launch).
void build_compact_plan(CompactPlan& plan, const cles_scheme& scheme, const int n3[3], int dim,
                        bool periodic, double h, int dtype, int lo_fold = 0, int hi_fold = 0,
                        bool lo_open = false, bool hi_open = false, int pow2_seg_max = 0, int force_S = 0,
                        int force_LB = 0);

// The LHS band of one line (or one rank's piece of a split line), row-major
// n x (2q+1): interior band, closure rows at closed ends, parity folds, and
// no couplings beyond a non-periodic end.  Unpivoted banded LU of the whole
// band; solve() applies its inverse in place.
struct LineBand {
    int n = 0, q = 1;
    std::vector<double> a;
    std::vector<double> L, U;
    void factor();
    void solve(double* x) const;
};
LineBand make_line_band(const cles_scheme& s, int n, int lo_fold, int hi_fold, bool lo_open, bool hi_open);

// Output modes of the compact operator.  OUT_RK finishes the flux divergence
// and applies the low-storage RK update in the store (see launch_compact_rk).
enum { OUT_STORE = 0, OUT_NEGATE = 1, OUT_SUBTRACT = 2, OUT_RK = 3 };

// Low-storage RK epilogue: with dq = out - D(f), v = A du + dt dq; du = v;
// Q += B v (src/timestep.jl:86-95).  Q and du share the layout of `out`.
struct RkEpilogue {
    double* Q;
    double* du;
    double A, B, dt;
    const double* dtp;  // when set, dt is read from device memory (graph mode)
};

// TMA-pipelined y/z launch; false when the plan or the views do not qualify.
bool try_launch_tma(const CompactPlan& plan, const FieldView& in, const FieldView& out, int count, int mode,
                    cudaStream_t st, const RkEpilogue* rk = nullptr);
// x lines of a plan with the general tile form: persistent kernel, cp.async
// staging into a transposed shared-memory tile; false if the plan does not fit.
bool try_launch_xt(const CompactPlan& plan, const FieldView& in, const FieldView& out, int count, int mode,
                   cudaStream_t st);
// Flux divergence of the last direction fused with the RK update; false (and
// nothing launched) when the plan does not take the TMA path.
bool launch_compact_rk(const CompactPlan& plan, const FieldView& in, const FieldView& out, int count,
                       const RkEpilogue& rk, cudaStream_t st);
// One rank's piece of a line split across `ranks` ranks along `dim`
// (src/decomposition.jl:73-78 local_range; src/tridiag.jl:85-170 and
// src/banded.jl:108-214 with P > 1).  `local` solves the rank's own rows with
// open (interface) ends.  V / W are this rank's spikes: the response of its
// local solve to the couplings of its first q rows to the previous rank's
// last q unknowns and of its last q rows to the next rank's first q.  Gsel
// holds the 2q rows of the inverse of the (2q ranks)^2 reduced system that
// give those 2q unknowns from every rank's local heads and tails.
struct SplitPlan {
    CompactPlan local;
    int ranks = 1, rank = 0, dim = 0, q = 1, M = 1, n = 0;
    int n3[3] = {0, 0, 0};
    int64_t lines = 0;
    bool lo_open = false, hi_open = false;
    int prev = -1, next = -1;   // neighbouring rank coordinates, -1 for none
    int dtype = CLES_F64;
    void* tab = nullptr;        // [V q x n][W q x n][Gsel 2q x 2q*ranks], plan dtype
    ~SplitPlan();
};
void build_split_plan(SplitPlan& sp, const cles_scheme& s, const int n3_local[3], int dim, bool periodic,
                      int n_global, int ranks, int rank, double h, int dtype);
// The M planes at each end of a local interior along `dim` (lines: the
// product of the other two extents, lower dimension fastest).
struct HaloSpec {
    int dim = 0;
    int n3[3] = {0, 0, 0};
    int M = 0;
    int64_t lines = 0;
    bool lo_open = false, hi_open = false;
};
HaloSpec halo_spec(const SplitPlan& sp);
// Copies the M planes next to each open end of the local interior into lo / hi
// ([count][M][lines]) when pack, or those buffers into the halo planes
// beyond each open end when !pack.
void halo_planes(const HaloSpec& hs, const FieldView& f, void* lo, void* hi, int count, bool pack, int dtype,
                 cudaStream_t st);
void split_halo(const SplitPlan& sp, const FieldView& f, void* lo, void* hi, int count, bool pack, cudaStream_t st);
// From every rank's heads and tails ([ranks][count][2q][lines]): the 2q
// neighbouring unknowns per line into zbuf ([count][2q][lines]), then
// out -= V z_prev + W z_next over the local interior.
void split_correct(const SplitPlan& sp, const void* gathered, void* zbuf, const FieldView& out, int count,
                   cudaStream_t st);
// The same with the local solution read from `loc` and the corrected value
// r = loc - V z_prev - W z_next written to `out` by mode: OUT_STORE out = r,
// OUT_NEGATE out = -r, OUT_SUBTRACT out -= r (loc may alias out except for
// OUT_SUBTRACT).
void split_correct(const SplitPlan& sp, const void* gathered, void* zbuf, const FieldView& loc, const FieldView& out,
                   int count, int mode, cudaStream_t st);
// dst = src over an n3 interior of `count` fields (views of equal extents,
// any strides).
void copy_view(const FieldView& src, const FieldView& dst, const int n3[3], int count, int dtype, cudaStream_t st);

// ---- batched line solves over many grids (batch_compact.cu) ----------------
// One grid's directional plan in a batched launch.  Its lines are cut into
// power-of-two segments (build_compact_plan with pow2_segments), and P.LB is
// the launch's threads / P.S, so every CTA of the launch runs LB x S threads.
// The grid's fields start at element `off` of the launch's arena blocks.
struct BatchLinePlan {
    CompactParams P;
    const void* tab;      // the plan's coefficient table (launch dtype)
    int64_t off;          // element offset of the grid's cell (0, 0, 0)
    int64_t sy, sz;       // strides of the grid's fields
    const double* clk;    // graph-mode clock of the grid (dt in slot 1)
};
constexpr int kBatchMaxThreads = 512;   // threads per CTA of a batched line-solve launch (at most)
// Kernel template of a batched launch (shared by all its plans).
struct BatchLaunchKind {
    int dtype;            // CLES_F64 / CLES_F32
    int q, M, xmode;
    int ms;               // register tile: 8, 16 or 32 points (>= every plan's longest segment)
    int threads;          // LB x S of every plan
    size_t smem;          // dynamic shared memory (max over the plans)
};
// Dynamic shared memory one plan needs with LB lines per CTA.
size_t batch_plan_smem(const CompactParams& P, int LB, int dtype);
// blocks[b] = (plan, first line); blockIdx.y = field.  in / out / Q / du are
// arena block starts (fields cells_total elements apart).  mode OUT_RK applies
// the low-storage RK update with coefficients (A, B) and each grid's dt
// (clk[1]); skip_idle leaves out every grid whose dt is 0 (done or failed).
void launch_compact_batch(const BatchLaunchKind& kind, const BatchLinePlan* plans, const int2* blocks, int nblocks,
                          const void* in, void* out, int64_t cells_total, int count, int mode, double* Q, double* du,
                          double A, double B, int skip_idle, cudaStream_t st);

// Bounded-wait timeouts recorded by device kernels since the last call (cleared).
int take_device_timeouts(cudaStream_t st);
// One CTA that waits limit_ns on an mbarrier nothing completes (the expiry
// path of the operators' bounded wait).
void launch_wait_selftest(uint64_t limit_ns, cudaStream_t st);

// Launch the operator over `count` fields of `in` into `out` (may alias).
void launch_compact(const CompactPlan& plan, const FieldView& in, const FieldView& out, int count, int mode,
                    cudaStream_t st);
// y/z lines of a split-line plan in the general tile form, the TMA box
// widened by the M halo rows at each end; false (nothing launched) when the
// plan or the views do not qualify.
bool try_launch_tg_split(const CompactPlan& plan, const FieldView& in, const FieldView& out, int count, void* iface,
                         cudaStream_t st);
// Local solve of a split-line plan (tile or generic kernel, OUT_STORE); the first and
// last q values of every line's local solution also go to iface, laid out
// [count][2q][lines] in the plan's dtype.
void launch_compact_split(const CompactPlan& plan, const FieldView& in, const FieldView& out, int count, void* iface,
                          cudaStream_t st);

}  // namespace cles
