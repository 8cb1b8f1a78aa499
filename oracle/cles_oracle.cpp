// CPU FP64 oracle for the RHS-and-step hot path of CompactLES.jl.
//
// TEST INFRASTRUCTURE ONLY.  This file restates the reference's Julia
// algorithm in C++ so that the CUDA library can be checked against it and so
// that the CPU baseline can be timed.  Only tests/, __graft_entry__.smoke()
// and bench.py's CPU-baseline / reference arm may load it.  Nothing in the
// product links or calls it.
//
// Parity status: the reference is Julia and Julia is not available where
// this runs, so bit-level agreement with the Julia runtime is unpinned.  The
// restatement is pinned by the reference's own known-answer tests (spectral
// accuracy, polynomial exactness, freestream, conservation, filter constants,
// convergence orders, Sod/Lax/Shu-Osher/Woodward-Colella measured numbers and
// stored profiles), which tests/test_oracle_*.py reproduce.
//
// Storage follows the reference (src/decomposition.jl:129-134): each field is
// a padded array, x fastest, n_local + 2*n_halo per active dimension, and the
// conserved state appends the component as the slowest index.  Loop order and
// floating-point association follow the cited Julia lines; the file is
// compiled with -ffp-contract=off so a*b+c is never fused, matching Julia
// without @fastmath/muladd.
//
// The distributed spike solve (LineSolver / BandLineSolver with P > 1 ranks
// along a dimension, src/tridiag.jl:85-170, src/banded.jl:108-214) is
// restated too: a plan may emulate P ranks along its dimension in one
// process, with the Allgather replaced by direct reads of every rank's ends.

#include "../include/cles.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <memory>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// ---------------------------------------------------------------- helpers --

// Julia's max/min on Float64: NaN wins, -0.0 < 0.0 (Base.max/min semantics).
inline double jl_max(double x, double y) {
    if (std::isnan(x)) return x;
    if (std::isnan(y)) return y;
    if (y > x) return y;
    if (x > y) return x;
    return std::signbit(x) ? y : x;
}
inline double jl_min(double x, double y) {
    if (std::isnan(x)) return x;
    if (std::isnan(y)) return y;
    if (y < x) return y;
    if (x < y) return x;
    return std::signbit(x) ? x : y;
}
inline int jl_mod(int a, int n) { int r = a % n; return r < 0 ? r + n : r; }

thread_local std::string g_err;

// Minimum work (grid points) for a threaded region, as THREAD_MIN_WORK = 2^15
// in src/threading.jl:47; below it loops run inline.
const long kThreadMinWork = 1L << 15;
void set_err(const std::string& s) { g_err = s; }

// ----------------------------------------------------------- decomposition --
// Single-process Decomp (src/decomposition.jl:80-122): n_local = n_global,
// one rank in every sub-communicator.
struct Decomp {
    int ng[3];
    bool periodic[3];
    int nh;
    bool active[3];
    int nhd[3];
    int nl[3];
    int full[3];
    size_t size() const { return (size_t)full[0] * full[1] * full[2]; }
    // 0-based padded index
    size_t at(int i, int j, int k) const { return (size_t)i + (size_t)full[0] * ((size_t)j + (size_t)full[1] * k); }
    // at_lo_edge / at_hi_edge (src/decomposition.jl:137-140), one rank per dim.
    bool closed(int d) const { return active[d] && !periodic[d]; }
};

Decomp make_decomp(const int ng[3], const int per[3], int nh) {
    Decomp D;
    D.nh = nh;
    for (int d = 0; d < 3; ++d) {
        D.ng[d] = ng[d];
        D.active[d] = ng[d] > 1;
        D.periodic[d] = D.active[d] ? (per[d] != 0) : true;
        D.nhd[d] = D.active[d] ? nh : 0;
        D.nl[d] = ng[d];
        D.full[d] = ng[d] + 2 * D.nhd[d];
    }
    return D;
}

// local_range (src/decomposition.jl:73-78)
void local_range(int N, int P, int r, int* n, int* off) {
    int base = N / P, rem = N % P;
    *n = base + (r < rem ? 1 : 0);
    *off = r * base + std::min(r, rem);
}

// ------------------------------------------------------------------- halos --
// wrap_dim! (src/halo.jl:27-36) for one field: periodic self-copy of n_halo
// planes.  Used under selfwrap (periodic, one rank) only; closed dims are
// left stale exactly like a PROC_NULL Sendrecv.
void wrap_dim(const Decomp& D, double* f, int d) {
    if (!D.active[d] || !D.periodic[d]) return;
    const int nh = D.nh, n = D.nl[d];
    const int F0 = D.full[0], F1 = D.full[1], F2 = D.full[2];
    auto copy_plane = [&](int dst, int src) {
        if (d == 0) {
            for (int k = 0; k < F2; ++k)
                for (int j = 0; j < F1; ++j) f[D.at(dst, j, k)] = f[D.at(src, j, k)];
        } else if (d == 1) {
            for (int k = 0; k < F2; ++k)
                std::memcpy(&f[D.at(0, dst, k)], &f[D.at(0, src, k)], sizeof(double) * F0);
        } else {
            std::memcpy(&f[D.at(0, 0, dst)], &f[D.at(0, 0, src)], sizeof(double) * (size_t)F0 * F1);
        }
    };
    // low halos 1:nh <- n+1:n+nh ; high halos n+nh+1:n+2nh <- nh+1:2nh (1-based)
    for (int t = 0; t < nh; ++t) copy_plane(t, n + t);
    for (int t = 0; t < nh; ++t) copy_plane(n + nh + t, nh + t);
}
// exchange_halos! (src/halo.jl:84-89): dims in order x, y, z.
void exchange_halos(const Decomp& D, double* f) {
    for (int d = 0; d < 3; ++d) wrap_dim(D, f, d);
}
// copy_interior! (src/halo.jl:102-112)
void copy_interior(const Decomp& D, double* dst, const double* src) {
    const int o1 = D.nhd[0], o2 = D.nhd[1], o3 = D.nhd[2];
    const long work = (long)D.nl[0] * D.nl[1] * D.nl[2];
#pragma omp parallel for collapse(2) schedule(static) if (work >= kThreadMinWork)
    for (int k = 0; k < D.nl[2]; ++k)
        for (int j = 0; j < D.nl[1]; ++j)
            for (int i = 0; i < D.nl[0]; ++i) dst[D.at(i + o1, j + o2, k + o3)] = src[D.at(i + o1, j + o2, k + o3)];
}

// ------------------------------------------------------------------ schemes --
// Presets restated from src/kernels.jl:61-111 and src/kernels_banded.jl:54-64.
void scheme_clear(cles_scheme* s) { std::memset(s, 0, sizeof(*s)); }

void set_tri_closure(cles_scheme* s, int j, double sub, double dia, double sup, std::initializer_list<double> rhs) {
    s->clo_lhs[j][0] = sub; s->clo_lhs[j][1] = dia; s->clo_lhs[j][2] = sup;
    int n = 0;
    for (double v : rhs) s->clo_rhs[j][n++] = v;
    s->clo_len[j] = n;
}

void preset_lele_d1_6(cles_scheme* s) {
    scheme_clear(s);
    std::snprintf(s->name, sizeof(s->name), "Lele C6 first derivative");
    s->q = 1; s->lhs[0] = 1.0 / 3.0; s->a0 = 0.0;
    s->M = 2; s->coeffs[0] = 7.0 / 9.0; s->coeffs[1] = 1.0 / 36.0;
    s->symmetric = 0; s->nc = 2;
    set_tri_closure(s, 0, 0.0, 1.0, 2.0, {-5.0 / 2.0, 2.0, 1.0 / 2.0});
    set_tri_closure(s, 1, 1.0 / 4.0, 1.0, 1.0 / 4.0, {-3.0 / 4.0, 0.0, 3.0 / 4.0});
}
void preset_pade_d1_4(cles_scheme* s) {
    scheme_clear(s);
    std::snprintf(s->name, sizeof(s->name), "Pade C4 first derivative");
    s->q = 1; s->lhs[0] = 1.0 / 4.0; s->a0 = 0.0;
    s->M = 1; s->coeffs[0] = 3.0 / 4.0;
    s->symmetric = 0; s->nc = 1;
    set_tri_closure(s, 0, 0.0, 1.0, 2.0, {-5.0 / 2.0, 2.0, 1.0 / 2.0});
}
void preset_compact_filter(double alphaf, cles_scheme* s) {
    scheme_clear(s);
    std::snprintf(s->name, sizeof(s->name), "Gaitonde-Visbal C8 filter");
    const double af = alphaf;
    const double a0 = (93 + 70 * af) / 128;
    const double a1 = (7 + 18 * af) / 16;
    const double a2 = (-7 + 14 * af) / 32;
    const double a3 = (1 - 2 * af) / 16;
    const double a4 = (-1 + 2 * af) / 128;
    s->q = 1; s->lhs[0] = af; s->a0 = a0;
    s->M = 4; s->coeffs[0] = a1 / 2; s->coeffs[1] = a2 / 2; s->coeffs[2] = a3 / 2; s->coeffs[3] = a4 / 2;
    s->symmetric = 1; s->nc = 4;
    // boundary cascade: row 1 identity; rows 2-4 centred filters of order 2,4,6
    const double b2[2] = {(1 + 2 * af) / 2, (1 + 2 * af) / 2};
    const double b4[3] = {(5 + 6 * af) / 8, (1 + 2 * af) / 2, (-1 + 2 * af) / 8};
    const double b6[4] = {(11 + 10 * af) / 16, (15 + 34 * af) / 32, (-3 + 6 * af) / 16, (1 - 2 * af) / 32};
    auto ctr = [&](int j, const double* c, int len) {
        // [c[m+1]/2 for m = len-1..1] ; c[1] ; [c[m+1]/2 for m = 1..len-1]
        int n = 0;
        for (int m = len - 1; m >= 1; --m) s->clo_rhs[j][n++] = c[m] / 2;
        s->clo_rhs[j][n++] = c[0];
        for (int m = 1; m <= len - 1; ++m) s->clo_rhs[j][n++] = c[m] / 2;
        s->clo_len[j] = n;
    };
    s->clo_lhs[0][0] = 0.0; s->clo_lhs[0][1] = 1.0; s->clo_lhs[0][2] = 0.0;
    s->clo_rhs[0][0] = 1.0; s->clo_len[0] = 1;
    for (int j = 1; j < 4; ++j) { s->clo_lhs[j][0] = af; s->clo_lhs[j][1] = 1.0; s->clo_lhs[j][2] = af; }
    ctr(1, b2, 2);
    ctr(2, b4, 3);
    ctr(3, b6, 4);
}
void preset_lele_d1_10(cles_scheme* s) {
    scheme_clear(s);
    std::snprintf(s->name, sizeof(s->name), "Lele C10 first derivative");
    s->q = 2; s->lhs[0] = 1.0 / 2.0; s->lhs[1] = 1.0 / 20.0; s->a0 = 0.0;
    s->M = 3; s->coeffs[0] = 17.0 / 24.0; s->coeffs[1] = 101.0 / 600.0; s->coeffs[2] = 1.0 / 600.0;
    s->symmetric = 0; s->nc = 3;
    const double l0[5] = {0, 0, 1, 2, 0}, l1[5] = {0, 1.0 / 4.0, 1, 1.0 / 4.0, 0}, l2[5] = {0, 1.0 / 3.0, 1, 1.0 / 3.0, 0};
    const double r0[3] = {-5.0 / 2.0, 2.0, 1.0 / 2.0}, r1[3] = {-3.0 / 4.0, 0.0, 3.0 / 4.0};
    const double r2[5] = {-1.0 / 36.0, -7.0 / 9.0, 0.0, 7.0 / 9.0, 1.0 / 36.0};
    for (int t = 0; t < 5; ++t) { s->clo_lhs[0][t] = l0[t]; s->clo_lhs[1][t] = l1[t]; s->clo_lhs[2][t] = l2[t]; }
    for (int t = 0; t < 3; ++t) { s->clo_rhs[0][t] = r0[t]; s->clo_rhs[1][t] = r1[t]; }
    for (int t = 0; t < 5; ++t) s->clo_rhs[2][t] = r2[t];
    s->clo_len[0] = 3; s->clo_len[1] = 3; s->clo_len[2] = 5;
}

// ------------------------------------------------------------- dense LU ------
// The reduced interface system is LU-factorised by LinearAlgebra.lu! (LAPACK
// getrf, partial pivoting) and solved by ldiv! (getrs) at src/tridiag.jl:123,157
// and src/banded.jl:169,199.  Restated as the unblocked right-looking getf2
// (pivot = first max |a|, column scaled by the reciprocal of the pivot) and
// getrs (row swaps, unit-lower forward, upper backward with division).
struct DenseLU {
    int n = 0;
    std::vector<double> a;  // column-major n x n, L\U
    std::vector<int> piv;
    void factor(std::vector<double> A, int nn) {
        n = nn; a = std::move(A); piv.assign(n, 0);
        for (int j = 0; j < n; ++j) {
            int jp = j; double best = std::fabs(a[j + (size_t)n * j]);
            for (int i = j + 1; i < n; ++i) {
                double v = std::fabs(a[i + (size_t)n * j]);
                if (v > best) { best = v; jp = i; }
            }
            piv[j] = jp;
            if (a[jp + (size_t)n * j] != 0.0) {
                if (jp != j)
                    for (int c = 0; c < n; ++c) std::swap(a[j + (size_t)n * c], a[jp + (size_t)n * c]);
                const double r = 1.0 / a[j + (size_t)n * j];
                for (int i = j + 1; i < n; ++i) a[i + (size_t)n * j] *= r;
            }
            for (int c = j + 1; c < n; ++c) {
                const double t = -a[j + (size_t)n * c];
                if (t != 0.0)
                    for (int i = j + 1; i < n; ++i) a[i + (size_t)n * c] += a[i + (size_t)n * j] * t;
            }
        }
    }
    void solve(double* b) const {  // one right-hand side, in place
        for (int j = 0; j < n; ++j) if (piv[j] != j) std::swap(b[j], b[piv[j]]);
        for (int k = 0; k < n; ++k)
            if (b[k] != 0.0)
                for (int i = k + 1; i < n; ++i) b[i] -= b[k] * a[i + (size_t)n * k];
        for (int k = n - 1; k >= 0; --k)
            if (b[k] != 0.0) {
                b[k] /= a[k + (size_t)n * k];
                for (int i = 0; i < k; ++i) b[i] -= b[k] * a[i + (size_t)n * k];
            }
    }
};

// ------------------------------------------------------------ line solvers ---
// TriFactor + solve_col! (src/tridiag.jl:24-57)
struct TriFactor {
    int n = 0;
    std::vector<double> l, dinv, c;
    void build(const std::vector<double>& a, const std::vector<double>& b, const std::vector<double>& cc) {
        n = (int)b.size();
        l.assign(n, 0.0); dinv.assign(n, 0.0); c = cc;
        double d = b[0];
        dinv[0] = 1.0 / d;
        for (int i = 1; i < n; ++i) {
            l[i] = a[i] * dinv[i - 1];
            d = b[i] - l[i] * c[i - 1];
            dinv[i] = 1.0 / d;
        }
    }
    // x: n values with stride st
    void solve(double* x, ptrdiff_t st) const {
        for (int i = 1; i < n; ++i) x[i * st] -= l[i] * x[(i - 1) * st];
        x[(n - 1) * st] *= dinv[n - 1];
        for (int i = n - 2; i >= 0; --i) x[i * st] = (x[i * st] - c[i] * x[(i + 1) * st]) * dinv[i];
    }
};

// BandFactor + solve_col! (src/banded.jl:31-80).  Ab[(q+s) + (2q+1)*i] = A[i,i+s].
struct BandFactor {
    int n = 0, q = 0;
    std::vector<double> L;  // q x n, L[(m-1) + q*k]
    std::vector<double> U;  // (q+1) x n, U[s + (q+1)*i]
    void build(const std::vector<double>& Ab, int nn, int qq) {
        n = nn; q = qq;
        const int W = 2 * q + 1;
        std::vector<double> Wk = Ab;
        L.assign((size_t)q * n, 0.0);
        for (int k = 0; k < n - 1; ++k) {
            const double piv = Wk[q + (size_t)W * k];
            const int mmax = std::min(q, n - 1 - k);
            for (int m = 1; m <= mmax; ++m) {
                const int i = k + m;
                const double lv = Wk[(q - m) + (size_t)W * i] / piv;
                L[(m - 1) + (size_t)q * k] = lv;
                for (int t = 1; t <= mmax; ++t)
                    Wk[(q + t - m) + (size_t)W * i] -= lv * Wk[(q + t) + (size_t)W * k];
            }
        }
        U.assign((size_t)(q + 1) * n, 0.0);
        for (int i = 0; i < n; ++i)
            for (int s = 0; s <= std::min(q, n - 1 - i); ++s) U[s + (size_t)(q + 1) * i] = Wk[(q + s) + (size_t)W * i];
    }
    // x path (solve_col!, division by the pivot)
    void solve(double* x, ptrdiff_t st) const {
        for (int k = 0; k < n - 1; ++k) {
            const double xk = x[k * st];
            for (int m = 1; m <= std::min(q, n - 1 - k); ++m) x[(k + m) * st] -= L[(m - 1) + (size_t)q * k] * xk;
        }
        for (int i = n - 1; i >= 0; --i) {
            double acc = x[i * st];
            for (int t = 1; t <= std::min(q, n - 1 - i); ++t) acc -= U[t + (size_t)(q + 1) * i] * x[(i + t) * st];
            x[i * st] = acc / U[(size_t)(q + 1) * i];
        }
    }
    // transposed path (solve_lines_t!, src/lines_transposed.jl:86-120):
    // sequential in-place updates and multiplication by inv(U[1,i]).
    void solve_t(double* x, ptrdiff_t st) const {
        for (int k = 0; k < n - 1; ++k)
            for (int m = 1; m <= std::min(q, n - 1 - k); ++m) {
                const double lm = L[(m - 1) + (size_t)q * k];
                if (lm == 0.0) continue;
                x[(k + m) * st] -= lm * x[k * st];
            }
        for (int i = n - 1; i >= 0; --i) {
            for (int t = 1; t <= std::min(q, n - 1 - i); ++t) x[i * st] -= U[t + (size_t)(q + 1) * i] * x[(i + t) * st];
            const double u0 = 1.0 / U[(size_t)(q + 1) * i];
            x[i * st] *= u0;
        }
    }
};

// One emulated rank's share of a line.
struct RankPart {
    int n = 0, off = 0;
    bool lo_closed = false, hi_closed = false;
    int fold_lo = 0, fold_hi = 0;   // parity fold sign of the solution at a folded edge (0 = none)
    TriFactor tf;             // q == 1 path
    BandFactor bf;            // q >= 2 path
    std::vector<double> V, W; // n x q each (column-major: V[i + n*t])
};

// LineSolver / BandLineSolver with P emulated ranks (src/tridiag.jl:59-170,
// src/banded.jl:82-214, src/lines_transposed.jl:22-151).
struct DistSolver {
    int n_global = 0, q = 1, P = 1;
    bool periodic = false, banded = false, hasred = false;
    std::vector<RankPart> parts;
    DenseLU red;

    void solve_local(const RankPart& rp, double* x, ptrdiff_t st, bool transposed) const {
        if (!banded) rp.tf.solve(x, st);
        else if (transposed) rp.bf.solve_t(x, st);
        else rp.bf.solve(x, st);
    }
};

// ------------------------------------------------------------------- plans ---
struct Plan {
    Decomp D;
    int dim = 0;           // 0-based
    int n = 0;
    int lines = 0;
    cles_scheme scheme;
    bool lo_closed = false, hi_closed = false;
    int lo_fold = 0, hi_fold = 0;   // sigma_g of a folded edge (0 = none)
    double a0 = 0.0;
    std::vector<double> ci;
    std::vector<std::vector<double>> clo, chi;
    DistSolver ls;
};

// Build one rank's local tridiagonal LHS (src/operators.jl:66-84) and its
// LineSolver pieces (src/tridiag.jl:85-100).
void build_tri_part(const cles_scheme& s, RankPart& rp) {
    const int n = rp.n, nc = s.nc;
    const double al = s.lhs[0];
    std::vector<double> a(n, al), b(n, 1.0), c(n, al);
    if (rp.lo_closed)
        for (int j = 0; j < nc; ++j) { a[j] = s.clo_lhs[j][0]; b[j] = s.clo_lhs[j][1]; c[j] = s.clo_lhs[j][2]; }
    if (rp.hi_closed)
        for (int j = 0; j < nc; ++j) {
            const int r = n - 1 - j;
            a[r] = s.clo_lhs[j][2]; b[r] = s.clo_lhs[j][1]; c[r] = s.clo_lhs[j][0];
        }
    // parity fold on a half-offset grid (src/operators.jl:61-70): the coupling
    // to the ghost unknown g_0 = sigma_g g_1 moves onto the diagonal
    if (rp.fold_lo) b[0] += (double)rp.fold_lo * al;
    if (rp.fold_hi) b[n - 1] += (double)rp.fold_hi * al;
    const double aL = (rp.lo_closed || rp.fold_lo) ? 0.0 : al;
    const double cR = (rp.hi_closed || rp.fold_hi) ? 0.0 : al;
    rp.tf.build(a, b, c);
    rp.V.assign(n, 0.0); rp.W.assign(n, 0.0);
    if (aL != 0.0) { rp.V[0] = aL; rp.tf.solve(rp.V.data(), 1); }
    if (cR != 0.0) { rp.W[n - 1] = cR; rp.tf.solve(rp.W.data(), 1); }
}

// One rank's banded LHS (src/operators_banded.jl:48-112) and BandLineSolver
// spikes (src/banded.jl:108-135).
bool build_band_part(const cles_scheme& s, RankPart& rp) {
    const int n = rp.n, q = s.q, nc = s.nc, W = 2 * q + 1;
    std::vector<double> Ab((size_t)W * n, 0.0);
    for (int i = 0; i < n; ++i) {
        Ab[q + (size_t)W * i] = 1.0;
        for (int t = 1; t <= q; ++t) { Ab[(q + t) + (size_t)W * i] = s.lhs[t - 1]; Ab[(q - t) + (size_t)W * i] = s.lhs[t - 1]; }
    }
    // parity folds (src/operators_banded.jl:58-77): row i's coupling to ghost
    // column i-m maps onto interior column m-i+1 (1-based) with sign sigma_g
    if (rp.fold_lo)
        for (int i = 1; i <= q; ++i)
            for (int m = 1; m <= q; ++m) {
                if (i - m >= 1) continue;
                const int jcol = m - i + 1;
                Ab[(q + (jcol - i)) + (size_t)W * (i - 1)] += (double)rp.fold_lo * s.lhs[m - 1];
            }
    if (rp.fold_hi)
        for (int i = n - q + 1; i <= n; ++i)
            for (int m = 1; m <= q; ++m) {
                if (i + m <= n) continue;
                const int jcol = 2 * n + 1 - (i + m);
                Ab[(q + (jcol - i)) + (size_t)W * (i - 1)] += (double)rp.fold_hi * s.lhs[m - 1];
            }
    if (rp.lo_closed)
        for (int j = 0; j < nc; ++j)
            for (int t = -q; t <= q; ++t) {
                if (j + t < 0 && s.clo_lhs[j][q + t] != 0.0) { set_err("closure row references a column before the edge"); return false; }
                Ab[(q + t) + (size_t)W * j] = s.clo_lhs[j][q + t];
            }
    if (rp.hi_closed)
        for (int j = 0; j < nc; ++j) {
            const int r = n - 1 - j;
            for (int t = -q; t <= q; ++t) Ab[(q + t) + (size_t)W * r] = s.clo_lhs[j][q - t];
        }
    // Coupling blocks AL[r,t] = lhs[q+r-t] (t >= r), CR[r,t] = lhs[t+q-r] (t <= r), 1-based.
    std::vector<double> AL((size_t)q * q, 0.0), CR((size_t)q * q, 0.0);
    if (!(rp.lo_closed || rp.fold_lo))
        for (int r = 1; r <= q; ++r) for (int t = r; t <= q; ++t) AL[(r - 1) + (size_t)q * (t - 1)] = s.lhs[q + r - t - 1];
    if (!(rp.hi_closed || rp.fold_hi))
        for (int r = 1; r <= q; ++r) for (int t = 1; t <= r; ++t) CR[(r - 1) + (size_t)q * (t - 1)] = s.lhs[t + q - r - 1];
    rp.bf.build(Ab, n, q);
    rp.V.assign((size_t)n * q, 0.0); rp.W.assign((size_t)n * q, 0.0);
    bool alz = true, crz = true;
    for (double v : AL) alz = alz && v == 0.0;
    for (double v : CR) crz = crz && v == 0.0;
    if (!alz)
        for (int t = 0; t < q; ++t) {
            for (int r = 0; r < q; ++r) rp.V[r + (size_t)n * t] = AL[r + (size_t)q * t];
            rp.bf.solve(&rp.V[(size_t)n * t], 1);
        }
    if (!crz)
        for (int t = 0; t < q; ++t) {
            for (int r = 0; r < q; ++r) rp.W[(n - q + r) + (size_t)n * t] = CR[r + (size_t)q * t];
            rp.bf.solve(&rp.W[(size_t)n * t], 1);
        }
    return true;
}

// Reduced matrix (src/tridiag.jl:100-123, src/banded.jl:136-169).
void build_reduced(DistSolver& ls) {
    const int q = ls.q, P = ls.P, m2 = 2 * q, N = m2 * P;
    std::vector<double> R((size_t)N * N, 0.0);
    auto Rat = [&](int r, int c) -> double& { return R[r + (size_t)N * c]; };
    for (int rk = 0; rk < P; ++rk) {
        const RankPart& rp = ls.parts[rk];
        const int n = rp.n;
        if (!ls.banded) {
            const double v1 = rp.V[0], vn = rp.V[n - 1], w1 = rp.W[0], wn = rp.W[n - 1];
            const int rlo = 2 * rk, rhi = 2 * rk + 1;
            Rat(rlo, rlo) += 1; Rat(rhi, rhi) += 1;
            const int cprev = 2 * jl_mod(rk - 1, P) + 1;
            const int cnext = 2 * jl_mod(rk + 1, P);
            Rat(rlo, cprev) += v1; Rat(rlo, cnext) += w1;
            Rat(rhi, cprev) += vn; Rat(rhi, cnext) += wn;
        } else {
            const int rh = m2 * rk, rt = m2 * rk + q;
            for (int r = 0; r < q; ++r) { Rat(rh + r, rh + r) += 1; Rat(rt + r, rt + r) += 1; }
            const int cprev = m2 * jl_mod(rk - 1, P) + q;
            const int cnext = m2 * jl_mod(rk + 1, P);
            for (int t = 0; t < q; ++t)
                for (int r = 0; r < q; ++r) {
                    Rat(rh + r, cprev + t) += rp.V[r + (size_t)n * t];
                    Rat(rt + r, cprev + t) += rp.V[(n - q + r) + (size_t)n * t];
                    Rat(rh + r, cnext + t) += rp.W[r + (size_t)n * t];
                    Rat(rt + r, cnext + t) += rp.W[(n - q + r) + (size_t)n * t];
                }
        }
    }
    ls.red.factor(R, N);
}

Plan* plan_create(const Decomp& D, const cles_scheme& s, int dim0, double h, int P, int lo_fold = 0, int hi_fold = 0) {
    const int n = D.nl[dim0];
    const int nc = s.nc, M = s.M, q = s.q;
    if (!D.active[dim0]) { set_err("dimension is collapsed"); return nullptr; }
    if (P < 1) P = 1;
    const int nmin = (q >= 2) ? std::max({2 * nc + 1, 2 * M + 1, 2 * q + 1}) : std::max(2 * nc + 1, 2 * M + 1);
    int nloc_min = n / P;
    if (nloc_min < nmin) {
        set_err("local extent " + std::to_string(nloc_min) + " along dim " + std::to_string(dim0 + 1) +
                " too small for scheme '" + s.name + "' (need >= " + std::to_string(nmin) + ")");
        return nullptr;
    }
    if (M > D.nh) { set_err("stencil half-width exceeds halo width"); return nullptr; }
    auto* p = new Plan();
    p->D = D; p->dim = dim0; p->n = n; p->scheme = s;
    p->lo_fold = D.closed(dim0) ? lo_fold : 0;
    p->hi_fold = D.closed(dim0) ? hi_fold : 0;
    p->lo_closed = D.closed(dim0) && !p->lo_fold;
    p->hi_closed = D.closed(dim0) && !p->hi_fold;
    p->lines = 1;
    for (int k = 0; k < 3; ++k) if (k != dim0) p->lines *= D.nl[k];
    const double hinv = 1.0 / h;
    const double sgn = s.symmetric ? 1.0 : -1.0;
    const double scale = s.symmetric ? 1.0 : hinv;
    p->a0 = s.a0;
    for (int m = 0; m < M; ++m) p->ci.push_back(s.coeffs[m] * scale);
    for (int j = 0; j < nc; ++j) {
        std::vector<double> lo, hi;
        for (int t = 0; t < s.clo_len[j]; ++t) { lo.push_back(s.clo_rhs[j][t] * scale); hi.push_back(s.clo_rhs[j][t] * (scale * sgn)); }
        p->clo.push_back(lo); p->chi.push_back(hi);
    }
    DistSolver& ls = p->ls;
    ls.n_global = n; ls.q = q; ls.P = P; ls.periodic = D.periodic[dim0]; ls.banded = (q >= 2);
    ls.hasred = (P > 1) || ls.periodic;
    ls.parts.resize(P);
    for (int r = 0; r < P; ++r) {
        RankPart& rp = ls.parts[r];
        local_range(n, P, r, &rp.n, &rp.off);
        rp.lo_closed = p->lo_closed && r == 0;
        rp.hi_closed = p->hi_closed && r == P - 1;
        rp.fold_lo = r == 0 ? p->lo_fold : 0;
        rp.fold_hi = r == P - 1 ? p->hi_fold : 0;
        if (!ls.banded) build_tri_part(s, rp);
        else if (!build_band_part(s, rp)) { delete p; return nullptr; }
    }
    if (ls.hasred) build_reduced(ls);
    return p;
}

// _fill_lines! / _fill_t! (src/operators.jl:113-174, :245-309) for one line;
// reads f through a strided pointer whose index 0 is local interior row 1.
inline void fill_line(const Plan& p, const double* fl, ptrdiff_t st, double* B, ptrdiff_t bst) {
    const int n = p.n, M = (int)p.ci.size(), nc = (int)p.clo.size();
    int i1 = 0, i2 = n - 1;
    if (p.lo_closed) {
        for (int jr = 0; jr < nc; ++jr) {
            const auto& rhs = p.clo[jr];
            double acc = 0.0;
            for (size_t k = 0; k < rhs.size(); ++k) acc += rhs[k] * fl[(ptrdiff_t)k * st];
            B[jr * bst] = acc;
        }
        i1 = nc;
    }
    if (p.hi_closed) {
        for (int jr = 0; jr < nc; ++jr) {
            const auto& rhs = p.chi[jr];
            double acc = 0.0;
            for (size_t k = 0; k < rhs.size(); ++k) acc += rhs[k] * fl[(ptrdiff_t)(n - 1 - (int)k) * st];
            B[(n - 1 - jr) * bst] = acc;
        }
        i2 = n - 1 - nc;
    }
    if (p.scheme.symmetric) {
        for (int i = i1; i <= i2; ++i) {
            double acc = p.a0 * fl[(ptrdiff_t)i * st];
            for (int m = 1; m <= M; ++m) acc += p.ci[m - 1] * (fl[(ptrdiff_t)(i + m) * st] + fl[(ptrdiff_t)(i - m) * st]);
            B[i * bst] = acc;
        }
    } else {
        for (int i = i1; i <= i2; ++i) {
            double acc = 0.0;
            for (int m = 1; m <= M; ++m) acc += p.ci[m - 1] * (fl[(ptrdiff_t)(i + m) * st] - fl[(ptrdiff_t)(i - m) * st]);
            B[i * bst] = acc;
        }
    }
}

// solve_lines! / solve_lines_t! for one full line B (n values, stride bst),
// emulating P ranks along it.
void solve_line(const Plan& p, double* B, ptrdiff_t bst, bool transposed) {
    const DistSolver& ls = p.ls;
    for (const RankPart& rp : ls.parts) ls.solve_local(rp, B + (ptrdiff_t)rp.off * bst, bst, transposed);
    if (!ls.hasred) return;
    const int q = ls.q, P = ls.P, m2 = 2 * q;
    std::vector<double> z((size_t)m2 * P);
    for (int rk = 0; rk < P; ++rk) {
        const RankPart& rp = ls.parts[rk];
        const double* Bl = B + (ptrdiff_t)rp.off * bst;
        for (int r = 0; r < q; ++r) {
            z[m2 * rk + r] = Bl[(ptrdiff_t)r * bst];
            z[m2 * rk + q + r] = Bl[(ptrdiff_t)(rp.n - q + r) * bst];
        }
    }
    ls.red.solve(z.data());
    for (int rk = 0; rk < P; ++rk) {
        const RankPart& rp = ls.parts[rk];
        double* Bl = B + (ptrdiff_t)rp.off * bst;
        const int n = rp.n;
        if (!ls.banded) {
            const int cprev = 2 * jl_mod(rk - 1, P) + 1;
            const int cnext = 2 * jl_mod(rk + 1, P);
            const double xl = z[cprev], xr = z[cnext];
            for (int i = 0; i < n; ++i) Bl[(ptrdiff_t)i * bst] -= rp.V[i] * xl + rp.W[i] * xr;
        } else {
            const int cprev = m2 * jl_mod(rk - 1, P) + q;
            const int cnext = m2 * jl_mod(rk + 1, P);
            if (!transposed) {
                for (int i = 0; i < n; ++i) {
                    double acc = 0.0;
                    for (int t = 0; t < q; ++t) acc += rp.V[i + (size_t)n * t] * z[cprev + t] + rp.W[i + (size_t)n * t] * z[cnext + t];
                    Bl[(ptrdiff_t)i * bst] -= acc;
                }
            } else {
                for (int i = 0; i < n; ++i)
                    for (int t = 0; t < q; ++t)
                        Bl[(ptrdiff_t)i * bst] -= rp.V[i + (size_t)n * t] * z[cprev + t] + rp.W[i + (size_t)n * t] * z[cnext + t];
            }
        }
    }
}

// apply_along! (src/operators.jl:199-215).  f must have current halos.
void apply_along(const Plan& p, double* out, const double* f) {
    const Decomp& D = p.D;
    const int d = p.dim, n = p.n;
    const int o1 = D.nhd[0], o2 = D.nhd[1], o3 = D.nhd[2];
    int od1, od2;
    if (d == 0) { od1 = 1; od2 = 2; } else if (d == 1) { od1 = 0; od2 = 2; } else { od1 = 0; od2 = 1; }
    const int n1 = D.nl[od1];
    const ptrdiff_t strides[3] = {1, (ptrdiff_t)D.full[0], (ptrdiff_t)D.full[0] * D.full[1]};
    const ptrdiff_t st = strides[d];
    const bool transposed = d > 0;
    const long work = (long)p.lines * n;
#pragma omp parallel if (work >= kThreadMinWork)
    {
        std::vector<double> B(n);
#pragma omp for schedule(static)
        for (int l = 0; l < p.lines; ++l) {
            const int jj = l % n1, kk = l / n1;
            int idx[3];
            idx[d] = 0; idx[od1] = jj; idx[od2] = kk;
            const size_t base = D.at(idx[0] + o1, idx[1] + o2, idx[2] + o3);
            fill_line(p, f + base, st, B.data(), 1);
            solve_line(p, B.data(), 1, transposed);
            for (int i = 0; i < n; ++i) out[base + (size_t)i * st] = B[i];
        }
    }
}

// -------------------------------------------------------------- the solver ---
struct Savepoint { std::vector<double> Q; double t; int64_t step; };

// Pairing of a folded dimension (PairSpec, src/folds.jl:50-60), one rank:
// every partner block is local.  pdim / revdim are 0-based, -1 = none.
struct PairSpec {
    int pdim = -1, revdim = -1;
};

// FoldSpec (src/folds.jl:62-75): folded ends, pairing, antipodal signs and
// the parity plans (index 0: sigma_g = +1, index 1: sigma_g = -1).
struct FoldSpec {
    int dim = 0;
    bool lo = false, hi = false;
    bool paired = false;
    PairSpec pair;
    int sigvel[3] = {1, 1, 1};
    std::vector<int> sigflux;
    std::unique_ptr<Plan> dp[2], fp[2];
};

struct Solver {
    cles_solver_desc desc;
    Decomp D;
    int Ns = 1, ncons = 5, i_mom[3], i_energy;
    double Rk[CLES_MAX_SPECIES], cvk[CLES_MAX_SPECIES], cpk[CLES_MAX_SPECIES];
    double h[3];
    std::unique_ptr<Plan> dplan[3], fplan[3];
    size_t fs;  // padded field size
    std::vector<double> Q, dQ, du;
    std::vector<double> rho, u, v, w, p, T, c, cp;
    std::vector<std::vector<double>> Y, D_art;
    std::vector<double> grad_u[3][3], grad_T[3];
    std::vector<std::vector<double>> grad_Y[3];
    std::vector<double> mu_art, beta_art, kappa_art, strain, sensor, sensor_sp, tmp_a, tmp_b;
    std::vector<double> flux[3][CLES_MAX_SPECIES + 4];
    // geometry (src/rhs.jl:53-55, src/metric.jl:109-140)
    int metric = CLES_METRIC_CARTESIAN;
    bool stretched[3] = {false, false, false};
    std::vector<double> st_x[3], st_m[3];   // stretch samples at the interior nodes
    double orig[3] = {0, 0, 0}, coord_shift[3] = {0, 0, 0};
    std::unique_ptr<FoldSpec> folds[3];
    std::vector<double> inv_J, area[3], inv_h[3], inv_r, cot_over_r, pairbuf, pairout;
    double t = 0.0, tstage = 0.0, dt_prev = 0.0, rate_prev = 0.0, cfl = 0.5;
    int64_t step = 0;
    bool switched[3][2] = {{false, false}, {false, false}, {false, false}};   // SwitchableBC state
    // DirichletBC(fun) / NSCBCInflowBC(target = fun): [dim][side][before/after]
    cles_face_fn ffn[3][2][2] = {};
    void* fuser[3][2][2] = {};

    // the condition a face acts as now (src/boundary.jl:170-183)
    int face_kind(int d, int s) const {
        return desc.bc_switchable[d][s] && switched[d][s] ? desc.bc_after[d][s] : desc.bc[d][s];
    }
    const cles_bc_params& face_params(int d, int s) const {
        return desc.bc_switchable[d][s] && switched[d][s] ? desc.bc_after_params[d][s] : desc.bc_params[d][s];
    }
    const double* face_state(int d, int s) const {
        return desc.bc_switchable[d][s] && switched[d][s] ? desc.bc_after_state[d][s] : desc.bc_state[d][s];
    }

    cles_face_fn face_fn(int d, int s, void** user) const {
        const int w = desc.bc_switchable[d][s] && switched[d][s] ? 1 : 0;
        *user = fuser[d][s][w];
        return ffn[d][s][w];
    }
    double* comp(std::vector<double>& A, int cidx) { return A.data() + fs * cidx; }
    double* vel(int j) { return j == 0 ? u.data() : j == 1 ? v.data() : w.data(); }
};

// ---- Nasa9Mixture (src/physics.jl:255-310, 402-570) ----
// cp/R and h/R of one interval; x^2, x^3, x^4 written as products.
double n9_cp_R(const cles_nasa9_interval& iv, double T) {
    const double* a = iv.a;
    const double T2 = T * T;
    return a[0] / T2 + a[1] / T + a[2] + a[3] * T + a[4] * T2 + a[5] * (T2 * T) + a[6] * (T2 * T2);
}
double n9_h_R(const cles_nasa9_interval& iv, double T) {
    const double* a = iv.a;
    const double T2 = T * T;
    return -a[0] / T + a[1] * std::log(T) + a[2] * T + a[3] * T2 / 2 + a[4] * (T2 * T) / 3 + a[5] * (T2 * T2) / 4 +
           a[6] * (T2 * T2 * T) / 5 + iv.b1;
}
// _nasa9_interval: the first interval whose Tmax >= T, else the last
const cles_nasa9_interval& n9_interval(const cles_solver_desc& d, int k, double T) {
    const int n = d.n_intervals[k];
    for (int i = 0; i < n - 1; ++i)
        if (T <= d.nasa9[k][i].Tmax) return d.nasa9[k][i];
    return d.nasa9[k][n - 1];
}
double n9_species_cp(const cles_solver_desc& d, int k, double T) { return d.R[k] * n9_cp_R(n9_interval(d, k, T), T); }
double n9_species_h(const cles_solver_desc& d, int k, double T) { return d.R[k] * n9_h_R(n9_interval(d, k, T), T); }
double n9_species_e(const cles_solver_desc& d, int k, double T) { return n9_species_h(d, k, T) - d.R[k] * T; }

// mixture_temperature (src/physics.jl:466-498)
double n9_temperature(const cles_solver_desc& d, double e, const double* Y) {
    const int n = d.n_species;
    double e0 = 0.0, cv0 = 0.0;
    for (int k = 0; k < n; ++k) {
        e0 += Y[k] * n9_species_e(d, k, d.T_guess);
        cv0 += Y[k] * (n9_species_cp(d, k, d.T_guess) - d.R[k]);
    }
    double T = d.T_guess;
    if (cv0 > 0) {
        const double x = d.T_guess + (e - e0) / cv0;
        T = x > 1e9 ? 1e9 : (x < 1e-3 ? 1e-3 : x);   // Julia clamp: NaN passes through
    }
    for (int it = 0; it < 30; ++it) {
        double f = -e, cvm = 0.0;
        for (int k = 0; k < n; ++k) {
            f += Y[k] * n9_species_e(d, k, T);
            cvm += Y[k] * (n9_species_cp(d, k, T) - d.R[k]);
        }
        if (!(cvm > 0)) break;
        const double dl = f / cvm;
        T = jl_max(T - dl, 0.25 * T);
        if (std::fabs(dl) <= 1e-14 * T) break;
    }
    return T;
}

// species_enthalpy of either equation of state
inline double species_h(const Solver& S, int k, double T) {
    return S.desc.eos == CLES_EOS_NASA9 ? n9_species_h(S.desc, k, T) : S.cpk[k] * T;
}

// _primitives!(::Nasa9Mixture) (src/physics.jl:501-570)
void primitives_nasa9(Solver& S) {
    const size_t fs = S.fs;
    const int Ns = S.Ns;
    const double* Q = S.Q.data();
#pragma omp parallel for schedule(static) if ((long)fs >= kThreadMinWork)
    for (size_t idx = 0; idx < fs; ++idx) {
        double rho = 0.0;
        for (int sp = 0; sp < Ns; ++sp) rho += Q[idx + fs * sp];
        if (rho > 0) {
            const double ri = 1 / rho;
            double Y[CLES_MAX_SPECIES];
            double Rm = 0.0;
            for (int sp = 0; sp < Ns; ++sp) {
                Y[sp] = Q[idx + fs * sp] * ri;
                S.Y[sp][idx] = Y[sp];
                Rm += Y[sp] * S.Rk[sp];
            }
            const double uu = Q[idx + fs * S.i_mom[0]] * ri;
            const double vv = Q[idx + fs * S.i_mom[1]] * ri;
            const double ww = Q[idx + fs * S.i_mom[2]] * ri;
            const double e = Q[idx + fs * S.i_energy] * ri - 0.5 * (uu * uu + vv * vv + ww * ww);
            const double Ti = n9_temperature(S.desc, e, Y);
            double cpm = 0.0;
            for (int sp = 0; sp < Ns; ++sp) cpm += Y[sp] * n9_species_cp(S.desc, sp, Ti);
            const double cvm = cpm - Rm;
            S.rho[idx] = rho; S.u[idx] = uu; S.v[idx] = vv; S.w[idx] = ww;
            S.p[idx] = rho * Rm * Ti; S.T[idx] = Ti;
            S.c[idx] = std::sqrt(jl_max((cpm / cvm) * Rm * Ti, 0.0));
            S.cp[idx] = cpm;
        } else {
            S.rho[idx] = 1; S.u[idx] = 0; S.v[idx] = 0; S.w[idx] = 0;
            S.p[idx] = 1; S.T[idx] = 1; S.c[idx] = 1; S.cp[idx] = 1;
            for (int sp = 0; sp < Ns; ++sp) S.Y[sp][idx] = sp == 0 ? 1.0 : 0.0;
        }
    }
}

// _primitives!(::IdealMixture) over the full padded arrays (src/physics.jl:604-653).
void primitives(Solver& S) {
    if (S.desc.eos == CLES_EOS_NASA9) { primitives_nasa9(S); return; }
    const size_t fs = S.fs;
    const int Ns = S.Ns;
    const double* Q = S.Q.data();
#pragma omp parallel for schedule(static) if ((long)fs >= kThreadMinWork)
    for (size_t idx = 0; idx < fs; ++idx) {
        double rho = 0.0;
        for (int sp = 0; sp < Ns; ++sp) rho += Q[idx + fs * sp];
        if (rho > 0) {
            const double ri = 1 / rho;
            double Rm = 0.0, cvm = 0.0;
            for (int sp = 0; sp < Ns; ++sp) {
                Rm += Q[idx + fs * sp] * S.Rk[sp];
                cvm += Q[idx + fs * sp] * S.cvk[sp];
                S.Y[sp][idx] = Q[idx + fs * sp] * ri;
            }
            Rm *= ri; cvm *= ri;
            const double uu = Q[idx + fs * S.i_mom[0]] * ri;
            const double vv = Q[idx + fs * S.i_mom[1]] * ri;
            const double ww = Q[idx + fs * S.i_mom[2]] * ri;
            const double e = Q[idx + fs * S.i_energy] * ri - 0.5 * (uu * uu + vv * vv + ww * ww);
            const double Ti = jl_max(e / cvm, 1e-300);
            const double pp = rho * Rm * Ti;
            const double gm = 1 + Rm / cvm;
            S.rho[idx] = rho; S.u[idx] = uu; S.v[idx] = vv; S.w[idx] = ww;
            S.p[idx] = pp; S.T[idx] = Ti;
            S.c[idx] = std::sqrt(gm * Rm * Ti);
            S.cp[idx] = cvm + Rm;
        } else {
            S.rho[idx] = 1; S.u[idx] = 0; S.v[idx] = 0; S.w[idx] = 0;
            S.p[idx] = 1; S.T[idx] = 1; S.c[idx] = 1; S.cp[idx] = 1;
            for (int sp = 0; sp < Ns; ++sp) S.Y[sp][idx] = sp == 0 ? 1.0 : 0.0;
        }
    }
}

void exchange_state(Solver& S) {
    // exchange_state! (src/halo.jl:93-99): per dim, every component.
    for (int d = 0; d < 3; ++d)
        for (int cc = 0; cc < S.ncons; ++cc) wrap_dim(S.D, S.comp(S.Q, cc), d);
}

template <class F>
void for_interior(const Decomp& D, F&& fn) {
    const int o1 = D.nhd[0], o2 = D.nhd[1], o3 = D.nhd[2];
    const long work = (long)D.nl[0] * D.nl[1] * D.nl[2];
#pragma omp parallel for collapse(2) schedule(static) if (work >= kThreadMinWork)
    for (int k = 0; k < D.nl[2]; ++k)
        for (int j = 0; j < D.nl[1]; ++j)
            for (int i = 0; i < D.nl[0]; ++i) fn(D.at(i + o1, j + o2, k + o3), i, j, k);
}

// ------------------------------------------------------------------ folds ---
// fold_fill! (src/folds.jl:83-124): mirror the halos beyond a folded end of
// dimension d with sign sig (half-offset mirror: ghost layer q <-> interior
// layer q), over the full padded extent of the other dimensions.
void fold_fill(const Decomp& D, double* f, int d, bool lo, bool hi, int sig) {
    const int pad = D.nhd[d], n = D.nl[d];
    const double sgn = (double)sig;
    const int o1 = d == 0 ? 1 : 0, o2 = d == 2 ? 1 : 2;
    for (int b = 0; b < D.full[o2]; ++b)
        for (int a = 0; a < D.full[o1]; ++a)
            for (int q = 1; q <= pad; ++q) {
                int g[3], c[3];
                g[o1] = c[o1] = a;
                g[o2] = c[o2] = b;
                if (lo) {
                    g[d] = pad - q;
                    c[d] = pad + q - 1;
                    f[D.at(g[0], g[1], g[2])] = sgn * f[D.at(c[0], c[1], c[2])];
                }
                if (hi) {
                    g[d] = pad + n + q - 1;
                    c[d] = pad + n - q;
                    f[D.at(g[0], g[1], g[2])] = sgn * f[D.at(c[0], c[1], c[2])];
                }
            }
}

// _pair_index (src/folds.jl:128-155), one rank: shift pdim by half its
// extent, reverse revdim.  c holds 0-based padded coordinates.
void pair_index(const Decomp& D, const PairSpec& pr, int c[3]) {
    if (pr.pdim >= 0) {
        const int pd = pr.pdim, half = D.nl[pd] / 2, Hp = D.nhd[pd];
        int v = c[pd] - Hp + 1;
        v = v <= half ? v + half : v - half;
        c[pd] = v - 1 + Hp;
    }
    if (pr.revdim >= 0) {
        const int rd = pr.revdim, Hr = D.nhd[rd];
        const int v = D.nl[rd] + 1 - (c[rd] - Hr + 1);
        c[rd] = v - 1 + Hr;
    }
}

inline int pair_dim(const PairSpec& pr) { return pr.pdim >= 0 ? pr.pdim : pr.revdim; }

// pair_forward! (src/folds.jl:162-215), on-rank butterfly: the lower half of
// the pairing dimension receives e, the partner slots o.
void pair_forward(Solver& S, double* w, const double* f, const FoldSpec& fold, int sig) {
    const Decomp& D = S.D;
    const double sf = (double)sig;
    const int sd = pair_dim(fold.pair), half = D.nl[sd] / 2;
    for (int k = 0; k < D.nl[2]; ++k)
        for (int j = 0; j < D.nl[1]; ++j)
            for (int i = 0; i < D.nl[0]; ++i) {
                int c[3] = {i + D.nhd[0], j + D.nhd[1], k + D.nhd[2]};
                const int v = (sd == 0 ? i : sd == 1 ? j : k) + 1;
                if (v > half) continue;
                const size_t I = D.at(c[0], c[1], c[2]);
                pair_index(D, fold.pair, c);
                const size_t Mx = D.at(c[0], c[1], c[2]);
                const double a = f[I], b = sf * f[Mx];
                w[I] = 0.5 * (a + b);
                w[Mx] = 0.5 * (a - b);
            }
}

// pair_backward! (src/folds.jl:217-262), on-rank inverse butterfly.
void pair_backward(Solver& S, double* out, const FoldSpec& fold, int sig) {
    const Decomp& D = S.D;
    const double sf = (double)sig;
    const int sd = pair_dim(fold.pair), half = D.nl[sd] / 2;
    for (int k = 0; k < D.nl[2]; ++k)
        for (int j = 0; j < D.nl[1]; ++j)
            for (int i = 0; i < D.nl[0]; ++i) {
                int c[3] = {i + D.nhd[0], j + D.nhd[1], k + D.nhd[2]};
                const int v = (sd == 0 ? i : sd == 1 ? j : k) + 1;
                if (v > half) continue;
                const size_t I = D.at(c[0], c[1], c[2]);
                pair_index(D, fold.pair, c);
                const size_t Mx = D.at(c[0], c[1], c[2]);
                const double Re = out[I], Ro = out[Mx];
                out[I] = Re + Ro;
                out[Mx] = sf * (Re - Ro);
            }
}

// _fold_plan / fold_apply! (src/folds.jl:271-322)
Plan& fold_plan(const FoldSpec& fold, int sig, bool isfilter) {
    const int sg = isfilter ? sig : -sig;
    return isfilter ? *fold.fp[sg > 0 ? 0 : 1] : *fold.dp[sg > 0 ? 0 : 1];
}
void fold_apply(Solver& S, double* out, double* f, const FoldSpec& fold, int sig, bool isfilter) {
    const Decomp& D = S.D;
    const int d = fold.dim;
    if (!fold.paired) {
        fold_fill(D, f, d, fold.lo, fold.hi, sig);
        apply_along(fold_plan(fold, sig, isfilter), out, f);
        return;
    }
    double* w = S.pairbuf.data();
    pair_forward(S, w, f, fold, sig);
    // exchange_dim_batch!([w], decomp, d): a folded dimension is closed, one rank
    fold_fill(D, w, d, fold.lo, fold.hi, sig);
    apply_along(fold_plan(fold, sig, isfilter), out, w);
    fold_fill(D, w, d, fold.lo, fold.hi, -1);
    apply_along(fold_plan(fold, -1, isfilter), S.pairout.data(), w);
    const int sd = pair_dim(fold.pair), half = D.nl[sd] / 2;
    for (int k = 0; k < D.nl[2]; ++k)
        for (int j = 0; j < D.nl[1]; ++j)
            for (int i = 0; i < D.nl[0]; ++i) {
                const int v = (sd == 0 ? i : sd == 1 ? j : k) + 1;
                if (v > half) {
                    const size_t I = D.at(i + D.nhd[0], j + D.nhd[1], k + D.nhd[2]);
                    out[I] = S.pairout[I];
                }
            }
    pair_backward(S, out, fold, sig);
}

// deriv_along! / filt_along! (src/rhs.jl:452-475): sig is the field's
// antipodal sign for the fold on d (ignored without one).
void deriv_along(Solver& S, double* out, double* f, int d, int sig = 1) {
    if (!S.folds[d]) apply_along(*S.dplan[d], out, f);
    else fold_apply(S, out, f, *S.folds[d], sig, false);
}
void filt_along(Solver& S, double* out, double* f, int d, int sig = 1) {
    if (!S.folds[d]) apply_along(*S.fplan[d], out, f);
    else fold_apply(S, out, f, *S.folds[d], sig, true);
}

// _scale_grad! (src/rhs.jl:477-483), over the full array
void scale_grad(Solver& S, std::vector<double>& g, int d) {
    const double* ih = S.inv_h[d].data();
    const size_t n = g.size();
#pragma omp parallel for schedule(static) if ((long)n >= kThreadMinWork)
    for (size_t I = 0; I < n; ++I) g[I] *= ih[I];
}

// vel_parity / cons_parity (src/rhs.jl:486-491, src/equations.jl:56-60)
int vel_parity(const Solver& S, int d, int j) { return S.folds[d] ? S.folds[d]->sigvel[j] : 1; }
int conserved_parity(const Solver& S, const int* sigvel, int c) {
    if (c < S.Ns) return 1;
    if (c == S.i_energy) return 1;
    return sigvel[c - S.Ns];
}
int cons_parity(const Solver& S, int d, int c) { return S.folds[d] ? conserved_parity(S, S.folds[d]->sigvel, c) : 1; }

// ---------------------------------------------------------------- metrics ---
// metric_correct_gradients! (src/metric.jl:177-221): curvature terms added to
// the 1/h-scaled coordinate derivatives.
void metric_correct_gradients(Solver& S) {
    if (S.metric == CLES_METRIC_CARTESIAN) return;
    auto& g = S.grad_u;
    for_interior(S.D, [&](size_t I, int, int, int) {
        const double ir = S.inv_r[I];
        if (S.metric == CLES_METRIC_CYLINDRICAL) {
            g[1][0][I] -= S.v[I] * ir;
            g[1][1][I] += S.u[I] * ir;
        } else {
            const double ctr = S.cot_over_r[I];
            const double ur = S.u[I], ut = S.v[I], up = S.w[I];
            g[1][0][I] -= ut * ir;
            g[1][1][I] += ur * ir;
            g[2][0][I] -= up * ir;
            g[2][1][I] -= up * ctr;
            g[2][2][I] += ur * ir + ut * ctr;
        }
    });
}

// _Pi (src/metric.jl:225-233): momentum flux tensor component (a, b), 0-based
double metric_Pi(const Solver& S, size_t I, int a, int b) {
    const auto& g = S.grad_u;
    const double mu = S.desc.mu0 + S.mu_art[I];
    const double be = S.beta_art[I];
    const double divu = g[0][0][I] + g[1][1][I] + g[2][2][I];
    const double tau = mu * (g[a][b][I] + g[b][a][I]) + (a == b ? (be - 2 * mu / 3) * divu : 0.0);
    const double uv[3] = {S.u[I], S.v[I], S.w[I]};
    return S.rho[I] * uv[a] * uv[b] + (a == b ? S.p[I] : 0.0) - tau;
}

// add_metric_sources! (src/metric.jl:235-269)
void add_metric_sources(Solver& S) {
    if (S.metric == CLES_METRIC_CARTESIAN) return;
    double* d1 = S.comp(S.dQ, S.i_mom[0]);
    double* d2 = S.comp(S.dQ, S.i_mom[1]);
    double* d3 = S.comp(S.dQ, S.i_mom[2]);
    for_interior(S.D, [&](size_t I, int, int, int) {
        const double ir = S.inv_r[I];
        if (S.metric == CLES_METRIC_CYLINDRICAL) {
            d1[I] += ir * metric_Pi(S, I, 1, 1);
            d2[I] -= ir * metric_Pi(S, I, 1, 0);
        } else {
            const double ctr = S.cot_over_r[I];
            const double Ptt = metric_Pi(S, I, 1, 1);
            const double Ppp = metric_Pi(S, I, 2, 2);
            d1[I] += ir * (Ptt + Ppp);
            d2[I] += -ir * metric_Pi(S, I, 1, 0) + ctr * Ppp;
            d3[I] += -ir * metric_Pi(S, I, 2, 0) - ctr * metric_Pi(S, I, 2, 1);
        }
    });
}

// curvature_rate (src/timestep.jl:185-200)
double curvature_rate(const Solver& S, size_t I, const double* uv) {
    if (S.metric == CLES_METRIC_CYLINDRICAL) return S.D.active[1] ? 0.0 : std::fabs(uv[1]) * S.inv_r[I];
    if (S.metric == CLES_METRIC_SPHERICAL) {
        double a = 0.0;
        if (!S.D.active[1]) a += std::fabs(uv[1]) * S.inv_r[I];
        if (!S.D.active[2]) a += std::fabs(uv[2]) * (S.inv_r[I] + std::fabs(S.cot_over_r[I]));
        return a;
    }
    return 0.0;
}

// _phys_and_jac (src/metric.jl:99-106): physical coordinate and mapping
// Jacobian of full-array index i0 (0-based) along d; halo layers beyond a
// stretched edge clamp to the edge node (their geometry is never read).
void phys_and_jac(const Solver& S, int d, int i0, double* x, double* m) {
    const double xi = S.orig[d] + S.coord_shift[d] + (double)(i0 - S.D.nhd[d]) * S.h[d];
    if (!S.stretched[d]) { *x = xi; *m = 1.0; return; }
    const int n = S.D.nl[d];
    const int i = std::min(std::max(i0 - S.D.nhd[d], 0), n - 1);
    *x = S.st_x[d][i];
    *m = S.st_m[d][i];
}

// gcl_cotr! (src/metric.jl:154-170): cot(theta)/r redefined as
// inv_J * D_theta(A_theta) with the theta-momentum flux's fold sign.
void gcl_cotr(Solver& S) {
    const int sig = S.folds[1] ? S.folds[1]->sigflux[S.i_mom[1]] : 1;
    deriv_along(S, S.tmp_a.data(), S.area[1].data(), 1, sig);
    for_interior(S.D, [&](size_t I, int, int, int) { S.cot_over_r[I] = S.inv_J[I] * S.tmp_a[I]; });
}

// init_geometry! (src/metric.jl:109-150) over the full padded extent
void init_geometry(Solver& S) {
    const Decomp& D = S.D;
    const double tiny = 1e-300;
    for (int k = 0; k < D.full[2]; ++k)
        for (int j = 0; j < D.full[1]; ++j)
            for (int i = 0; i < D.full[0]; ++i) {
                double x1, m1, x2, m2, x3, m3;
                phys_and_jac(S, 0, i, &x1, &m1);
                phys_and_jac(S, 1, j, &x2, &m2);
                phys_and_jac(S, 2, k, &x3, &m3);
                double h1 = 1.0, h2 = 1.0, h3 = 1.0;
                if (S.metric == CLES_METRIC_CYLINDRICAL) h2 = x1;
                else if (S.metric == CLES_METRIC_SPHERICAL) { h2 = x1; h3 = x1 * std::sin(x2); }
                h1 *= m1; h2 *= m2; h3 *= m3;
                h1 = jl_max(h1, tiny); h2 = jl_max(h2, tiny); h3 = jl_max(h3, tiny);
                const double J = h1 * h2 * h3;
                const size_t I = D.at(i, j, k);
                S.inv_J[I] = 1 / J;
                S.area[0][I] = J / h1;
                S.area[1][I] = J / h2;
                S.area[2][I] = J / h3;
                S.inv_h[0][I] = 1 / h1;
                S.inv_h[1][I] = 1 / h2;
                S.inv_h[2][I] = 1 / h3;
                if (S.metric == CLES_METRIC_CYLINDRICAL) {
                    S.inv_r[I] = 1 / jl_max(x1, tiny);
                } else if (S.metric == CLES_METRIC_SPHERICAL) {
                    S.inv_r[I] = 1 / jl_max(x1, tiny);
                    S.cot_over_r[I] = std::cos(x2) / jl_max(x1 * std::sin(x2), tiny);
                }
            }
    if (S.metric == CLES_METRIC_SPHERICAL && D.active[1]) gcl_cotr(S);
}

// compute_primitives_and_gradients! (src/rhs.jl:591-606)
void primitives_and_gradients(Solver& S, bool primitives_current) {
    if (!primitives_current) { exchange_state(S); primitives(S); }
    for (int jj = 0; jj < 3; ++jj)
        for (int d = 0; d < 3; ++d) {
            if (S.D.active[d]) {
                deriv_along(S, S.grad_u[d][jj].data(), S.vel(jj), d, vel_parity(S, d, jj));
                scale_grad(S, S.grad_u[d][jj], d);
            } else {
                std::fill(S.grad_u[d][jj].begin(), S.grad_u[d][jj].end(), 0.0);
            }
        }
    metric_correct_gradients(S);
}

// delta4_sum! (src/artificial.jl:67-94)
void delta4_sum(Solver& S, std::vector<double>& out, const double* f, int wpow) {
    const Decomp& D = S.D;
    std::fill(out.begin(), out.end(), 0.0);
    static const double D4[5] = {1.0, -4.0, 6.0, -4.0, 1.0};
    for (int d = 0; d < 3; ++d) {
        if (!D.active[d]) continue;
        const double wd = wpow == 2 ? S.h[d] * S.h[d] : S.h[d];
        const int nd = D.nl[d];
        const int lomin = D.closed(d) ? 1 : -1;
        const int himax = D.closed(d) ? nd : nd + 2;
        const ptrdiff_t st = d == 0 ? 1 : d == 1 ? (ptrdiff_t)D.full[0] : (ptrdiff_t)D.full[0] * D.full[1];
        double* o = out.data();
        for_interior(D, [&](size_t I, int i, int j, int k) {
            const int il = (d == 0 ? i : d == 1 ? j : k) + 1;
            double acc = 0.0;
            for (int m = -2; m <= 2; ++m) {
                const int ilm = std::min(std::max(il + m, lomin), himax);
                acc += D4[m + 2] * f[(ptrdiff_t)I + (ptrdiff_t)(ilm - il) * st];
            }
            o[I] += wd * std::fabs(acc);
        });
    }
}

// smooth! (src/artificial.jl:98-111)
void smooth(Solver& S, double* f) {
    for (int d = 0; d < 3; ++d) {
        if (!S.D.active[d]) continue;
        wrap_dim(S.D, f, d);
        filt_along(S, S.tmp_a.data(), f, d, 1);
        copy_interior(S.D, f, S.tmp_a.data());
    }
}

const double DUCROS_EPS = 1e-32;
inline double compression_switch(Solver& S, size_t I) {
    auto g = [&](int d, int j) { return S.grad_u[d][j][I]; };
    const double div = g(0, 0) + g(1, 1) + g(2, 2);
    if (!(div < 0)) return 0.0;
    const double w1 = g(1, 2) - g(2, 1);
    const double w2 = g(2, 0) - g(0, 2);
    const double w3 = g(0, 1) - g(1, 0);
    return div * div / (div * div + w1 * w1 + w2 * w2 + w3 * w3 + DUCROS_EPS);
}

// compute_artificial! (src/artificial.jl:261-359)
void compute_artificial(Solver& S) {
    const cles_solver_desc& A = S.desc;
    if (!A.art_enabled) return;
    const Decomp& D = S.D;
    const double C_mu = A.C_mu, C_beta = A.C_beta, C_kappa = A.C_kappa, C_D = A.C_D;
    for_interior(D, [&](size_t I, int, int, int) {
        double ss = 0.0;
        for (int b = 0; b < 3; ++b)
            for (int a = 0; a < 3; ++a) {
                const double Sab = 0.5 * (S.grad_u[a][b][I] + S.grad_u[b][a][I]);
                ss += Sab * Sab;
            }
        S.strain[I] = std::sqrt(ss);
    });
    exchange_halos(D, S.strain.data());
    delta4_sum(S, S.sensor, S.strain.data(), 2);
    smooth(S, S.sensor.data());
    for_interior(D, [&](size_t I, int, int, int) {
        const double rs = S.rho[I] * jl_max(S.sensor[I], 0.0);
        S.mu_art[I] = C_mu * rs;
        S.beta_art[I] = C_beta * rs;
    });
    if (A.beta_sensor == CLES_BETA_GATED_STRAIN) {
        for_interior(D, [&](size_t I, int, int, int) { S.beta_art[I] *= compression_switch(S, I); });
    } else if (A.beta_sensor == CLES_BETA_DILATATION) {
        for_interior(D, [&](size_t I, int, int, int) {
            S.tmp_a[I] = S.grad_u[0][0][I] + S.grad_u[1][1][I] + S.grad_u[2][2][I];
            S.tmp_b[I] = compression_switch(S, I);
        });
        exchange_halos(D, S.tmp_a.data());
        delta4_sum(S, S.sensor, S.tmp_a.data(), 2);
        smooth(S, S.sensor.data());
        for_interior(D, [&](size_t I, int, int, int) {
            S.beta_art[I] = C_beta * S.rho[I] * jl_max(S.sensor[I], 0.0) * S.tmp_b[I];
        });
    }
    // internal energy over the full padded array
    {
        const size_t fs = S.fs;
        const double* Q = S.Q.data();
        const int m1 = S.i_mom[0], m2 = S.i_mom[1], m3 = S.i_mom[2], ie = S.i_energy;
#pragma omp parallel for schedule(static) if ((long)fs >= kThreadMinWork)
        for (size_t I = 0; I < fs; ++I) {
            const double r = jl_max(S.rho[I], 1e-300);
            const double q1 = Q[I + fs * m1], q2 = Q[I + fs * m2], q3 = Q[I + fs * m3];
            const double ke = 0.5 * (q1 * q1 + q2 * q2 + q3 * q3) / r;
            S.tmp_a[I] = (Q[I + fs * ie] - ke) / r;
        }
    }
    exchange_halos(D, S.tmp_a.data());
    delta4_sum(S, S.sensor, S.tmp_a.data(), 1);
    smooth(S, S.sensor.data());
    const double eps = std::numeric_limits<double>::epsilon();
    for_interior(D, [&](size_t I, int, int, int) {
        const double scale = S.rho[I] * S.c[I] / jl_max(S.T[I], eps);
        S.kappa_art[I] = C_kappa * scale * jl_max(S.sensor[I], 0.0);
    });
    if (S.Ns > 1) {
        for (int sp = 0; sp < S.Ns; ++sp) {
            delta4_sum(S, S.sensor_sp, S.Y[sp].data(), 1);
            smooth(S, S.sensor_sp.data());
            for_interior(D, [&](size_t I, int, int, int) {
                S.D_art[sp][I] = C_D * S.c[I] * jl_max(S.sensor_sp[I], 0.0);
            });
        }
    }
}

// _assemble_fluxes! (src/rhs.jl:495-556)
void assemble_fluxes(Solver& S) {
    const cles_solver_desc& A = S.desc;
    const double mu0 = A.mu0, Pr = A.Pr, Sc = A.Sc;
    const int Ns = S.Ns, m1 = S.i_mom[0], m2 = S.i_mom[1], m3 = S.i_mom[2], ie = S.i_energy;
    const size_t fs = S.fs;
    for_interior(S.D, [&](size_t I, int, int, int) {
        auto g = [&](int d, int j) { return S.grad_u[d][j][I]; };
        const double r = S.rho[I];
        const double uv[3] = {S.u[I], S.v[I], S.w[I]};
        const double pp = S.p[I], Tp = S.T[I], E = S.Q[I + fs * ie];
        const double mu = mu0 + S.mu_art[I];
        const double be = S.beta_art[I];
        const double ka = mu0 * S.cp[I] / Pr + S.kappa_art[I];
        const double D0 = mu0 / (Sc * r);
        const double divu = g(0, 0) + g(1, 1) + g(2, 2);
        const double t11 = mu * (2 * g(0, 0) - (2.0 / 3.0) * divu) + be * divu;
        const double t22 = mu * (2 * g(1, 1) - (2.0 / 3.0) * divu) + be * divu;
        const double t33 = mu * (2 * g(2, 2) - (2.0 / 3.0) * divu) + be * divu;
        const double t12 = mu * (g(0, 1) + g(1, 0));
        const double t13 = mu * (g(0, 2) + g(2, 0));
        const double t23 = mu * (g(1, 2) + g(2, 1));
        const double tau[3][3] = {{t11, t12, t13}, {t12, t22, t23}, {t13, t23, t33}};
        for (int d = 0; d < 3; ++d) {
            const double ud = uv[d];
            const double* td = tau[d];
            double Vc = 0.0;
            for (int sp = 0; sp < Ns; ++sp) Vc += (D0 + S.D_art[sp][I]) * S.grad_Y[d][sp][I];
            double hdiff = 0.0;
            for (int sp = 0; sp < Ns; ++sp) {
                const double Dk = D0 + S.D_art[sp][I];
                const double Jkd = r * (-Dk * S.grad_Y[d][sp][I] + S.Y[sp][I] * Vc);
                S.flux[d][sp][I] = r * S.Y[sp][I] * ud + Jkd;
                hdiff += species_h(S, sp, Tp) * Jkd;
            }
            S.flux[d][m1][I] = r * ud * uv[0] + (d == 0 ? pp : 0.0) - td[0];
            S.flux[d][m2][I] = r * ud * uv[1] + (d == 1 ? pp : 0.0) - td[1];
            S.flux[d][m3][I] = r * ud * uv[2] + (d == 2 ? pp : 0.0) - td[2];
            S.flux[d][ie][I] = (E + pp) * ud - (uv[0] * td[0] + uv[1] * td[1] + uv[2] * td[2]) - ka * S.grad_T[d][I] + hdiff;
        }
    });
}

// Physical coordinate of interior node i along e (global_xcoord, src/rhs.jl:331-335).
double node_coord(const Solver& S, int e, int i) {
    if (S.stretched[e]) return S.st_x[e][(size_t)i];
    return S.orig[e] + S.coord_shift[e] + (double)i * S.h[e];
}

// A face function evaluated at the stage time for the nodes of face (d, side)
// in wall-plane order: nvals values per node, [value][node].
std::vector<double> eval_face(const Solver& S, int d, int side, int nvals) {
    void* user = nullptr;
    const cles_face_fn fn = S.face_fn(d, side, &user);
    const int o1 = d == 0 ? 1 : 0, o2 = d == 2 ? 1 : 2;
    const int64_t np = (int64_t)S.D.nl[o1] * S.D.nl[o2];
    std::vector<double> x[3];
    for (int e = 0; e < 3; ++e) x[e].resize((size_t)np);
    for (int64_t t = 0; t < np; ++t) {
        int c[3];
        c[o1] = (int)(t % S.D.nl[o1]);
        c[o2] = (int)(t / S.D.nl[o1]);
        c[d] = side == 0 ? 0 : S.D.nl[d] - 1;
        for (int e = 0; e < 3; ++e) x[e][(size_t)t] = node_coord(S, e, c[e]);
    }
    std::vector<double> out((size_t)(np * nvals), std::numeric_limits<double>::quiet_NaN());
    fn(user, d, side, S.tstage, np, x[0].data(), x[1].data(), x[2].data(), out.data());
    return out;
}

// Visit the interior points of the wall plane of (d, side).
template <class Fn>
void for_wallplane(const Decomp& D, int d, int side, Fn&& fn) {
    const int wall = side == 0 ? 0 : D.nl[d] - 1;
    int lo[3], hi[3];
    for (int k = 0; k < 3; ++k) { lo[k] = 0; hi[k] = D.nl[k]; }
    lo[d] = wall; hi[d] = wall + 1;
    for (int k = lo[2]; k < hi[2]; ++k)
        for (int j = lo[1]; j < hi[1]; ++j)
            for (int i = lo[0]; i < hi[0]; ++i) fn(D.at(i + D.nhd[0], j + D.nhd[1], k + D.nhd[2]));
}

// eos_phi / eos_dphi_dY (src/physics.jl:142-152, 457-470); cv_k at T
double eos_phi(double rho, double p, double T, double cp) {
    const double Rm = p / (rho * T);
    return cp / Rm - 1;
}
double eos_dphi_dY(const Solver& S, int k, double rho, double p, double T, double cp) {
    const double Rm = p / (rho * T);
    const double cvm = cp - Rm;
    const double cvk = S.desc.eos == CLES_EOS_NASA9 ? n9_species_cp(S.desc, k, T) - S.Rk[k] : S.cvk[k];
    return (cvk * Rm - S.Rk[k] * cvm) / (Rm * Rm);
}

// correct_rhs!(::NSCBCOutflowBC) (src/nscbc.jl:59-157), Cartesian (inv_h = 1)
void nscbc_outflow(Solver& S, int d, int side) {
    const cles_bc_params& bc = S.face_params(d, side);
    deriv_along(S, S.tmp_a.data(), S.p.data(), d);
    const int t1 = d == 0 ? 1 : 0, t2 = d == 2 ? 1 : 2;
    const bool act1 = S.D.active[t1], act2 = S.D.active[t2];
    if (act1) deriv_along(S, S.tmp_b.data(), S.p.data(), t1);
    if (act2) deriv_along(S, S.sensor_sp.data(), S.p.data(), t2);
    const double Lref = bc.Lref > 0 ? bc.Lref : S.desc.L[d];
    const size_t fs = S.fs;
    const double sgn = side == 1 ? -1.0 : 1.0;
    for_wallplane(S.D, d, side, [&](size_t I) {
        const double rho = S.rho[I], c = S.c[I], p = S.p[I];
        const double uv[3] = {S.u[I], S.v[I], S.w[I]};
        const double un = uv[d];
        const double Ma = std::fabs(un) / c;
        if (!(Ma < 1)) return;
        const double dpn = S.inv_h[d][I] * S.tmp_a[I];
        const double dun = S.grad_u[d][d][I];
        const double Lcomp = side == 1 ? (un - c) * (dpn - rho * c * dun) : (un + c) * (dpn + rho * c * dun);
        double tin = 0.0;
        if (act1) {
            const double ut = uv[t1];
            tin += ut * S.inv_h[t1][I] * S.tmp_b[I] + rho * c * c * S.grad_u[t1][t1][I] + sgn * rho * c * ut * S.grad_u[t1][d][I];
        }
        if (act2) {
            const double ut = uv[t2];
            tin += ut * S.inv_h[t2][I] * S.sensor_sp[I] + rho * c * c * S.grad_u[t2][t2][I] + sgn * rho * c * ut * S.grad_u[t2][d][I];
        }
        const double bt = bc.beta_t < 0 ? Ma : bc.beta_t;
        const double K = bc.sigma * (1 - Ma * Ma) * c / Lref;
        const double dL = K * (p - bc.pinf) - bt * tin - Lcomp;
        const double d1 = dL / (2 * c * c), d2 = dL / 2, d3 = sgn * dL / (2 * rho * c);
        const double phi = eos_phi(rho, p, S.T[I], S.cp[I]);
        const double ke = 0.5 * (uv[0] * uv[0] + uv[1] * uv[1] + uv[2] * uv[2]);
        for (int k = 0; k < S.Ns; ++k) S.dQ[I + fs * k] -= S.Y[k][I] * d1;
        for (int a = 0; a < 3; ++a) S.dQ[I + fs * S.i_mom[a]] -= uv[a] * d1 + (a == d ? rho * d3 : 0.0);
        S.dQ[I + fs * S.i_energy] -= ke * d1 + phi * d2 + rho * un * d3;
    });
}

// correct_rhs!(::NSCBCInflowBC) (src/nscbc.jl:220-307): constant targets, or
// the stage-time values of the target function per node
void nscbc_inflow(Solver& S, int d, int side) {
    const cles_bc_params& bc = S.face_params(d, side);
    void* fu = nullptr;
    std::vector<double> tv;
    int64_t tnp = 0, tp = 0;
    if (S.face_fn(d, side, &fu)) {
        tv = eval_face(S, d, side, 4 + S.Ns);
        tnp = (int64_t)(tv.size() / (4 + S.Ns));
    }
    deriv_along(S, S.tmp_a.data(), S.p.data(), d);
    deriv_along(S, S.tmp_b.data(), S.rho.data(), d);
    const double Lref = bc.Lref > 0 ? bc.Lref : S.desc.L[d];
    const int t1 = d == 0 ? 1 : 0, t2 = d == 2 ? 1 : 2;
    const size_t fs = S.fs;
    const bool low = side == 0;
    for_wallplane(S.D, d, side, [&](size_t I) {
        const int64_t q = tp++;
        double uT[3] = {bc.u[0], bc.u[1], bc.u[2]}, TT = bc.T_ion, YT[CLES_MAX_SPECIES];
        for (int k = 0; k < S.Ns; ++k) YT[k] = bc.Y[k];
        if (tnp) {
            for (int a = 0; a < 3; ++a) uT[a] = tv[(size_t)(a * tnp + q)];
            TT = tv[(size_t)(3 * tnp + q)];
            for (int k = 0; k < S.Ns; ++k) YT[k] = tv[(size_t)((4 + k) * tnp + q)];
        }
        const double rho = S.rho[I], c = S.c[I], p = S.p[I], Tp = S.T[I];
        const double uv[3] = {S.u[I], S.v[I], S.w[I]};
        const double un = uv[d];
        const double Ma = std::fabs(un) / c;
        if (!(Ma < 1)) return;
        const double dpn = S.inv_h[d][I] * S.tmp_a[I], drn = S.inv_h[d][I] * S.tmp_b[I], dun = S.grad_u[d][d][I];
        const double K = c / Lref;
        const double L1c = (un - c) * (dpn - rho * c * dun);
        const double L5c = (un + c) * (dpn + rho * c * dun);
        const double L2c = un * (c * c * drn - dpn);
        const double rel = bc.eta_u * rho * c * c * (1 - Ma * Ma) / Lref * (un - uT[d]);
        const double dL1 = low ? 0.0 : (-rel - L1c);
        const double dL5 = low ? (rel - L5c) : 0.0;
        const double dL2 = bc.eta_T * rho * (c * c * c) * (TT - Tp) / (Lref * Tp) - L2c;
        const double d1 = dL2 / (c * c) + (dL5 + dL1) / (2 * c * c);
        const double d2 = (dL5 + dL1) / 2;
        const double d3 = (dL5 - dL1) / (2 * rho * c);
        const double d4 = bc.eta_t * K * (uv[t1] - uT[t1]) - un * S.grad_u[d][t1][I];
        const double d5 = bc.eta_t * K * (uv[t2] - uT[t2]) - un * S.grad_u[d][t2][I];
        const double cpm = S.cp[I];
        const double phi = eos_phi(rho, p, Tp, cpm);
        const double ke = 0.5 * (uv[0] * uv[0] + uv[1] * uv[1] + uv[2] * uv[2]);
        double sphiY = 0.0;
        for (int k = 0; k < S.Ns; ++k) {
            const double dLs = bc.eta_Y * K * (S.Y[k][I] - YT[k]) - un * S.grad_Y[d][k][I];
            S.dQ[I + fs * k] -= S.Y[k][I] * d1 + rho * dLs;
            sphiY += eos_dphi_dY(S, k, rho, p, Tp, cpm) * dLs;
        }
        for (int a = 0; a < 3; ++a) {
            const double extra = a == d ? rho * d3 : (a == t1 ? rho * d4 : rho * d5);
            S.dQ[I + fs * S.i_mom[a]] -= uv[a] * d1 + extra;
        }
        S.dQ[I + fs * S.i_energy] -= ke * d1 + phi * d2 + p * sphiY + rho * (un * d3 + uv[t1] * d4 + uv[t2] * d5);
    });
}

// compute_rhs! (src/rhs.jl:624-694), unitgeom branch.
void compute_rhs(Solver& S, bool primitives_current) {
    const Decomp& D = S.D;
    primitives_and_gradients(S, primitives_current);
    compute_artificial(S);
    for (int d = 0; d < 3; ++d) {
        if (!D.active[d]) continue;
        deriv_along(S, S.grad_T[d].data(), S.T.data(), d, 1);
        scale_grad(S, S.grad_T[d], d);
        for (int sp = 0; sp < S.Ns; ++sp) {
            deriv_along(S, S.grad_Y[d][sp].data(), S.Y[sp].data(), d, 1);
            scale_grad(S, S.grad_Y[d][sp], d);
        }
    }
    assemble_fluxes(S);
    for (int d = 0; d < 3; ++d)
        for (int cc = 0; cc < S.ncons; ++cc) wrap_dim(D, S.flux[d][cc].data(), d);
    // unit geometry (Cartesian, unstretched): A_d = inv_J = 1 and the general
    // path's products are skipped (src/rhs.jl:643-649)
    bool unitgeom = S.metric == CLES_METRIC_CARTESIAN;
    for (int d = 0; d < 3; ++d) unitgeom = unitgeom && !S.stretched[d];
    for (int cc = 0; cc < S.ncons; ++cc) {
        double* dq = S.comp(S.dQ, cc);
        for_interior(D, [&](size_t I, int, int, int) { dq[I] = 0; });
        for (int d = 0; d < 3; ++d) {
            if (!D.active[d]) continue;
            const int sig = S.folds[d] ? S.folds[d]->sigflux[cc] : 1;
            if (unitgeom) {
                deriv_along(S, S.tmp_a.data(), S.flux[d][cc].data(), d, sig);
                for_interior(D, [&](size_t I, int, int, int) { dq[I] -= S.tmp_a[I]; });
            } else {
                // tmp_b = A_d F_d over the full array, then dQ -= inv_J D_d(tmp_b)
                const double* Ad = S.area[d].data();
                const double* Fd = S.flux[d][cc].data();
                for (size_t I = 0; I < S.fs; ++I) S.tmp_b[I] = Ad[I] * Fd[I];
                deriv_along(S, S.tmp_a.data(), S.tmp_b.data(), d, sig);
                for_interior(D, [&](size_t I, int, int, int) { dq[I] -= S.inv_J[I] * S.tmp_a[I]; });
            }
        }
    }
    add_metric_sources(S);
    for (int d = 0; d < 3; ++d)
        for (int side = 0; side < 2; ++side) {
            if (!D.active[d]) continue;
            const int bc = S.face_kind(d, side);
            if (bc == CLES_BC_NSCBC_OUTFLOW) nscbc_outflow(S, d, side);
            else if (bc == CLES_BC_NSCBC_INFLOW) nscbc_inflow(S, d, side);
        }
    // add_sources! (src/sources.jl:42-82): every ConstantBodyForce in order
    const size_t fs = S.fs;
    const int m1 = S.i_mom[0], m2 = S.i_mom[1], m3 = S.i_mom[2], ie = S.i_energy;
    for (int f = 0; f < S.desc.n_body_forces; ++f) {
        const double g1 = S.desc.body_force[f][0], g2 = S.desc.body_force[f][1], g3 = S.desc.body_force[f][2];
        for_interior(D, [&](size_t I, int, int, int) {
            double rho = 0.0;
            for (int sp = 0; sp < S.Ns; ++sp) rho += S.Q[I + fs * sp];
            S.dQ[I + fs * m1] += rho * g1;
            S.dQ[I + fs * m2] += rho * g2;
            S.dQ[I + fs * m3] += rho * g3;
            S.dQ[I + fs * ie] += S.Q[I + fs * m1] * g1 + S.Q[I + fs * m2] * g2 + S.Q[I + fs * m3] * g3;
        });
    }
}

// enforce! for SlipWallBC (src/boundary.jl:232-243) and DirichletBC, with a
// constant state or the stage-time state of its function (src/problem.jl:194-207).
void apply_bcs(Solver& S) {
    const Decomp& D = S.D;
    const size_t fs = S.fs;
    for (int d = 0; d < 3; ++d)
        for (int side = 0; side < 2; ++side) {
            if (!D.active[d]) continue;
            const int bc = S.face_kind(d, side);
            if (bc == CLES_BC_PERIODIC || bc == CLES_BC_NSCBC_OUTFLOW || bc == CLES_BC_NSCBC_INFLOW) continue;
            if (bc == CLES_BC_AXIS || bc == CLES_BC_ORIGIN || bc == CLES_BC_POLE) continue;   // src/boundary.jl:173-175
            const double* bstate = S.face_state(d, side);
            const double Twall = S.face_params(d, side).Twall;
            void* fu = nullptr;
            std::vector<double> fvals;
            int64_t fp = 0, fnp = 0;
            if (bc == CLES_BC_DIRICHLET && S.face_fn(d, side, &fu)) {
                fvals = eval_face(S, d, side, S.ncons);
                fnp = (int64_t)(fvals.size() / S.ncons);
            }
            int shift[3] = {0, 0, 0};
            shift[d] = side == 0 ? 1 : -1;
            const long sh = (long)D.at(D.nhd[0] + shift[0], D.nhd[1] + shift[1], D.nhd[2] + shift[2]) -
                            (long)D.at(D.nhd[0], D.nhd[1], D.nhd[2]);
            const int wall = side == 0 ? 0 : D.nl[d] - 1;
            int lo[3], hi[3];
            for (int k = 0; k < 3; ++k) { lo[k] = 0; hi[k] = D.nl[k]; }
            lo[d] = wall; hi[d] = wall + 1;
            for (int k = lo[2]; k < hi[2]; ++k)
                for (int j = lo[1]; j < hi[1]; ++j)
                    for (int i = lo[0]; i < hi[0]; ++i) {
                        const size_t I = D.at(i + D.nhd[0], j + D.nhd[1], k + D.nhd[2]);
                        if (bc == CLES_BC_SLIPWALL) {
                            double r = 0.0;
                            for (int sp = 0; sp < S.Ns; ++sp) r += S.Q[I + fs * sp];
                            const int mc = S.i_mom[d];
                            const double mn = S.Q[I + fs * mc];
                            S.Q[I + fs * S.i_energy] -= 0.5 * mn * mn / r;
                            S.Q[I + fs * mc] = 0;
                        } else if (bc == CLES_BC_DIRICHLET) {
                            if (fnp) {
                                for (int cc = 0; cc < S.ncons; ++cc) S.Q[I + fs * cc] = fvals[(size_t)(cc * fnp + fp)];
                                ++fp;
                            } else {
                                for (int cc = 0; cc < S.ncons; ++cc) S.Q[I + fs * cc] = bstate[cc];
                            }
                        } else if (bc == CLES_BC_NOSLIP_WALL) {
                            // enforce!(::NoSlipWallBC) (src/boundary.jl:245-265)
                            double r = 0.0;
                            for (int sp = 0; sp < S.Ns; ++sp) r += S.Q[I + fs * sp];
                            const double q1 = S.Q[I + fs * S.i_mom[0]], q2 = S.Q[I + fs * S.i_mom[1]],
                                         q3 = S.Q[I + fs * S.i_mom[2]];
                            const double ke = 0.5 * (q1 * q1 + q2 * q2 + q3 * q3) / r;
                            S.Q[I + fs * S.i_energy] -= ke;
                            for (int a = 0; a < 3; ++a) S.Q[I + fs * S.i_mom[a]] = 0;
                            if (!std::isnan(Twall)) {
                                // wall_internal_energy (src/boundary.jl:194-211)
                                double re = 0.0;
                                if (S.desc.eos == CLES_EOS_NASA9) {
                                    for (int sp = 0; sp < S.Ns; ++sp)
                                        re += S.Q[I + fs * sp] * n9_species_e(S.desc, sp, Twall);
                                } else {
                                    for (int sp = 0; sp < S.Ns; ++sp) re += S.Q[I + fs * sp] * S.cvk[sp];
                                    re *= Twall;
                                }
                                S.Q[I + fs * S.i_energy] = re;
                            }
                        } else if (bc == CLES_BC_EXTRAPOLATION) {
                            // enforce!(::ExtrapolationBC) (src/boundary.jl:267-278)
                            for (int cc = 0; cc < S.ncons; ++cc) S.Q[I + fs * cc] = S.Q[(size_t)((long)I + sh) + fs * cc];
                        }
                    }
        }
}

const double RKA[5] = {0.0, -567301805773.0 / 1357537059087.0, -2404267990393.0 / 2016746695238.0,
                       -3550918686646.0 / 2091501179385.0, -1275806237668.0 / 842570457699.0};
const double RKB[5] = {1432997174477.0 / 9575080441755.0, 5161836677717.0 / 13612068292357.0,
                       1720146321549.0 / 2090206949498.0, 3134564353537.0 / 4481467310338.0,
                       2277821191437.0 / 14882151754819.0};
const double RKC[5] = {0.0, 1432997174477.0 / 9575080441755.0, 2526269341429.0 / 6820363962896.0,
                       2006345519317.0 / 3224310063776.0, 2802321613138.0 / 2924317926251.0};

// step! (src/timestep.jl:72-99)
void step(Solver& S, double dt, bool prepared) {
    for (int stage = 0; stage < 5; ++stage) {
        S.tstage = S.t + RKC[stage] * dt;
        const bool first_prepared = prepared && stage == 0;
        if (!first_prepared) apply_bcs(S);
        compute_rhs(S, first_prepared);
        const double A = RKA[stage], B = RKB[stage];
        for (int cc = 0; cc < S.ncons; ++cc) {
            double* du = S.comp(S.du, cc);
            double* dq = S.comp(S.dQ, cc);
            double* q = S.comp(S.Q, cc);
            for_interior(S.D, [&](size_t I, int, int, int) {
                const double vv = A * du[I] + dt * dq[I];
                du[I] = vv;
                q[I] += B * vv;
            });
        }
    }
    S.tstage = S.t + dt;
    apply_bcs(S);
}

// max_rate (src/timestep.jl:125-175)
void max_rate(Solver& S, double* rate_out, double* rho_min_out) {
    exchange_state(S);
    primitives(S);
    const Decomp& D = S.D;
    const cles_solver_desc& A = S.desc;
    const double mu0 = A.mu0, Pr = A.Pr, Sc = A.Sc;
    const size_t fs = S.fs;
    double rate = 0.0, rmin = std::numeric_limits<double>::infinity();
    const int o1 = D.nhd[0], o2 = D.nhd[1], o3 = D.nhd[2];
    for (int k = 0; k < D.nl[2]; ++k)
        for (int j = 0; j < D.nl[1]; ++j)
            for (int i = 0; i < D.nl[0]; ++i) {
                const size_t I = D.at(i + o1, j + o2, k + o3);
                double rq = 0.0;
                for (int sp = 0; sp < S.Ns; ++sp) rq += S.Q[I + fs * sp];
                rmin = jl_min(rmin, rq);
                const double r = S.rho[I];
                const double ri = 1 / r;
                const double cc = S.c[I], cpp = S.cp[I];
                const double uv[3] = {S.u[I], S.v[I], S.w[I]};
                double acc = 0.0, dsum = 0.0;
                for (int d = 0; d < 3; ++d) {
                    if (!D.active[d]) continue;
                    const double idx = S.inv_h[d][I] / S.h[d];   // inverse physical spacing
                    acc += (std::fabs(uv[d]) + cc) * idx;
                    dsum += idx * idx;
                }
                acc += curvature_rate(S, I, uv);
                double Dmax = mu0 / (Sc * r);
                for (int sp = 0; sp < S.Ns; ++sp) Dmax = jl_max(Dmax, mu0 / (Sc * r) + S.D_art[sp][I]);
                const double nu = (mu0 + S.mu_art[I] + S.beta_art[I]) * ri +
                                  (mu0 * cpp / Pr + S.kappa_art[I]) * ri / cpp + Dmax;
                acc += 2 * nu * dsum;
                rate = jl_max(rate, acc);
            }
    *rate_out = rate;
    *rho_min_out = rmin;
}

// filter_state! (src/timestep.jl:414-426)
void filter_state(Solver& S) {
    for (int d = 0; d < 3; ++d) {
        if (!S.D.active[d]) continue;
        for (int cc = 0; cc < S.ncons; ++cc) wrap_dim(S.D, S.comp(S.Q, cc), d);
        for (int cc = 0; cc < S.ncons; ++cc) {
            filt_along(S, S.tmp_a.data(), S.comp(S.Q, cc), d, cons_parity(S, d, cc));
            copy_interior(S.D, S.comp(S.Q, cc), S.tmp_a.data());
        }
    }
}

const double PLANCK_TIME = 5.391247e-44;

// check_step (src/stepcontrol.jl:184-204)
int check_step(const cles_step_control& c, double dt, double rho_min, double dt_seen) {
    if (!std::isfinite(dt)) return CLES_FAIL_NONFINITE;
    if (!(rho_min > 0)) return CLES_FAIL_NEGATIVE_DENSITY;
    if (!(dt > PLANCK_TIME)) return CLES_FAIL_PLANCK;
    if (!(dt >= c.dt_min)) return CLES_FAIL_DT_MIN;
    if (c.dt_min_ratio > 0 && dt_seen > 0)
        if (!(dt >= c.dt_min_ratio * dt_seen)) return CLES_FAIL_DT_COLLAPSE;
    return CLES_FAIL_NONE;
}

// predicted_dt (src/timestep.jl:29-42)
double predicted_dt(Solver& S, const cles_step_control& c, double rate) {
    double r = rate;
    if (c.predict > 0 && S.rate_prev > 0) r = jl_max(r, r + c.predict * (r - S.rate_prev));
    double dt = S.cfl / r;
    if (c.max_growth > 0 && S.dt_prev > 0) dt = jl_min(dt, c.max_growth * S.dt_prev);
    return dt;
}

// run! without callbacks (src/timestep.jl:277-405)
int run(Solver& S, double tfinal, int64_t nmax, cles_run_result* res) {
    const cles_step_control& ctl = S.desc.control;
    std::unique_ptr<Savepoint> save;
    if (ctl.retries > 0) save.reset(new Savepoint{S.Q, S.t, S.step});
    int attempts = 0;
    double dt_seen = 0.0;
    int64_t guard_step = -1, done = 0;
    double last_dt = 0.0;
    int failure = CLES_FAIL_NONE;
    while (S.t < tfinal && S.step < nmax) {
        S.tstage = S.t;
        apply_bcs(S);
        double rate, rmin;
        max_rate(S, &rate, &rmin);
        double dt = predicted_dt(S, ctl, rate);
        const int f = check_step(ctl, dt, rmin, dt_seen);
        if (f != CLES_FAIL_NONE) {
            if (!save || attempts >= ctl.retries) { failure = f; break; }
            attempts += 1;
            const int64_t fail_step = S.step;
            S.Q = save->Q;
            S.t = save->t;
            S.step = save->step;
            S.cfl *= ctl.cfl_backoff;
            guard_step = fail_step;
            S.dt_prev = 0.0; S.rate_prev = 0.0;
            dt_seen = 0.0;
            continue;
        }
        if (save && ctl.savepoint_interval > 0 && S.step > guard_step && S.step % ctl.savepoint_interval == 0) {
            save->Q = S.Q; save->t = S.t; save->step = S.step;
        }
        dt_seen = jl_max(dt_seen, dt);
        dt = jl_min(dt, tfinal - S.t);
        step(S, dt, true);
        S.t += dt;
        S.step += 1;
        S.dt_prev = dt;
        S.rate_prev = rate;
        last_dt = dt;
        ++done;
        if (S.desc.filter_interval > 0 && S.step % S.desc.filter_interval == 0) filter_state(S);
    }
    if (res) {
        res->steps = done; res->t = S.t; res->last_dt = last_dt; res->cfl = S.cfl;
        res->failure = failure; res->retries_used = attempts;
    }
    return failure == CLES_FAIL_NONE ? CLES_OK : CLES_EFAILURE;
}

// quad_weight / volume_integral (src/diagnostics.jl:41-80), no folds.
double quad_weight(const Solver& S, int d, int i) {
    // 1 in the interior and on a folded (half-offset) edge, 1/2 on a
    // node-centred closed edge (src/diagnostics.jl:41-49)
    const Decomp& D = S.D;
    if (!(D.active[d] && !D.periodic[d])) return 1.0;
    if (i == 0) return (S.folds[d] && S.folds[d]->lo) ? 1.0 : 0.5;
    if (i == D.ng[d] - 1) return (S.folds[d] && S.folds[d]->hi) ? 1.0 : 0.5;
    return 1.0;
}
double volume_integral(Solver& S, const double* f) {
    const Decomp& D = S.D;
    double dV = 1.0;
    for (int d = 0; d < 3; ++d) dV *= D.active[d] ? S.h[d] : 1.0;
    double acc = 0.0;
    for (int k = 0; k < D.nl[2]; ++k) {
        const double wk = quad_weight(S, 2, k);
        for (int j = 0; j < D.nl[1]; ++j) {
            const double wj = wk * quad_weight(S, 1, j);
            for (int i = 0; i < D.nl[0]; ++i) {
                const size_t I = D.at(i + D.nhd[0], j + D.nhd[1], k + D.nhd[2]);
                acc += wj * quad_weight(S, 0, i) * f[I] / S.inv_J[I];   // J = 1/inv_J
            }
        }
    }
    return acc * dV;
}

// dissipation_rate (src/diagnostics.jl:354-378)
double dissipation_rate(Solver& S) {
    primitives_and_gradients(S, false);
    compute_artificial(S);
    const double mu0 = S.desc.mu0;
    std::fill(S.tmp_b.begin(), S.tmp_b.end(), 0.0);
    for_interior(S.D, [&](size_t I, int, int, int) {
        const double mu = mu0 + S.mu_art[I];
        const double be = S.beta_art[I];
        const double divu = S.grad_u[0][0][I] + S.grad_u[1][1][I] + S.grad_u[2][2][I];
        double acc = 0.0;
        for (int b = 0; b < 3; ++b)
            for (int a = 0; a < 3; ++a) {
                const double tau = mu * (S.grad_u[a][b][I] + S.grad_u[b][a][I]) + (a == b ? (be - 2 * mu / 3) * divu : 0.0);
                acc += tau * S.grad_u[a][b][I];
            }
        S.tmp_b[I] = acc;
    });
    return volume_integral(S, S.tmp_b.data()) / volume_integral(S, S.rho.data());
}

// kinetic energy per unit volume (bench/tgv_energy.jl:175-184 uses rho = Q[1];
// here the mixture density), divided by the domain volume.
double kinetic_energy(Solver& S) {
    const Decomp& D = S.D;
    const size_t fs = S.fs;
    double ke = 0.0;
    for (int k = 0; k < D.nl[2]; ++k)
        for (int j = 0; j < D.nl[1]; ++j)
            for (int i = 0; i < D.nl[0]; ++i) {
                const size_t I = D.at(i + D.nhd[0], j + D.nhd[1], k + D.nhd[2]);
                double r = 0.0;
                for (int sp = 0; sp < S.Ns; ++sp) r += S.Q[I + fs * sp];
                const double q1 = S.Q[I + fs * S.i_mom[0]], q2 = S.Q[I + fs * S.i_mom[1]], q3 = S.Q[I + fs * S.i_mom[2]];
                ke += 0.5 * (q1 * q1 + q2 * q2 + q3 * q3) / r;
            }
    double cellvol = 1.0, vol = 1.0;
    for (int d = 0; d < 3; ++d) {
        cellvol *= D.active[d] ? S.h[d] : 1.0;
        vol *= D.active[d] ? S.desc.L[d] : 1.0;
    }
    return ke * cellvol / vol;
}

inline bool is_fold_bc(int bc) { return bc == CLES_BC_AXIS || bc == CLES_BC_ORIGIN || bc == CLES_BC_POLE; }

// unit_scalefactor (src/metric.jl:91-93)
bool unit_scalefactor(int metric, int d) {
    if (metric == CLES_METRIC_CYLINDRICAL) return d != 1;
    if (metric == CLES_METRIC_SPHERICAL) return d == 0;
    return true;
}

Solver* solver_create(const cles_solver_desc& A) {
    for (int d = 0; d < 3; ++d) {
        const bool p0 = A.bc[d][0] == CLES_BC_PERIODIC, p1 = A.bc[d][1] == CLES_BC_PERIODIC;
        if (p0 != p1) { set_err("dimension " + std::to_string(d + 1) + " mixes periodic and non-periodic conditions"); return nullptr; }
        if (A.n_global[d] < 1) { set_err("n_global must be >= 1"); return nullptr; }
        if (A.n_global[d] == 1 && !p0) { set_err("collapsed dimension must use (PeriodicBC(), PeriodicBC())"); return nullptr; }
        for (int s = 0; s < 2; ++s) {
            if (A.bc[d][s] < CLES_BC_PERIODIC || A.bc[d][s] > CLES_BC_POLE) { set_err("unknown boundary condition"); return nullptr; }
            if (A.bc_switchable[d][s] && ((A.bc_after[d][s] == CLES_BC_PERIODIC) != (A.bc[d][s] == CLES_BC_PERIODIC))) {
                set_err("SwitchableBC: both conditions must agree on periodicity");
                return nullptr;
            }
            if (A.bc_switchable[d][s] && (is_fold_bc(A.bc[d][s]) || is_fold_bc(A.bc_after[d][s]))) {
                set_err("SwitchableBC cannot wrap a fold condition (AxisBC, OriginBC, PoleBC); setup detects those by type");
                return nullptr;
            }
        }
    }
    if (A.n_species < 1 || A.n_species > CLES_MAX_SPECIES) { set_err("bad species count"); return nullptr; }
    if (A.n_body_forces < 0 || A.n_body_forces > CLES_MAX_BODY_FORCES) { set_err("at most 4 body forces"); return nullptr; }
    if (A.metric < CLES_METRIC_CARTESIAN || A.metric > CLES_METRIC_SPHERICAL) { set_err("unknown metric"); return nullptr; }
    bool stretched[3];
    for (int d = 0; d < 3; ++d) {
        stretched[d] = A.stretch_x[d] != nullptr;
        if (stretched[d] != (A.stretch_dxdxi[d] != nullptr)) { set_err("a Stretch needs both x and dx/dxi samples"); return nullptr; }
    }
    // NSCBC faces: the characteristic analysis covers faces whose normal scale
    // factor is one (src/nscbc.jl:309-323); this restatement, like the device
    // path, takes them on a uniform Cartesian grid only
    for (int d = 0; d < 3; ++d)
        for (int s = 0; s < 2; ++s)
            for (int which = 0; which < 2; ++which) {
                const int bc = which == 0 ? A.bc[d][s] : (A.bc_switchable[d][s] ? A.bc_after[d][s] : -1);
                if (bc != CLES_BC_NSCBC_OUTFLOW && bc != CLES_BC_NSCBC_INFLOW) continue;
                if (!unit_scalefactor(A.metric, d)) {
                    set_err("characteristic boundary conditions need a face whose normal metric scale factor is one");
                    return nullptr;
                }
            }
    // coordinate-singularity folds (src/rhs.jl:149-190)
    const bool axis = A.bc[0][0] == CLES_BC_AXIS;
    const bool orig1 = A.bc[0][0] == CLES_BC_ORIGIN;
    const bool pole_l = A.bc[1][0] == CLES_BC_POLE, pole_h = A.bc[1][1] == CLES_BC_POLE;
    if (pole_l != pole_h) { set_err("PoleBC must be applied at both ends of θ"); return nullptr; }
    const bool poles = pole_l;
    const double PI = 3.14159265358979323846;
    if (axis) {
        if (A.metric != CLES_METRIC_CYLINDRICAL) { set_err("AxisBC requires CylindricalMetric"); return nullptr; }
        if (stretched[0]) { set_err("folded dimensions cannot be stretched"); return nullptr; }
        if (!(std::fabs(A.origin[0]) < 1e-14)) { set_err("AxisBC requires origin[1] = 0"); return nullptr; }
        if (!(A.n_global[1] == 1 || A.n_global[1] % 2 == 0)) { set_err("resolved-θ AxisBC requires an even θ point count over 2π"); return nullptr; }
    }
    if (orig1) {
        if (A.metric != CLES_METRIC_SPHERICAL) { set_err("OriginBC requires SphericalMetric"); return nullptr; }
        if (stretched[0]) { set_err("folded dimensions cannot be stretched"); return nullptr; }
        if (!(std::fabs(A.origin[0]) < 1e-14)) { set_err("OriginBC requires origin[1] = 0"); return nullptr; }
        if (!(A.n_global[2] == 1 || A.n_global[2] % 2 == 0)) { set_err("resolved-φ OriginBC requires an even φ point count over 2π"); return nullptr; }
        const double tsum = 2 * A.origin[1] + A.L[1];
        if (!(A.n_global[1] == 1 || std::fabs(tsum - PI) <= 1e-10)) { set_err("OriginBC requires a θ range symmetric about π/2"); return nullptr; }
        // with phi collapsed the pairing is the theta reversal alone; an odd
        // theta count would leave the middle line without a partner
        if (A.n_global[2] == 1 && A.n_global[1] > 1 && A.n_global[1] % 2 != 0) {
            set_err("OriginBC pairs θ with π - θ: the θ point count must be even");
            return nullptr;
        }
    }
    if (poles) {
        if (A.metric != CLES_METRIC_SPHERICAL) { set_err("PoleBC requires SphericalMetric"); return nullptr; }
        if (stretched[1]) { set_err("folded dimensions cannot be stretched"); return nullptr; }
        if (!(std::fabs(A.origin[1]) < 1e-14 && std::fabs(A.L[1] - PI) <= 1e-10)) { set_err("PoleBC requires the θ domain (0, π)"); return nullptr; }
        if (!(A.n_global[2] == 1 || A.n_global[2] % 2 == 0)) { set_err("resolved-φ PoleBC requires an even φ point count over 2π"); return nullptr; }
    }
    int per[3];
    for (int d = 0; d < 3; ++d) per[d] = A.n_global[d] > 1 ? (A.bc[d][0] == CLES_BC_PERIODIC) : 1;
    if (axis || orig1) per[0] = 0;
    if (poles) per[1] = 0;
    for (int d = 0; d < 3; ++d)
        if (stretched[d] && per[d]) { set_err("dimension " + std::to_string(d + 1) + ": stretched dimensions must be non-periodic"); return nullptr; }
    // the area factors vary along r (and along theta on a sphere): a periodic
    // wrap of those dimensions would pair unlike halos; not supported
    if (A.metric != CLES_METRIC_CARTESIAN &&
        ((A.n_global[0] > 1 && per[0]) || (A.metric == CLES_METRIC_SPHERICAL && A.n_global[1] > 1 && per[1]))) {
        set_err("a periodic radial (or spherical polar) dimension is not supported");
        return nullptr;
    }
    auto S = std::make_unique<Solver>();
    S->desc = A;
    S->metric = A.metric;
    for (int d = 0; d < 3; ++d) {
        S->desc.stretch_x[d] = S->desc.stretch_dxdxi[d] = nullptr;
        S->stretched[d] = stretched[d];
        if (stretched[d]) {
            S->st_x[d].assign(A.stretch_x[d], A.stretch_x[d] + A.n_global[d]);
            S->st_m[d].assign(A.stretch_dxdxi[d], A.stretch_dxdxi[d] + A.n_global[d]);
        }
    }
    S->D = make_decomp(A.n_global, per, A.n_halo);
    S->Ns = A.n_species; S->ncons = A.n_species + 4;
    S->i_mom[0] = S->Ns; S->i_mom[1] = S->Ns + 1; S->i_mom[2] = S->Ns + 2; S->i_energy = S->Ns + 3;
    if (A.eos != CLES_EOS_IDEAL && A.eos != CLES_EOS_NASA9) { set_err("unknown equation of state"); return nullptr; }
    for (int k = 0; k < S->Ns; ++k) {
        S->Rk[k] = A.R[k];
        S->cvk[k] = A.eos == CLES_EOS_IDEAL ? A.R[k] / (A.gamma[k] - 1) : 0.0;
        S->cpk[k] = S->Rk[k] + S->cvk[k];
        if (A.eos == CLES_EOS_NASA9 && (A.n_intervals[k] < 1 || A.n_intervals[k] > CLES_MAX_NASA9_INTERVALS)) {
            set_err("NASA-9 species needs 1..4 intervals");
            return nullptr;
        }
    }
    // grid spacing: computational xi in [0, 1] for stretched dims, half-offset
    // grids on folded dims (src/rhs.jl:191-205)
    const bool fold_lo_dim[3] = {axis || orig1, poles, false};
    const bool fold_hi_dim[3] = {false, poles, false};
    for (int d = 0; d < 3; ++d) {
        const int n = A.n_global[d];
        if (!S->D.active[d]) S->h[d] = 1.0;
        else if (stretched[d]) S->h[d] = 1.0 / (n - 1);
        else if (fold_lo_dim[d] && fold_hi_dim[d]) S->h[d] = A.L[d] / n;
        else if (fold_lo_dim[d]) S->h[d] = A.L[d] / (n - 0.5);
        else S->h[d] = S->D.periodic[d] ? A.L[d] / n : A.L[d] / (n - 1);
        S->coord_shift[d] = fold_lo_dim[d] ? S->h[d] / 2 : 0.0;
        S->orig[d] = stretched[d] ? 0.0 : A.origin[d];
    }
    // fold specs (src/rhs.jl:216-280)
    auto foldspec = [&](int d, bool lo, bool hi, int pdim, int revdim, const int sv[3], int area_parity) -> bool {
        auto F = std::make_unique<FoldSpec>();
        F->dim = d; F->lo = lo; F->hi = hi;
        for (int j = 0; j < 3; ++j) F->sigvel[j] = sv[j];
        for (int cc = 0; cc < S->ncons; ++cc)
            F->sigflux.push_back(conserved_parity(*S, sv, cc) * sv[d] * area_parity);
        const bool shift_needed = pdim >= 0 && S->D.active[pdim];
        const bool rev_needed = revdim >= 0 && S->D.active[revdim];
        F->paired = shift_needed || rev_needed;
        F->pair.pdim = shift_needed ? pdim : -1;
        F->pair.revdim = rev_needed ? revdim : -1;
        if (shift_needed && S->D.nl[pdim] % 2 != 0) {
            set_err("pairing dim " + std::to_string(pdim + 1) + " local extent must be even");
            return false;
        }
        for (int t = 0; t < 2; ++t) {
            const int sg = t == 0 ? 1 : -1;
            Plan* dp = plan_create(S->D, A.deriv, d, S->h[d], 1, lo ? sg : 0, hi ? sg : 0);
            if (!dp) return false;
            F->dp[t].reset(dp);
            Plan* fp = plan_create(S->D, A.filt, d, S->h[d], 1, lo ? sg : 0, hi ? sg : 0);
            if (!fp) return false;
            F->fp[t].reset(fp);
        }
        S->folds[d] = std::move(F);
        return true;
    };
    if (axis) {
        const int sv[3] = {-1, -1, 1};
        if (!foldspec(0, true, false, 1, -1, sv, -1)) return nullptr;   // A_1 = r is odd
    } else if (orig1) {
        const int sv[3] = {-1, 1, -1};
        if (!foldspec(0, true, false, 2, 1, sv, 1)) return nullptr;    // A_1 = r^2 sin(theta) is even
    }
    if (poles) {
        const int sv[3] = {1, -1, -1};
        if (!foldspec(1, true, true, 2, -1, sv, -1)) return nullptr;    // A_2 = r sin(theta) is odd in theta
    }
    for (int d = 0; d < 3; ++d) {
        if (!S->D.active[d] || S->folds[d]) continue;
        Plan* dp = plan_create(S->D, A.deriv, d, S->h[d], 1);
        if (!dp) return nullptr;
        S->dplan[d].reset(dp);
        Plan* fp = plan_create(S->D, A.filt, d, S->h[d], 1);
        if (!fp) return nullptr;
        S->fplan[d].reset(fp);
    }
    const size_t fs = S->D.size();
    S->fs = fs;
    auto F = [&]() { return std::vector<double>(fs, 0.0); };
    S->Q.assign(fs * S->ncons, 0.0); S->dQ.assign(fs * S->ncons, 0.0); S->du.assign(fs * S->ncons, 0.0);
    S->rho = F(); S->u = F(); S->v = F(); S->w = F(); S->p = F(); S->T = F(); S->c = F(); S->cp = F();
    for (int sp = 0; sp < S->Ns; ++sp) { S->Y.push_back(F()); S->D_art.push_back(F()); }
    for (int d = 0; d < 3; ++d) {
        for (int j = 0; j < 3; ++j) S->grad_u[d][j] = F();
        S->grad_T[d] = F();
        for (int sp = 0; sp < S->Ns; ++sp) S->grad_Y[d].push_back(F());
        for (int cc = 0; cc < S->ncons; ++cc) S->flux[d][cc] = F();
        S->area[d] = F();
        S->inv_h[d] = F();
    }
    S->mu_art = F(); S->beta_art = F(); S->kappa_art = F(); S->strain = F();
    S->sensor = F(); S->sensor_sp = F(); S->tmp_a = F(); S->tmp_b = F();
    S->inv_J = F(); S->inv_r = F(); S->cot_over_r = F();
    if (S->folds[0] || S->folds[1] || S->folds[2]) { S->pairbuf = F(); S->pairout = F(); }
    S->cfl = A.cfl;
    init_geometry(*S);
    return S.release();
}

}  // namespace

// ======================================================================
// C interface (consumed by tests/ and bench.py through ctypes)
// ======================================================================
struct orc_plan { Plan* p; };
struct orc_solver { Solver* s; };

extern "C" {

const char* orc_last_error(void) { return g_err.c_str(); }

int orc_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
    return omp_get_max_threads();
#else
    (void)n;
    return 1;
#endif
}

int orc_scheme_lele_d1_6(cles_scheme* s) { preset_lele_d1_6(s); return 0; }
int orc_scheme_pade_d1_4(cles_scheme* s) { preset_pade_d1_4(s); return 0; }
int orc_scheme_compact_filter(double af, cles_scheme* s) { preset_compact_filter(af, s); return 0; }
int orc_scheme_lele_d1_10(cles_scheme* s) { preset_lele_d1_10(s); return 0; }

orc_plan* orc_plan_create(const cles_grid* g, const cles_scheme* s, int dim, double h, int P) {
    Decomp D = make_decomp(g->n_global, g->periodic, g->n_halo);
    if (dim < 1 || dim > 3) { set_err("dim must be 1..3"); return nullptr; }
    Plan* p = plan_create(D, *s, dim - 1, h, P);
    if (!p) return nullptr;
    return new orc_plan{p};
}
void orc_plan_destroy(orc_plan* p) { if (p) { delete p->p; delete p; } }
int orc_apply_along(orc_plan* p, const double* f, double* out) { apply_along(*p->p, out, f); return 0; }

void orc_exchange_halos(const cles_grid* g, double* f) {
    Decomp D = make_decomp(g->n_global, g->periodic, g->n_halo);
    exchange_halos(D, f);
}
void orc_exchange_dim(const cles_grid* g, double* f, int dim) {
    Decomp D = make_decomp(g->n_global, g->periodic, g->n_halo);
    wrap_dim(D, f, dim - 1);
}

// BandFactor + solve_col! (src/banded.jl:31-80) on one (2q+1) x n band,
// Ab[(q + t) + (2q+1) i] = A[i, i + t]; b is overwritten with A^-1 b.
int orc_band_solve(int q, int n, const double* Ab, double* b) {
    if (q < 1 || n < 1) { set_err("band_solve: q >= 1 and n >= 1"); return CLES_EINVAL; }
    BandFactor F;
    F.build(std::vector<double>(Ab, Ab + (size_t)(2 * q + 1) * n), n, q);
    F.solve(b, 1);
    return 0;
}

orc_solver* orc_solver_create(const cles_solver_desc* d) {
    Solver* s = solver_create(*d);
    if (!s) return nullptr;
    return new orc_solver{s};
}
void orc_solver_destroy(orc_solver* s) { if (s) { delete s->s; delete s; } }
// The same Solver on a Decomp split `P` ways along `dim` (1-based): the
// derivative and filter plans along dim emulate P ranks (Decomp dims,
// src/decomposition.jl:80-122; LineSolver / BandLineSolver with P > 1,
// src/tridiag.jl:85-170, src/banded.jl:108-214).  Halo exchange needs no
// emulation: the oracle holds the whole field.  Folded dimensions are refused.
int orc_solver_split(orc_solver* s, int dim, int P) {
    Solver& S = *s->s;
    const int d = dim - 1;
    if (d < 0 || d > 2 || !S.D.active[d]) { set_err("split dimension must be an active 1, 2 or 3"); return CLES_EINVAL; }
    if (S.folds[d]) { set_err("folds on a split dimension are not supported"); return CLES_EINVAL; }
    Plan* dp = plan_create(S.D, S.desc.deriv, d, S.h[d], P);
    if (!dp) return CLES_EINVAL;
    Plan* fp = plan_create(S.D, S.desc.filt, d, S.h[d], P);
    if (!fp) { delete dp; return CLES_EINVAL; }
    S.dplan[d].reset(dp);
    S.fplan[d].reset(fp);
    return 0;
}
int64_t orc_field_size(orc_solver* s) { return (int64_t)s->s->fs; }
int orc_set_state(orc_solver* s, const double* Q) { std::memcpy(s->s->Q.data(), Q, sizeof(double) * s->s->Q.size()); return 0; }
int orc_get_state(orc_solver* s, double* Q) { std::memcpy(Q, s->s->Q.data(), sizeof(double) * s->s->Q.size()); return 0; }
int orc_get_rhs(orc_solver* s, double* dQ) { std::memcpy(dQ, s->s->dQ.data(), sizeof(double) * s->s->dQ.size()); return 0; }
int orc_apply_bcs(orc_solver* s) { apply_bcs(*s->s); return 0; }
int orc_compute_rhs(orc_solver* s, int primitives_current) { compute_rhs(*s->s, primitives_current != 0); return 0; }
int orc_max_rate(orc_solver* s, double* rate, double* rmin) { max_rate(*s->s, rate, rmin); return 0; }
int orc_step(orc_solver* s, double dt, int prepared) { step(*s->s, dt, prepared != 0); return 0; }
int orc_filter_state(orc_solver* s) { filter_state(*s->s); return 0; }
int orc_run(orc_solver* s, double tfinal, int64_t nmax, cles_run_result* r) { return run(*s->s, tfinal, nmax, r); }
double orc_kinetic_energy(orc_solver* s) { return kinetic_energy(*s->s); }
// volume_integral(solver, f) (src/diagnostics.jl:41-80) of a padded field
double orc_volume_integral(orc_solver* s, const double* f) { return volume_integral(*s->s, f); }
double orc_dissipation_rate(orc_solver* s) { return dissipation_rate(*s->s); }
int orc_get_clock(orc_solver* s, double* t, int64_t* step_, double* cfl) { *t = s->s->t; *step_ = s->s->step; *cfl = s->s->cfl; return 0; }
int orc_set_clock(orc_solver* s, double t, int64_t step_, double cfl) { s->s->t = t; s->s->step = step_; s->s->cfl = cfl; return 0; }

// Padded full-array copies of named fields (same codes as CLES_FIELD_*).
int orc_get_field(orc_solver* so, int which, double* out) {
    Solver& S = *so->s;
    const std::vector<double>* src = nullptr;
    switch (which) {
        case CLES_FIELD_RHO: src = &S.rho; break;
        case CLES_FIELD_U: src = &S.u; break;
        case CLES_FIELD_V: src = &S.v; break;
        case CLES_FIELD_W: src = &S.w; break;
        case CLES_FIELD_P: src = &S.p; break;
        case CLES_FIELD_T: src = &S.T; break;
        case CLES_FIELD_C: src = &S.c; break;
        case CLES_FIELD_CP: src = &S.cp; break;
        case CLES_FIELD_MU_ART: src = &S.mu_art; break;
        case CLES_FIELD_BETA_ART: src = &S.beta_art; break;
        case CLES_FIELD_KAPPA_ART: src = &S.kappa_art; break;
        case CLES_FIELD_SENSOR: src = &S.sensor; break;
        default:
            if (which >= CLES_FIELD_Y0 && which < CLES_FIELD_Y0 + S.Ns) src = &S.Y[which - CLES_FIELD_Y0];
            else if (which >= CLES_FIELD_D_ART0 && which < CLES_FIELD_D_ART0 + S.Ns) src = &S.D_art[which - CLES_FIELD_D_ART0];
            else if (which >= CLES_FIELD_GRAD_U0 && which < CLES_FIELD_GRAD_U0 + 9) {
                const int k = which - CLES_FIELD_GRAD_U0;
                src = &S.grad_u[k / 3][k % 3];
            }
    }
    if (!src) { set_err("unknown field"); return CLES_EINVAL; }
    std::memcpy(out, src->data(), sizeof(double) * src->size());
    return 0;
}

// flux[d][c] of the last compute_rhs (padded field), for parity scales.
int orc_get_flux(orc_solver* so, int d, int c, double* out) {
    Solver& S = *so->s;
    if (d < 0 || d > 2 || c < 0 || c >= S.ncons) { set_err("bad flux index"); return CLES_EINVAL; }
    std::memcpy(out, S.flux[d][c].data(), sizeof(double) * S.fs);
    return 0;
}

// NASA-9 species functions and the Newton inversion, for the thermodynamic tests
double orc_nasa9_cp(const cles_solver_desc* d, int k, double T) { return n9_species_cp(*d, k, T); }
double orc_nasa9_h(const cles_solver_desc* d, int k, double T) { return n9_species_h(*d, k, T); }
double orc_nasa9_e(const cles_solver_desc* d, int k, double T) { return n9_species_e(*d, k, T); }
double orc_nasa9_temperature(const cles_solver_desc* d, double e, const double* Y) { return n9_temperature(*d, e, Y); }

int orc_switch_bc(orc_solver* s, int d, int side) {
    if (d < 0 || d > 2 || side < 0 || side > 1 || !s->s->desc.bc_switchable[d][side]) {
        set_err("face is not a SwitchableBC");
        return CLES_EINVAL;
    }
    s->s->switched[d][side] = true;
    return 0;
}

// Geometry arrays (padded): 0 inv_J, 1..3 A_d, 4..6 1/h_d, 7 1/r, 8 cot(theta)/r.
int orc_get_geometry(orc_solver* so, int which, double* out) {
    Solver& S = *so->s;
    const std::vector<double>* src = nullptr;
    if (which == 0) src = &S.inv_J;
    else if (which >= 1 && which <= 3) src = &S.area[which - 1];
    else if (which >= 4 && which <= 6) src = &S.inv_h[which - 4];
    else if (which == 7) src = &S.inv_r;
    else if (which == 8) src = &S.cot_over_r;
    if (!src) { set_err("unknown geometry array"); return CLES_EINVAL; }
    std::memcpy(out, src->data(), sizeof(double) * src->size());
    return 0;
}
// Grid spacing and coordinate shift per dimension.
int orc_grid_spacing(orc_solver* so, double* h, double* shift, double* orig) {
    Solver& S = *so->s;
    for (int d = 0; d < 3; ++d) { h[d] = S.h[d]; shift[d] = S.coord_shift[d]; orig[d] = S.orig[d]; }
    return 0;
}
// deriv_along!(out, f, solver, d, sig) followed by _scale_grad! on padded
// fields (f must hold current halos on periodic dims).
int orc_solver_deriv(orc_solver* so, double* f, double* out, int d, int sig, int scale) {
    Solver& S = *so->s;
    if (d < 0 || d > 2 || !S.D.active[d]) { set_err("dimension is collapsed"); return CLES_EINVAL; }
    exchange_halos(S.D, f);
    deriv_along(S, out, f, d, sig);
    if (scale) {
        const double* ih = S.inv_h[d].data();
        for (size_t I = 0; I < S.fs; ++I) out[I] *= ih[I];
    }
    return 0;
}
int orc_solver_filter(orc_solver* so, double* f, double* out, int d, int sig) {
    Solver& S = *so->s;
    if (d < 0 || d > 2 || !S.D.active[d]) { set_err("dimension is collapsed"); return CLES_EINVAL; }
    exchange_halos(S.D, f);
    filt_along(S, out, f, d, sig);
    return 0;
}

int orc_solver_set_face_fn(orc_solver* so, int d, int side, int which, cles_face_fn fn, void* user) {
    Solver& S = *so->s;
    if (d < 0 || d > 2 || side < 0 || side > 1 || which < 0 || which > 1) { set_err("no such face"); return CLES_EINVAL; }
    if (which == 1 && !S.desc.bc_switchable[d][side]) { set_err("face is not a SwitchableBC"); return CLES_EINVAL; }
    const int bc = which == 0 ? S.desc.bc[d][side] : S.desc.bc_after[d][side];
    if (fn && bc != CLES_BC_DIRICHLET && bc != CLES_BC_NSCBC_INFLOW) {
        set_err("only DirichletBC and NSCBCInflowBC faces take a function");
        return CLES_EINVAL;
    }
    S.ffn[d][side][which] = fn;
    S.fuser[d][side][which] = user;
    return 0;
}

int orc_check_step(const cles_step_control* c, double dt, double rho_min, double dt_seen) {
    return check_step(*c, dt, rho_min, dt_seen);
}

}  // extern "C"
