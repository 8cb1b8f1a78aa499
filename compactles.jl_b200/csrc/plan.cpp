// Host-side construction of directional compact plans.
//
// A line of n points is the global banded system of plan_direction
// (src/operators.jl:44-101, src/operators_banded.jl:29-125): interior rows
// carry the scheme's LHS band, closed edges carry the closure rows (mirrored at
// the high edge), periodic lines wrap.  The device solves it with the
// reduced-interface ("spike") method of src/tridiag.jl:1-22 and
// src/banded.jl:1-27, applied inside one line: the line is cut into S
// segments of at most kMaxSeg points (one per thread), each segment is solved
// locally with its own factorisation, the 2q head/tail values of all segments
// form a (2qS)^2 reduced system whose inverse is precomputed here, and every
// segment is corrected with its spike vectors.  With S = 1 and a periodic line
// this is exactly the reference's single-rank self-coupled solve; with S > 1
// it is the reference's P-rank distributed solve with ranks mapped to threads.
// Closed tridiagonal lines with more than 32 segments replace the dense
// inverse by block cyclic reduction of the same reduced system (coefficients
// precomputed here), which keeps long single lines (1-D tubes of thousands of
// cells) at O(log S) depth.

#include <array>
#include <algorithm>
#include <cmath>
#include <cstring>

#include "cles_internal.h"

namespace cles {

namespace {

struct Band {
    int n, q;
    bool periodic;
    std::vector<double> a;  // n x (2q+1), a[i*(2q+1) + q + s] = A[i, i+s]
    double at(int r, int c) const {
        int s = c - r;
        if (periodic) {
            if (s > n / 2) s -= n;
            if (s < -n / 2) s += n;
        }
        if (s < -q || s > q) return 0.0;
        return a[(size_t)r * (2 * q + 1) + q + s];
    }
};

// LU with partial pivoting of a dense N x N row-major matrix; returns inverse.
std::vector<double> dense_inverse(std::vector<double> A, int N) {
    std::vector<int> piv(N);
    for (int k = 0; k < N; ++k) {
        int p = k;
        double best = std::fabs(A[(size_t)k * N + k]);
        for (int i = k + 1; i < N; ++i)
            if (std::fabs(A[(size_t)i * N + k]) > best) { best = std::fabs(A[(size_t)i * N + k]); p = i; }
        if (best == 0.0) throw Error(CLES_EINVAL, "singular reduced interface system");
        piv[k] = p;
        if (p != k)
            for (int j = 0; j < N; ++j) std::swap(A[(size_t)k * N + j], A[(size_t)p * N + j]);
        const double inv = 1.0 / A[(size_t)k * N + k];
        for (int i = k + 1; i < N; ++i) {
            const double l = A[(size_t)i * N + k] * inv;
            A[(size_t)i * N + k] = l;
            if (l != 0.0)
                for (int j = k + 1; j < N; ++j) A[(size_t)i * N + j] -= l * A[(size_t)k * N + j];
        }
    }
    std::vector<double> X((size_t)N * N, 0.0), b(N);
    for (int c = 0; c < N; ++c) {
        std::fill(b.begin(), b.end(), 0.0);
        b[c] = 1.0;
        for (int k = 0; k < N; ++k) std::swap(b[k], b[piv[k]]);
        for (int i = 0; i < N; ++i)
            for (int k = 0; k < i; ++k) b[i] -= A[(size_t)i * N + k] * b[k];
        for (int i = N - 1; i >= 0; --i) {
            double acc = b[i];
            for (int k = i + 1; k < N; ++k) acc -= A[(size_t)i * N + k] * b[k];
            b[i] = acc / A[(size_t)i * N + i];
        }
        for (int r = 0; r < N; ++r) X[(size_t)r * N + c] = b[r];
    }
    return X;
}

// Local banded factorisation of rows/cols [off, off+m) of the band.
struct LocalFactor {
    int m, q;
    std::vector<double> L;   // L[(t-1)*m + k]: multiplier eliminating row k+t with pivot row k
    std::vector<double> U;   // U[t*m + i] = U[i, i+t], t = 0..q
    void build(const Band& B, int off, int mm) {
        m = mm; q = B.q;
        const int W = 2 * q + 1;
        std::vector<double> w((size_t)m * W, 0.0);
        for (int i = 0; i < m; ++i)
            for (int s = -q; s <= q; ++s) {
                const int c = i + s;
                if (c < 0 || c >= m) continue;
                w[(size_t)i * W + q + s] = B.at(off + i, off + c);
            }
        L.assign((size_t)q * m, 0.0);
        for (int k = 0; k < m - 1; ++k) {
            const double piv = w[(size_t)k * W + q];
            if (piv == 0.0) throw Error(CLES_EINVAL, "zero pivot in a segment factorisation");
            const int tmax = std::min(q, m - 1 - k);
            for (int t = 1; t <= tmax; ++t) {
                const int i = k + t;
                const double l = w[(size_t)i * W + q - t] / piv;
                L[(size_t)(t - 1) * m + k] = l;
                for (int u = 1; u <= tmax; ++u) w[(size_t)i * W + q + u - t] -= l * w[(size_t)k * W + q + u];
            }
        }
        U.assign((size_t)(q + 1) * m, 0.0);
        for (int i = 0; i < m; ++i)
            for (int t = 0; t <= std::min(q, m - 1 - i); ++t) U[(size_t)t * m + i] = w[(size_t)i * W + q + t];
    }
    void solve(double* x) const {
        for (int k = 0; k < m - 1; ++k)
            for (int t = 1; t <= std::min(q, m - 1 - k); ++t) x[k + t] -= L[(size_t)(t - 1) * m + k] * x[k];
        for (int i = m - 1; i >= 0; --i) {
            double acc = x[i];
            for (int t = 1; t <= std::min(q, m - 1 - i); ++t) acc -= U[(size_t)t * m + i] * x[i + t];
            x[i] = acc / U[i];
        }
    }
};

void mat2_mul(const double* a, const double* b, double* o) {  // o = a b (2x2 row-major)
    const double t0 = a[0] * b[0] + a[1] * b[2], t1 = a[0] * b[1] + a[1] * b[3];
    const double t2 = a[2] * b[0] + a[3] * b[2], t3 = a[2] * b[1] + a[3] * b[3];
    o[0] = t0; o[1] = t1; o[2] = t2; o[3] = t3;
}
void mat2_inv(const double* a, double* o) {
    const double det = a[0] * a[3] - a[1] * a[2];
    if (det == 0.0) throw Error(CLES_EINVAL, "singular 2x2 block in the interface reduction");
    const double t0 = a[3] / det, t1 = -a[1] / det, t2 = -a[2] / det, t3 = a[0] / det;
    o[0] = t0; o[1] = t1; o[2] = t2; o[3] = t3;
}

// Warp-per-line parameters (periodic, q = 1, n = 32 * XP).  The interface
// system of the 32 lane segments is block tridiagonal and cyclic in
// X_s = (head_s, tail_s):  A X_{s-1} + X_s + C X_{s+1} = (y_s[0], y_s[XP-1]),
// A = [[0, v_0], [0, v_{XP-1}]], C = [[w_0, 0], [w_{XP-1}, 0]].  Parallel cyclic
// reduction at distances 1, 2, 4, 8 makes every equation couple only to the
// lane 16 away, which in a 32-cycle is the same unknown on both sides; the
// final pairing then leaves a 2x2 system per lane.  Every matrix is the same
// for all lanes, so they are computed here once.
void build_warp_line(CompactPlan& plan, const Band& B, const cles_scheme& s, int n, int dim, bool periodic) {
    plan.has_xw = false;
    if (dim != 0 || !periodic || s.q != 1 || n % 32 != 0) return;
    const int XP = n / 32;
    // an even count of points per lane, for the lane's vector loads
    if (XP != 2 && XP != 4 && XP != 6 && XP != 8 && XP != 12 && XP != 16) return;
    if (XP < s.M) return;
    WarpLineParams& W = plan.XW;
    std::memset(&W, 0, sizeof(W));
    W.XP = XP;
    // local factorisation of one lane segment (rows 0..XP-1 of the Toeplitz band)
    LocalFactor F;
    F.build(B, 0, XP);
    for (int i = 0; i < XP; ++i) {
        W.l[i] = i > 0 ? F.L[(size_t)i - 1] : 0.0;
        W.dinv[i] = 1.0 / F.U[i];
        W.c[i] = i < XP - 1 ? F.U[(size_t)XP + i] : 0.0;
    }
    std::vector<double> v(XP, 0.0), w(XP, 0.0);
    v[0] = B.at(0, n - 1);            // row 0 couples to the previous segment's tail
    w[XP - 1] = B.at(XP - 1, XP);     // row XP-1 couples to the next segment's head
    F.solve(v.data());
    F.solve(w.data());
    for (int i = 0; i < XP; ++i) { W.v[i] = v[i]; W.w[i] = w[i]; }
    double A[4] = {0.0, v[0], 0.0, v[XP - 1]};
    double Bm[4] = {1.0, 0.0, 0.0, 1.0};
    double Cm[4] = {w[0], 0.0, w[XP - 1], 0.0};
    for (int k = 0; k < 4; ++k) {
        double Bi[4], al[4], ga[4], t1[4], t2[4];
        mat2_inv(Bm, Bi);
        mat2_mul(A, Bi, al);
        mat2_mul(Cm, Bi, ga);
        for (int e = 0; e < 4; ++e) { al[e] = -al[e]; ga[e] = -ga[e]; }
        double nA[4], nC[4], nB[4];
        mat2_mul(al, A, nA);
        mat2_mul(ga, Cm, nC);
        mat2_mul(al, Cm, t1);
        mat2_mul(ga, A, t2);
        for (int e = 0; e < 4; ++e) nB[e] = Bm[e] + t1[e] + t2[e];
        for (int e = 0; e < 4; ++e) { W.alpha[k][e] = al[e]; W.gamma[k][e] = ga[e]; A[e] = nA[e]; Bm[e] = nB[e]; Cm[e] = nC[e]; }
    }
    double E[4], Bi[4], af[4], t[4], Bf[4];
    for (int e = 0; e < 4; ++e) E[e] = A[e] + Cm[e];
    mat2_inv(Bm, Bi);
    mat2_mul(E, Bi, af);
    for (int e = 0; e < 4; ++e) af[e] = -af[e];
    mat2_mul(af, E, t);
    for (int e = 0; e < 4; ++e) Bf[e] = Bm[e] + t[e];
    mat2_inv(Bf, W.binv_f);
    for (int e = 0; e < 4; ++e) W.alpha_f[e] = af[e];
    for (int i = 0; i < kMaxXP; ++i) {
        W.lf[i] = (float)W.l[i]; W.dinvf[i] = (float)W.dinv[i]; W.cf[i] = (float)W.c[i];
        W.vf[i] = (float)W.v[i]; W.wf[i] = (float)W.w[i];
    }
    for (int k = 0; k < 4; ++k)
        for (int e = 0; e < 4; ++e) { W.alphaf[k][e] = (float)W.alpha[k][e]; W.gammaf[k][e] = (float)W.gamma[k][e]; }
    for (int e = 0; e < 4; ++e) { W.alpha_ff[e] = (float)W.alpha_f[e]; W.binv_ff[e] = (float)W.binv_f[e]; }
    plan.has_xw = true;
}

}  // namespace

CompactPlan::~CompactPlan() {
    if (tab64) cudaFree(tab64);
    if (tab32) cudaFree(tab32);
}

LineBand make_line_band(const cles_scheme& s, int n, int lo_fold, int hi_fold, bool lo_open, bool hi_open) {
    const int q = s.q, nc = s.nc, W = 2 * q + 1;
    LineBand b;
    b.n = n;
    b.q = q;
    b.a.assign((size_t)n * W, 0.0);
    for (int i = 0; i < n; ++i) {
        b.a[(size_t)i * W + q] = 1.0;
        for (int t = 1; t <= q; ++t) {
            b.a[(size_t)i * W + q + t] = s.lhs[t - 1];
            b.a[(size_t)i * W + q - t] = s.lhs[t - 1];
        }
    }
    // parity folds (src/operators.jl:61-70, src/operators_banded.jl:58-77):
    // the coupling of row i to a ghost column maps onto its mirror column
    // with the solution's sign sigma_g (the field's parity for a filter,
    // its opposite for a derivative)
    const int sg_lo = s.symmetric ? lo_fold : -lo_fold;
    const int sg_hi = s.symmetric ? hi_fold : -hi_fold;
    if (lo_fold)
        for (int i = 1; i <= q; ++i)
            for (int m = 1; m <= q; ++m) {
                if (i - m >= 1) continue;
                const int jcol = m - i + 1;
                b.a[(size_t)(i - 1) * W + q + (jcol - i)] += (double)sg_lo * s.lhs[m - 1];
            }
    if (hi_fold)
        for (int i = n - q + 1; i <= n; ++i)
            for (int m = 1; m <= q; ++m) {
                if (i + m <= n) continue;
                const int jcol = 2 * n + 1 - (i + m);
                b.a[(size_t)(i - 1) * W + q + (jcol - i)] += (double)sg_hi * s.lhs[m - 1];
            }
    // closure rows at closed ends; an open end (rank interface) keeps the
    // interior rows (src/operators.jl:66-84, src/operators_banded.jl:48-112)
    for (int j = 0; j < nc && !lo_fold && !lo_open; ++j)
        for (int t = -q; t <= q; ++t) {
            double v = s.clo_lhs[j][q + t];
            if (j + t < 0) {
                if (q >= 2 && v != 0.0) throw Error(CLES_EINVAL, "closure row references a column before the edge");
                v = 0.0;  // tridiagonal row 1 ignores its sub-diagonal
            }
            b.a[(size_t)j * W + q + t] = v;
        }
    for (int j = 0; j < nc && !hi_fold && !hi_open; ++j) {
        const int r = n - 1 - j;
        for (int t = -q; t <= q; ++t) {
            double v = s.clo_lhs[j][q - t];
            if (r + t >= n) v = 0.0;
            b.a[(size_t)r * W + q + t] = v;
        }
    }
    // the first/last rows have no couplings beyond the edge (at an open end
    // they are the rank-level spike columns)
    for (int i = 0; i < n; ++i)
        for (int t = -q; t <= q; ++t)
            if (i + t < 0 || i + t >= n) b.a[(size_t)i * W + q + t] = 0.0;
    return b;
}

void LineBand::factor() {
    Band B;
    B.n = n; B.q = q; B.periodic = false; B.a = a;
    LocalFactor F;
    F.build(B, 0, n);
    L = std::move(F.L);
    U = std::move(F.U);
}

void LineBand::solve(double* x) const {
    const int m = n;
    for (int k = 0; k < m - 1; ++k)
        for (int t = 1; t <= std::min(q, m - 1 - k); ++t) x[k + t] -= L[(size_t)(t - 1) * m + k] * x[k];
    for (int i = m - 1; i >= 0; --i) {
        double acc = x[i];
        for (int t = 1; t <= std::min(q, m - 1 - i); ++t) acc -= U[(size_t)t * m + i] * x[i + t];
        x[i] = acc / U[i];
    }
}

// The pieces of a SigPlan: P = ceil(n / 128) (at most 64) pieces, the middle
// ones of equal length n / P and the remainder shared by the first and last;
// S segments of at most 16 points in every piece (32 beyond 512-point
// pieces), two pieces per CTA.  Spikes of each class and the reduced system
// over all pieces as in build_split_plan (the rank-level spikes of
// src/tridiag.jl:85-123 and src/banded.jl:108-169), its dense inverse whole.
static void build_sig_plan(CompactPlan& plan, const cles_scheme& s, const int n3[3], double h, int dtype) {
    const int n = n3[0], q = s.q;
    const int P = std::min(64, (n + 127) / 128);
    if (P < 4) return;
    // pieces of at most 1024 points (the correction's four points a thread)
    if ((n / P) + (n % P) > 1024) return;
    const int mid = n / P, rem = n - P * mid;
    const int len[3] = {mid + rem / 2, mid, mid + (rem - rem / 2)};
    const int maxlen = std::max(len[0], len[2]);
    int S = (maxlen + 15) / 16;
    if (S > 32) S = (maxlen + kMaxSeg - 1) / kMaxSeg;
    if (S > 32 || mid / S < std::max(2 * q + 1, q + 1)) return;
    const int LB = 2;
    auto sp = std::unique_ptr<SigPlan>(new SigPlan());
    sp->P = P;
    sp->q = q;
    sp->lines = plan.P.lines;
    sp->dtype = dtype;
    for (int c = 0; c < 3; ++c) sp->len[c] = len[c];
    const int L = (int)plan.P.lines;
    for (int c = 0; c < 3; ++c) {
        // the middle class enumerates (piece - 1) fastest, then the line
        int nc3[3] = {len[c], c == 1 ? P - 2 : L, c == 1 ? L : 1};
        build_compact_plan(sp->cls[c], s, nc3, 0, false, h, dtype, 0, 0, c > 0, c < 2, 0, S, LB);
        if (sp->cls[c].P.pcr || sp->cls[c].P.S != S || sp->cls[c].P.LB != LB) return;
    }
    // spikes per class, reduced system in z = (head_0, tail_0, head_1, ...)
    std::vector<double> Vc[3], Wc[3];
    for (int c = 0; c < 3; ++c) {
        const int m = len[c];
        const bool lo = c > 0, hi = c < 2;
        LineBand b = make_line_band(s, m, 0, 0, lo, hi);
        b.factor();
        Vc[c].assign((size_t)q * m, 0.0);
        Wc[c].assign((size_t)q * m, 0.0);
        for (int t = 0; t < q; ++t) {
            double* v = &Vc[c][(size_t)t * m];
            double* w = &Wc[c][(size_t)t * m];
            if (lo) {
                for (int r = 0; r < q; ++r) {
                    const int d = r + q - t;
                    if (d >= 1 && d <= q) v[r] = s.lhs[d - 1];
                }
                b.solve(v);
            }
            if (hi) {
                for (int i = m - q; i < m; ++i) {
                    const int d = m + t - i;
                    if (d >= 1 && d <= q) w[i] = s.lhs[d - 1];
                }
                b.solve(w);
            }
        }
    }
    const int N = 2 * q * P;
    std::vector<double> R((size_t)N * N, 0.0);
    for (int rr = 0; rr < P; ++rr) {
        const int c = rr == 0 ? 0 : (rr == P - 1 ? 2 : 1), m = len[c];
        for (int r = 0; r < q; ++r) {
            const int rh = 2 * q * rr + r, rt = 2 * q * rr + q + r;
            R[(size_t)rh * N + rh] += 1.0;
            R[(size_t)rt * N + rt] += 1.0;
            for (int t = 0; t < q; ++t) {
                if (rr > 0) {
                    const int cprev = 2 * q * (rr - 1) + q + t;
                    R[(size_t)rh * N + cprev] += Vc[c][(size_t)t * m + r];
                    R[(size_t)rt * N + cprev] += Vc[c][(size_t)t * m + (m - q + r)];
                }
                if (rr < P - 1) {
                    const int cnext = 2 * q * (rr + 1) + t;
                    R[(size_t)rh * N + cnext] += Wc[c][(size_t)t * m + r];
                    R[(size_t)rt * N + cnext] += Wc[c][(size_t)t * m + (m - q + r)];
                }
            }
        }
    }
    const std::vector<double> G = dense_inverse(R, N);
    std::vector<double> tab;
    for (int c = 0; c < 3; ++c) {
        sp->off_V[c] = (int64_t)tab.size();
        tab.insert(tab.end(), Vc[c].begin(), Vc[c].end());
        sp->off_W[c] = (int64_t)tab.size();
        tab.insert(tab.end(), Wc[c].begin(), Wc[c].end());
    }
    sp->off_G = (int64_t)tab.size();
    tab.insert(tab.end(), G.begin(), G.end());
    const size_t el = dtype == CLES_F64 ? sizeof(double) : sizeof(float);
    CLES_CUDA(cudaMalloc(&sp->tab, el * tab.size()));
    if (dtype == CLES_F64) {
        CLES_CUDA(cudaMemcpy(sp->tab, tab.data(), sizeof(double) * tab.size(), cudaMemcpyHostToDevice));
    } else {
        std::vector<float> t32(tab.begin(), tab.end());
        CLES_CUDA(cudaMemcpy(sp->tab, t32.data(), sizeof(float) * t32.size(), cudaMemcpyHostToDevice));
    }
    CLES_CUDA(cudaMalloc(&sp->loc, el * (size_t)kSigFields * (size_t)L * (size_t)n));
    for (int c = 0; c < 3; ++c)
        CLES_CUDA(cudaMalloc(&sp->iface[c], el * (size_t)kSigFields * 2 * q * (size_t)sp->cls[c].P.lines));
    plan.sig = std::move(sp);
}

void build_compact_plan(CompactPlan& plan, const cles_scheme& s, const int n3[3], int dim, bool periodic,
                        double h, int dtype, int lo_fold, int hi_fold, bool lo_open, bool hi_open, int pow2_seg_max,
                        int force_S, int force_LB) {
    const int n = n3[dim];
    const int q = s.q, M = s.M, nc = s.nc;
    if (q < 1 || q > CLES_MAX_Q) throw Error(CLES_EINVAL, "scheme LHS half-bandwidth q must be 1 or 2");
    if (M < 1 || M > CLES_MAX_M) throw Error(CLES_EINVAL, "scheme RHS half-width M must be 1..4");
    if (nc < 0 || nc > CLES_MAX_NC) throw Error(CLES_EINVAL, "too many closure rows");
    const int nmin = q >= 2 ? std::max({2 * nc + 1, 2 * M + 1, 2 * q + 1}) : std::max(2 * nc + 1, 2 * M + 1);
    if (n < nmin)
        throw Error(CLES_EINVAL, "local extent " + std::to_string(n) + " along dim " + std::to_string(dim + 1) +
                                     " too small for scheme '" + std::string(s.name) + "' (need >= " +
                                     std::to_string(nmin) + ")");
    if (periodic) lo_fold = hi_fold = 0;
    if (periodic && (lo_open || hi_open)) throw Error(CLES_EINVAL, "a periodic line has no rank interface");
    if (lo_open && lo_fold) lo_fold = 0;
    if (hi_open && hi_fold) hi_fold = 0;
    const bool lo_clo = !periodic && !lo_fold && !lo_open, hi_clo = !periodic && !hi_fold && !hi_open;
    if (M > nc && (lo_clo || hi_clo))
        throw Error(CLES_EINVAL, "closed lines need the RHS half-width M <= closure rows nc (halos are never read)");
    for (int j = 0; j < nc; ++j)
        if (s.clo_len[j] < 0 || s.clo_len[j] > CLES_MAX_CLO_LEN || s.clo_len[j] > n)
            throw Error(CLES_EINVAL, "bad closure stencil length");

    CompactParams& P = plan.P;
    std::memset(&P, 0, sizeof(P));
    P.n = n; P.dim = dim; P.nx = n3[0]; P.ny = n3[1]; P.nz = n3[2];
    P.q = q; P.M = M; P.symmetric = s.symmetric; P.periodic = periodic ? 1 : 0;
    P.lo_closed = (periodic || lo_open) ? 0 : 1;
    P.hi_closed = (periodic || hi_open) ? 0 : 1;
    P.lo_open = lo_open ? 1 : 0;
    P.hi_open = hi_open ? 1 : 0;
    // A folded end carries rows of the interior stencil whose reads beyond the
    // edge are the half-offset mirror f[-1-g] = sigma f[g] (the fold_fill! halo,
    // src/folds.jl:83-124), written as closure rows over the interior; both
    // ends then hold the same number of rows.
    const int ncr = (lo_fold || hi_fold) ? std::max(nc, M) : nc;
    if (ncr > CLES_MAX_NC || ((lo_fold || hi_fold) && ncr + M > CLES_MAX_CLO_LEN))
        throw Error(CLES_EINVAL, "folded rows exceed the closure-row tables");
    if (n < 2 * ncr + 1) throw Error(CLES_EINVAL, "line too short for the folded rows");
    P.nc = ncr;
    P.lines = 1;
    for (int k = 0; k < 3; ++k) if (k != dim) P.lines *= n3[k];
    if (P.lines >= (int64_t)1 << 31) throw Error(CLES_EINVAL, "too many lines for one plan (2^31)");

    // RHS coefficients prescaled by 1/h (derivatives) and the high-edge sign
    // (src/operators.jl:87-92).
    const double hinv = 1.0 / h;
    const double sgn = s.symmetric ? 1.0 : -1.0;
    const double scale = s.symmetric ? 1.0 : hinv;
    P.a0 = s.a0;
    for (int m = 0; m < M; ++m) P.ci[m] = s.coeffs[m] * scale;
    // row r's interior stencil over a line with mirrored ends, as weights per index
    auto folded_row = [&](int r, double* w, int len) {
        std::fill(w, w + len, 0.0);
        auto add = [&](int g, double c) {
            double sg = 1.0;
            if (g < 0) { g = -1 - g; sg = (double)lo_fold; }
            else if (g >= n) { g = 2 * n - 1 - g; sg = (double)hi_fold; }
            w[g] += sg * c;
        };
        if (s.symmetric) add(r, P.a0);
        for (int m = 1; m <= M; ++m) {
            add(r + m, P.ci[m - 1]);
            add(r - m, s.symmetric ? P.ci[m - 1] : -P.ci[m - 1]);
        }
    };
    std::vector<double> wrow((size_t)n, 0.0);
    for (int j = 0; j < ncr; ++j) {
        // low end: row j, stencil on f[0 .. len-1]
        if (lo_fold) {
            const int len = j + M + 1;
            folded_row(j, wrow.data(), n);
            P.clo_len[j] = len;
            for (int t = 0; t < len; ++t) P.clo[j][t] = wrow[t];
        } else {
            for (int t = 0; t < s.clo_len[j]; ++t) P.clo[j][t] = s.clo_rhs[j][t] * scale;
            P.clo_len[j] = s.clo_len[j];
        }
        // high end: row n-1-j, stencil on f[n-1-t]; the table length is shared
        // with the low end (unused weights are zero), so it covers the longer
        if (hi_fold) {
            const int len = j + M + 1;
            folded_row(n - 1 - j, wrow.data(), n);
            for (int t = 0; t < len; ++t) P.chi[j][t] = wrow[n - 1 - t];
            P.clo_len[j] = std::max(P.clo_len[j], len);
        } else {
            for (int t = 0; t < s.clo_len[j]; ++t) P.chi[j][t] = s.clo_rhs[j][t] * (scale * sgn);
            P.clo_len[j] = std::max(P.clo_len[j], s.clo_len[j]);
        }
    }

    // Global band with closures (src/operators.jl:66-84, src/operators_banded.jl:48-112).
    Band B;
    B.n = n; B.q = q; B.periodic = periodic;
    if (periodic) {
        const int W = 2 * q + 1;
        B.a.assign((size_t)n * W, 0.0);
        for (int i = 0; i < n; ++i) {
            B.a[(size_t)i * W + q] = 1.0;
            for (int t = 1; t <= q; ++t) {
                B.a[(size_t)i * W + q + t] = s.lhs[t - 1];
                B.a[(size_t)i * W + q - t] = s.lhs[t - 1];
            }
        }
    } else {
        B.a = make_line_band(s, n, lo_fold, hi_fold, lo_open, hi_open).a;
    }

    // Segmentation: S segments of at most kMaxSeg points, local_range split.
    // Plans of a handful of lines (1-D and very thin 2-D problems) are pure
    // latency: they take segments of 8-16 points, more threads per line.
    P.pcr = (!periodic && q == 1) ? 1 : 0;
    int seg_target = kMaxSeg;
    // a split line's piece of 32 points (or of 16k points, k odd) takes 16-point
    // segments so that it has equal segments, more than one, for the tile kernels
    if ((lo_open || hi_open) && n % 16 == 0 && (n == 32 || n % 32 != 0) && n / 16 <= 8) seg_target = 16;
    if (P.pcr && P.lines <= 16) {
        seg_target = 8;
        while (seg_target < kMaxSeg && (n + seg_target - 1) / seg_target > 512) seg_target *= 2;
    }
    int S = (n + seg_target - 1) / seg_target;
    if (S < 1) S = 1;
    const int base = n / S;
    if (base < std::max(2 * q + 1, q + 1)) S = 1;  // tiny lines: one segment
    if (pow2_seg_max > 0) {
        // batched plans: the fewest power-of-two segments of at most
        // pow2_seg_max points, so that every plan's lines-per-CTA times
        // segments equals the batched launch's thread count
        S = 1;
        while ((n + S - 1) / S > std::min(pow2_seg_max, kMaxSeg)) S *= 2;
        if (n / S < std::max(2 * q + 1, q + 1)) throw Error(CLES_EINVAL, "batched segments too short for the scheme");
    }
    if (force_S > 0) {
        S = force_S;
        if (n / S < std::max(2 * q + 1, q + 1)) throw Error(CLES_EINVAL, "forced segments too short for the scheme");
    }
    P.S = S;
    P.seg_base = n / S;
    P.seg_rem = n % S;
    if (P.seg_base + (P.seg_rem ? 1 : 0) > kMaxSeg) throw Error(CLES_EINVAL, "segment longer than the register tile");
    // cyclic reduction only where the dense inverse would be large (2S > 64);
    // below that one dot product per interface value is cheaper than log2(S) barriers
    if (S == 1 || 2 * S <= 64) P.pcr = 0;
    int LB = 32;
    while (LB > 1 && LB * S > 512) LB /= 2;
    if (dim == 0) {
        // x lines are staged in a transposed shared-memory tile of n x (LB+1)
        const size_t el = dtype == CLES_F64 ? sizeof(double) : sizeof(float);
        while (LB > 1 && (size_t)n * (LB + 1) * el > 110 * 1024) LB /= 2;
        if ((size_t)n * (LB + 1) * el > 200 * 1024) throw Error(CLES_EINVAL, "x line too long for the shared-memory tile");
    }
    if (force_LB > 0) LB = force_LB;
    if (LB * S > 512) throw Error(CLES_EINVAL, "line too long for one CTA");
    const int LB_full = LB;
    if (P.lines < LB && force_LB <= 0) {
        int l = 1;
        while (l < P.lines) l *= 2;
        LB = std::max(1, std::min(LB, l));
    }
    P.LB = LB;
    P.hasred = (periodic || S > 1) ? 1 : 0;

    auto seg_off = [&](int sg) { return sg * P.seg_base + std::min(sg, P.seg_rem); };
    auto seg_len = [&](int sg) { return P.seg_base + (sg < P.seg_rem ? 1 : 0); };

    // Table layout (elements): 5 coefficient arrays [S][kMaxSeg], V/W [S][q][kMaxSeg], G [N][N].
    const int N = 2 * q * S;
    const int64_t arr = (int64_t)S * kMaxSeg;
    P.off_f0 = 0; P.off_f1 = arr; P.off_f2 = 2 * arr; P.off_f3 = 3 * arr; P.off_f4 = 4 * arr;
    P.off_V = 5 * arr;
    P.off_W = P.off_V + (int64_t)S * q * kMaxSeg;
    P.off_G = P.off_W + (int64_t)S * q * kMaxSeg;
    const int L = [&] { int l = 0; while ((1 << l) < S) ++l; return l; }();
    P.pcr_levels = P.pcr ? L : 0;
    // the dense inverse is kept for every plan with a small reduced system
    // (the tile kernel reads it from shared memory), and for all periodic ones
    const bool with_g = P.hasred && (!P.pcr || N <= 64);
    P.off_pcr = P.off_G + (with_g ? (int64_t)N * N : 0);
    const int64_t total = P.off_pcr + (P.pcr ? (int64_t)(L + 1) * S * 8 : 0);
    std::vector<double> tab((size_t)total, 0.0);

    std::vector<LocalFactor> fac(S);
    std::vector<std::vector<double>> Vs(S), Ws(S);
    for (int sg = 0; sg < S; ++sg) {
        const int off = seg_off(sg), m = seg_len(sg);
        LocalFactor& F = fac[sg];
        F.build(B, off, m);
        // coefficients
        for (int i = 0; i < m; ++i) {
            if (q == 1) {
                // Thomas form of the same factorisation: l, 1/pivot, super-diagonal
                tab[P.off_f0 + (size_t)sg * kMaxSeg + i] = i > 0 ? F.L[(size_t)i - 1] : 0.0;
                tab[P.off_f1 + (size_t)sg * kMaxSeg + i] = 1.0 / F.U[i];
                tab[P.off_f2 + (size_t)sg * kMaxSeg + i] = i < m - 1 ? F.U[(size_t)m + i] : 0.0;
            } else {
                tab[P.off_f0 + (size_t)sg * kMaxSeg + i] = F.L[i];                       // eliminates row i+1
                tab[P.off_f1 + (size_t)sg * kMaxSeg + i] = F.L[(size_t)m + i];           // eliminates row i+2
                tab[P.off_f2 + (size_t)sg * kMaxSeg + i] = F.U[(size_t)m + i];           // U[i, i+1]
                tab[P.off_f3 + (size_t)sg * kMaxSeg + i] = F.U[(size_t)2 * m + i];       // U[i, i+2]
                tab[P.off_f4 + (size_t)sg * kMaxSeg + i] = 1.0 / F.U[i];
            }
        }
        // spikes: V[:, t] = T^-1 (coupling of rows 0..q-1 to the previous
        // segment's tail unknown t), W[:, t] likewise for the next head.
        Vs[sg].assign((size_t)q * m, 0.0);
        Ws[sg].assign((size_t)q * m, 0.0);
        const bool has_prev = periodic || sg > 0;
        const bool has_next = periodic || sg < S - 1;
        const int prev = (sg - 1 + S) % S, next = (sg + 1) % S;
        for (int t = 0; t < q; ++t) {
            std::vector<double> v(m, 0.0), w(m, 0.0);
            bool nzv = false, nzw = false;
            if (has_prev) {
                const int col = seg_off(prev) + seg_len(prev) - q + t;  // tail unknown t of prev
                for (int r = 0; r < std::min(q, m); ++r) { v[r] = B.at(off + r, col); nzv = nzv || v[r] != 0.0; }
            }
            if (has_next) {
                const int col = seg_off(next) + t;  // head unknown t of next
                for (int r = std::max(0, m - q); r < m; ++r) { w[r] = B.at(off + r, col); nzw = nzw || w[r] != 0.0; }
            }
            if (nzv) F.solve(v.data());
            if (nzw) F.solve(w.data());
            for (int i = 0; i < m; ++i) {
                Vs[sg][(size_t)t * m + i] = v[i];
                Ws[sg][(size_t)t * m + i] = w[i];
                tab[P.off_V + ((size_t)sg * q + t) * kMaxSeg + i] = v[i];
                tab[P.off_W + ((size_t)sg * q + t) * kMaxSeg + i] = w[i];
            }
        }
    }
    if (P.pcr) {
        // Interface system of a closed tridiagonal line in X_s = (head_s, tail_s):
        //   X_s + A_s X_{s-1} + C_s X_{s+1} = (y_s[0], y_s[m-1]),
        //   A_s = [[0, v_s[0]], [0, v_s[m-1]]], C_s = [[w_s[0], 0], [w_s[m-1], 0]],
        // A_0 = C_{S-1} = 0.  Cyclic reduction level l (distance k = 2^l), all
        // segments at once from the previous level's blocks:
        //   alpha = -A_s B_{s-k}^-1, gamma = -C_s B_{s+k}^-1 (zero past the ends),
        //   B_s += alpha C_{s-k} + gamma A_{s+k}, A_s = alpha A_{s-k}, C_s = gamma C_{s+k},
        // and on the device R_s += alpha R_{s-k} + gamma R_{s+k}.  After
        // ceil(log2 S) levels no coupling is left and X_s = B_s^-1 R_s.
        std::vector<std::array<double, 4>> A(S), Bm(S), C(S);
        for (int sg = 0; sg < S; ++sg) {
            const int m = seg_len(sg);
            A[sg] = {0.0, Vs[sg][0], 0.0, Vs[sg][(size_t)m - 1]};
            C[sg] = {Ws[sg][0], 0.0, Ws[sg][(size_t)m - 1], 0.0};
            Bm[sg] = {1.0, 0.0, 0.0, 1.0};
        }
        for (int l = 0; l < L; ++l) {
            const int k = 1 << l;
            std::vector<std::array<double, 4>> nA(S), nB(S), nC(S);
            for (int sg = 0; sg < S; ++sg) {
                double al[4] = {0, 0, 0, 0}, ga[4] = {0, 0, 0, 0}, t[4], bi[4];
                nB[sg] = Bm[sg];
                nA[sg] = {0, 0, 0, 0};
                nC[sg] = {0, 0, 0, 0};
                if (sg - k >= 0) {
                    mat2_inv(Bm[sg - k].data(), bi);
                    mat2_mul(A[sg].data(), bi, al);
                    for (double& e : al) e = -e;
                    mat2_mul(al, C[sg - k].data(), t);
                    for (int e = 0; e < 4; ++e) nB[sg][e] += t[e];
                    mat2_mul(al, A[sg - k].data(), nA[sg].data());
                }
                if (sg + k < S) {
                    mat2_inv(Bm[sg + k].data(), bi);
                    mat2_mul(C[sg].data(), bi, ga);
                    for (double& e : ga) e = -e;
                    mat2_mul(ga, A[sg + k].data(), t);
                    for (int e = 0; e < 4; ++e) nB[sg][e] += t[e];
                    mat2_mul(ga, C[sg + k].data(), nC[sg].data());
                }
                double* dst = &tab[P.off_pcr + ((size_t)l * S + sg) * 8];
                for (int e = 0; e < 4; ++e) { dst[e] = al[e]; dst[4 + e] = ga[e]; }
            }
            A.swap(nA);
            Bm.swap(nB);
            C.swap(nC);
        }
        for (int sg = 0; sg < S; ++sg) mat2_inv(Bm[sg].data(), &tab[P.off_pcr + ((size_t)L * S + sg) * 8]);
    }
    if (with_g) {
        // Reduced system in z = (head_0, tail_0, head_1, tail_1, ...), 2q per segment.
        std::vector<double> R((size_t)N * N, 0.0);
        for (int sg = 0; sg < S; ++sg) {
            const int m = seg_len(sg);
            const int prev = (sg - 1 + S) % S, next = (sg + 1) % S;
            for (int r = 0; r < q; ++r) {
                const int rh = 2 * q * sg + r, rt = 2 * q * sg + q + r;
                R[(size_t)rh * N + rh] += 1.0;
                R[(size_t)rt * N + rt] += 1.0;
                for (int t = 0; t < q; ++t) {
                    const int cprev = 2 * q * prev + q + t, cnext = 2 * q * next + t;
                    R[(size_t)rh * N + cprev] += Vs[sg][(size_t)t * m + r];
                    R[(size_t)rt * N + cprev] += Vs[sg][(size_t)t * m + (m - q + r)];
                    R[(size_t)rh * N + cnext] += Ws[sg][(size_t)t * m + r];
                    R[(size_t)rt * N + cnext] += Ws[sg][(size_t)t * m + (m - q + r)];
                }
            }
        }
        std::vector<double> G = dense_inverse(R, N);
        std::copy(G.begin(), G.end(), tab.begin() + P.off_G);
    }

    build_warp_line(plan, B, s, n, dim, periodic);
    plan.has_tl = false;
    if (q == 1 && periodic && dim > 0 && P.seg_rem == 0 && n <= 256 && LB_full == 32) {
        TileLineParams& T = plan.TL;
        std::memset(&T, 0, sizeof(T));
        T.m = P.seg_base;
        for (int i = 0; i < T.m; ++i) {
            T.l[i] = tab[P.off_f0 + i];
            T.dinv[i] = tab[P.off_f1 + i];
            T.c[i] = tab[P.off_f2 + i];
            T.v[i] = tab[P.off_V + i];
            T.w[i] = tab[P.off_W + i];
            T.lf[i] = (float)T.l[i]; T.dinvf[i] = (float)T.dinv[i]; T.cf[i] = (float)T.c[i];
            T.vf[i] = (float)T.v[i]; T.wf[i] = (float)T.w[i];
        }
        // every segment of a periodic line with equal segments is the same block
        bool same = true;
        for (int sg = 1; sg < S && same; ++sg)
            for (int i = 0; i < T.m; ++i) {
                const size_t o = (size_t)sg * kMaxSeg + i;
                same = same && tab[P.off_f0 + o] == T.l[i] && tab[P.off_f1 + o] == T.dinv[i] &&
                       tab[P.off_f2 + o] == T.c[i] && tab[P.off_V + o] == T.v[i] && tab[P.off_W + o] == T.w[i];
            }
        plan.has_tl = same;
    }
    // general tile kernels (closed or periodic lines, q = 1 or the C10
    // pentadiagonal; y/z lines by TMA tiles, x lines by cp.async transposed
    // tiles): equal segments of 16 or 32 points, at most 8 per line
    plan.has_tg = false;
    if (with_g && P.seg_rem == 0 && (P.seg_base == 16 || P.seg_base == 32) && S * 32 <= 256 && n <= 256 &&
        ((q == 1 && (M == 1 || M == 2 || M == 4)) || (q == 2 && M == 3))) {
        TileGenParams& G = plan.TG;
        std::memset(&G, 0, sizeof(G));
        const int nf = q == 1 ? 3 : 5;
        const int64_t offs[5] = {P.off_f0, P.off_f1, P.off_f2, P.off_f3, P.off_f4};
        const int src[3] = {0, S > 2 ? 1 : 0, S - 1};
        bool alike = true;   // interior segments must all be equal to segment 1
        for (int sg = 2; sg < S - 1 && alike; ++sg)
            for (int i = 0; i < P.seg_base; ++i) {
                for (int a = 0; a < nf; ++a)
                    alike = alike && tab[offs[a] + (size_t)sg * kMaxSeg + i] == tab[offs[a] + (size_t)kMaxSeg + i];
                for (int t = 0; t < q; ++t) {
                    alike = alike && tab[P.off_V + ((size_t)sg * q + t) * kMaxSeg + i] ==
                                         tab[P.off_V + ((size_t)q + t) * kMaxSeg + i];
                    alike = alike && tab[P.off_W + ((size_t)sg * q + t) * kMaxSeg + i] ==
                                         tab[P.off_W + ((size_t)q + t) * kMaxSeg + i];
                }
            }
        for (int cls = 0; cls < 3; ++cls) {
            const int sg = src[cls];
            for (int i = 0; i < kMaxSeg; ++i) {
                for (int a = 0; a < nf; ++a) G.f[cls][a][i] = tab[offs[a] + (size_t)sg * kMaxSeg + i];
                for (int t = 0; t < q; ++t) {
                    G.v[cls][t][i] = tab[P.off_V + ((size_t)sg * q + t) * kMaxSeg + i];
                    G.w[cls][t][i] = tab[P.off_W + ((size_t)sg * q + t) * kMaxSeg + i];
                }
            }
        }
        for (int cls = 0; cls < 3; ++cls)
            for (int i = 0; i < kMaxSeg; ++i) {
                for (int a = 0; a < 5; ++a) G.ff[cls][a][i] = (float)G.f[cls][a][i];
                for (int t = 0; t < 2; ++t) {
                    G.vf[cls][t][i] = (float)G.v[cls][t][i];
                    G.wf[cls][t][i] = (float)G.w[cls][t][i];
                }
            }
        plan.has_tg = alike;
    }

    plan.dtype = dtype;
    plan.tab_elems = (size_t)total;
    CLES_CUDA(cudaMalloc(&plan.tab64, sizeof(double) * total));
    CLES_CUDA(cudaMemcpy(plan.tab64, tab.data(), sizeof(double) * total, cudaMemcpyHostToDevice));
    if (dtype == CLES_F32) {
        std::vector<float> t32(tab.begin(), tab.end());
        CLES_CUDA(cudaMalloc(&plan.tab32, sizeof(float) * total));
        CLES_CUDA(cudaMemcpy(plan.tab32, t32.data(), sizeof(float) * total, cudaMemcpyHostToDevice));
    }
    // a handful of long closed x lines is latency-bound in one CTA per line:
    // cut it into pieces solved side by side (SigPlan)
    if (dim == 0 && !periodic && !lo_fold && !hi_fold && !lo_open && !hi_open && pow2_seg_max == 0 &&
        force_S == 0 && P.lines <= 16 && n >= 2048 && (n3[1] == 1 || n3[2] == 1))
        build_sig_plan(plan, s, n3, h, dtype);
}

SigPlan::~SigPlan() {
    if (tab) cudaFree(tab);
    if (loc) cudaFree(loc);
    for (void* p : iface)
        if (p) cudaFree(p);
}

SplitPlan::~SplitPlan() {
    if (tab) cudaFree(tab);
}

void build_split_plan(SplitPlan& sp, const cles_scheme& s, const int n3[3], int dim, bool periodic, int n_global,
                      int ranks, int rank, double h, int dtype) {
    if (ranks < 1 || rank < 0 || rank >= ranks) throw Error(CLES_EINVAL, "rank must lie in [0, ranks)");
    if (dim < 0 || dim > 2) throw Error(CLES_EINVAL, "dim must be 1, 2 or 3");
    const int q = s.q;
    if (q < 1 || q > CLES_MAX_Q) throw Error(CLES_EINVAL, "scheme LHS half-bandwidth q must be 1 or 2");
    // every rank's extent (src/decomposition.jl:73-78)
    auto range = [&](int r, int* nr, int* off) {
        const int base = n_global / ranks, rem = n_global % ranks;
        *nr = base + (r < rem ? 1 : 0);
        *off = r * base + std::min(r, rem);
    };
    int nr = 0, off = 0;
    range(rank, &nr, &off);
    if (n3[dim] != nr)
        throw Error(CLES_EINVAL, "local extent " + std::to_string(n3[dim]) + " along dim " + std::to_string(dim + 1) +
                                     " is not rank " + std::to_string(rank) + "'s share " + std::to_string(nr) +
                                     " of " + std::to_string(n_global));
    // the smallest piece decides, so every rank refuses the same split
    // (src/operators.jl:50-53, src/operators_banded.jl:37-41)
    const int nmin = q >= 2 ? std::max({2 * s.nc + 1, 2 * s.M + 1, 2 * q + 1}) : std::max(2 * s.nc + 1, 2 * s.M + 1);
    if (n_global / ranks < nmin)
        throw Error(CLES_EINVAL, "local extent " + std::to_string(n_global / ranks) + " along dim " +
                                     std::to_string(dim + 1) + " too small for scheme '" + std::string(s.name) +
                                     "' (need >= " + std::to_string(nmin) + ")");
    sp.ranks = ranks; sp.rank = rank; sp.dim = dim; sp.q = q; sp.M = s.M; sp.n = nr; sp.dtype = dtype;
    for (int k = 0; k < 3; ++k) sp.n3[k] = n3[k];
    sp.lo_open = periodic || rank > 0;
    sp.hi_open = periodic || rank < ranks - 1;
    sp.prev = sp.lo_open ? (rank - 1 + ranks) % ranks : -1;
    sp.next = sp.hi_open ? (rank + 1) % ranks : -1;
    build_compact_plan(sp.local, s, n3, dim, false, h, dtype, 0, 0, sp.lo_open, sp.hi_open);
    sp.lines = sp.local.P.lines;

    // rank-level spikes of every rank and the reduced system in
    // z = (head_0, tail_0, head_1, tail_1, ...), 2q per rank
    const int N = 2 * q * ranks;
    std::vector<double> R((size_t)N * N, 0.0);
    std::vector<double> Vme, Wme;
    for (int rr = 0; rr < ranks; ++rr) {
        int m = 0, o = 0;
        range(rr, &m, &o);
        const bool lo = periodic || rr > 0, hi = periodic || rr < ranks - 1;
        LineBand b = make_line_band(s, m, 0, 0, lo, hi);
        b.factor();
        std::vector<double> V((size_t)q * m, 0.0), W((size_t)q * m, 0.0);
        for (int t = 0; t < q; ++t) {
            double* v = &V[(size_t)t * m];
            double* w = &W[(size_t)t * m];
            // row r couples to the previous rank's tail unknown t at distance
            // r + q - t, row i to the next rank's head unknown t at m + t - i
            if (lo) {
                for (int r = 0; r < q; ++r) {
                    const int d = r + q - t;
                    if (d >= 1 && d <= q) v[r] = s.lhs[d - 1];
                }
                b.solve(v);
            }
            if (hi) {
                for (int i = m - q; i < m; ++i) {
                    const int d = m + t - i;
                    if (d >= 1 && d <= q) w[i] = s.lhs[d - 1];
                }
                b.solve(w);
            }
        }
        const int prev = (rr - 1 + ranks) % ranks, next = (rr + 1) % ranks;
        for (int r = 0; r < q; ++r) {
            const int rh = 2 * q * rr + r, rt = 2 * q * rr + q + r;
            R[(size_t)rh * N + rh] += 1.0;
            R[(size_t)rt * N + rt] += 1.0;
            for (int t = 0; t < q; ++t) {
                const int cprev = 2 * q * prev + q + t, cnext = 2 * q * next + t;
                R[(size_t)rh * N + cprev] += V[(size_t)t * m + r];
                R[(size_t)rt * N + cprev] += V[(size_t)t * m + (m - q + r)];
                R[(size_t)rh * N + cnext] += W[(size_t)t * m + r];
                R[(size_t)rt * N + cnext] += W[(size_t)t * m + (m - q + r)];
            }
        }
        if (rr == rank) { Vme = std::move(V); Wme = std::move(W); }
    }
    const std::vector<double> G = dense_inverse(R, N);
    const size_t nv = (size_t)q * nr;
    std::vector<double> tab(2 * nv + (size_t)2 * q * N, 0.0);
    std::copy(Vme.begin(), Vme.end(), tab.begin());
    std::copy(Wme.begin(), Wme.end(), tab.begin() + nv);
    double* Gs = tab.data() + 2 * nv;
    for (int t = 0; t < q; ++t) {
        if (sp.lo_open)
            for (int j = 0; j < N; ++j) Gs[(size_t)t * N + j] = G[(size_t)(2 * q * sp.prev + q + t) * N + j];
        if (sp.hi_open)
            for (int j = 0; j < N; ++j) Gs[(size_t)(q + t) * N + j] = G[(size_t)(2 * q * sp.next + t) * N + j];
    }
    if (dtype == CLES_F64) {
        CLES_CUDA(cudaMalloc(&sp.tab, sizeof(double) * tab.size()));
        CLES_CUDA(cudaMemcpy(sp.tab, tab.data(), sizeof(double) * tab.size(), cudaMemcpyHostToDevice));
    } else {
        std::vector<float> t32(tab.begin(), tab.end());
        CLES_CUDA(cudaMalloc(&sp.tab, sizeof(float) * t32.size()));
        CLES_CUDA(cudaMemcpy(sp.tab, t32.data(), sizeof(float) * t32.size(), cudaMemcpyHostToDevice));
    }
}

}  // namespace cles
