// Device-resident solver runtime.
//
// Orchestrates the kernels of compact.cu and pointwise.cu in the order of the
// reference's compute_rhs! (src/rhs.jl:624-694), step! (src/timestep.jl:72-99),
// max_rate (:125-175), filter_state! (:414-426) and run! (:277-405).  All
// fields live on the device in the interior layout (x fastest, no halos);
// periodic wraps and closed-edge closures are handled inside the kernels, so
// the reference's halo exchanges have no device counterpart.

#include "solver.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>

namespace cles {

void DevBuf::alloc(cles_ctx* c, size_t b) {
    release();
    ctx = c;
    if (b == 0) return;
    if (ctx->budget && ctx->allocated + b > ctx->budget)
        throw Error(CLES_ENOMEM, "HBM budget exceeded: need " + std::to_string(ctx->allocated + b) + " bytes of " +
                                     std::to_string(ctx->budget));
    cudaError_t e = cudaMalloc(&p, b);
    if (e != cudaSuccess) {
        p = nullptr;
        cudaGetLastError();
        throw Error(CLES_ENOMEM, std::string("cudaMalloc failed: ") + cudaGetErrorString(e));
    }
    bytes = b;
    ctx->allocated += b;
}

void DevBuf::release() {
    if (p) {
        cudaFree(p);
        if (ctx) ctx->allocated -= bytes;
    }
    p = nullptr;
    bytes = 0;
}

// LSRK(5,4) coefficients (src/timestep.jl:5-21)
const double kLsrkA[5] = {0.0, -567301805773.0 / 1357537059087.0, -2404267990393.0 / 2016746695238.0,
                          -3550918686646.0 / 2091501179385.0, -1275806237668.0 / 842570457699.0};
const double kLsrkB[5] = {1432997174477.0 / 9575080441755.0, 5161836677717.0 / 13612068292357.0,
                          1720146321549.0 / 2090206949498.0, 3134564353537.0 / 4481467310338.0,
                          2277821191437.0 / 14882151754819.0};
const double kLsrkC[5] = {0.0, 1432997174477.0 / 9575080441755.0, 2526269341429.0 / 6820363962896.0,
                          2006345519317.0 / 3224310063776.0, 2802321613138.0 / 2924317926251.0};

namespace {

const double (&RKA)[5] = kLsrkA;
const double (&RKB)[5] = kLsrkB;
const double (&RKC)[5] = kLsrkC;
const double PLANCK_TIME = 5.391247e-44;

inline double jmax(double x, double y) {
    if (std::isnan(x)) return x;
    if (std::isnan(y)) return y;
    return y > x ? y : x;
}
inline double jmin(double x, double y) {
    if (std::isnan(x)) return x;
    if (std::isnan(y)) return y;
    return y < x ? y : x;
}

template <typename F>
class Solver final : public SolverBase {
public:
    Solver(cles_ctx* ctx, const cles_solver_desc& d, const cles_decomp* dc = nullptr,
           const cles_exchange* ex = nullptr)
        : ctx_(ctx) {
        desc = d;
        st_ = ctx->stream;
        for (int k = 0; k < 3; ++k) {
            const bool p0 = d.bc[k][0] == CLES_BC_PERIODIC, p1 = d.bc[k][1] == CLES_BC_PERIODIC;
            if (p0 != p1) throw Error(CLES_EINVAL, "dimension " + std::to_string(k + 1) + " mixes periodic and non-periodic conditions");
            if (d.n_global[k] < 1) throw Error(CLES_EINVAL, "n_global must be >= 1");
            if (d.n_global[k] == 1 && !p0) throw Error(CLES_EINVAL, "collapsed dimension must use (PeriodicBC(), PeriodicBC())");
            for (int s = 0; s < 2; ++s) {
                if (d.bc[k][s] < CLES_BC_PERIODIC || d.bc[k][s] > CLES_BC_POLE)
                    throw Error(CLES_EINVAL, "unknown boundary condition");
                if (d.bc_switchable[k][s]) {
                    // SwitchableBC(before, after) (src/boundary.jl:113-148)
                    if (d.bc_after[k][s] < CLES_BC_PERIODIC || d.bc_after[k][s] > CLES_BC_POLE)
                        throw Error(CLES_EINVAL, "unknown boundary condition");
                    if (is_fold_bc(d.bc[k][s]) || is_fold_bc(d.bc_after[k][s]))
                        throw Error(CLES_EINVAL, "SwitchableBC cannot wrap a fold condition (AxisBC, OriginBC, PoleBC); "
                                                 "setup detects those by type");
                    if ((d.bc_after[k][s] == CLES_BC_PERIODIC) != (d.bc[k][s] == CLES_BC_PERIODIC))
                        throw Error(CLES_EINVAL, "SwitchableBC: both conditions must agree on periodicity");
                }
            }
            g_.n[k] = d.n_global[k];
            g_.active[k] = d.n_global[k] > 1;
            g_.periodic[k] = g_.active[k] ? p0 : 1;
            pad_[k] = g_.active[k] ? d.n_halo : 0;
            h_[k] = !g_.active[k] ? 1.0 : (g_.periodic[k] ? d.L[k] / d.n_global[k] : d.L[k] / (d.n_global[k] - 1));
        }
        if (dc) decompose(d, *dc, ex);
        if (d.n_species < 1 || d.n_species > CLES_MAX_SPECIES) throw Error(CLES_EINVAL, "bad species count");
        if (d.beta_sensor < 0 || d.beta_sensor > 2) throw Error(CLES_EINVAL, "unknown beta sensor");
        if (d.n_body_forces < 0 || d.n_body_forces > CLES_MAX_BODY_FORCES)
            throw Error(CLES_EINVAL, "at most 4 body forces");
        Ns_ = d.n_species;
        ncons_ = Ns_ + 4;
        if (d.eos != CLES_EOS_IDEAL && d.eos != CLES_EOS_NASA9) throw Error(CLES_EINVAL, "unknown equation of state");
        for (int k = 0; k < Ns_; ++k) {
            pc_.Rk[k] = d.R[k];
            pc_.cvk[k] = d.eos == CLES_EOS_IDEAL ? d.R[k] / (d.gamma[k] - 1) : 0.0;
            pc_.cpk[k] = pc_.Rk[k] + pc_.cvk[k];
        }
        nasa9_setup(pc_, d);
        cells_ = (int64_t)g_.n[0] * g_.n[1] * g_.n[2];
        cfl = d.cfl;
        setup_geometry(d);
        if (decomposed_) check_decomposable(d);
        const int dt = sizeof(F) == 8 ? CLES_F64 : CLES_F32;
        for (int k = 0; k < 3; ++k) {
            if (!g_.active[k]) continue;
            if (split_[k].on) {
                build_split_plans(d, k, dt);
                continue;
            }
            // a folded dim carries one plan per field parity (src/rhs.jl:256-261)
            const int nt = fold_[k].on ? 2 : 1;
            for (int t = 0; t < nt; ++t) {
                const int sg = t == 0 ? 1 : -1;
                const int lo = fold_[k].on && fold_[k].lo ? sg : 0, hi = fold_[k].on && fold_[k].hi ? sg : 0;
                deriv_[k][t].reset(new CompactPlan());
                build_compact_plan(*deriv_[k][t], d.deriv, g_.n, k, g_.periodic[k] != 0, h_[k], dt, lo, hi);
                filt_[k][t].reset(new CompactPlan());
                build_compact_plan(*filt_[k][t], d.filt, g_.n, k, g_.periodic[k] != 0, h_[k], dt, lo, hi);
                if (dt != CLES_F64) {
                    qfilt_[k][t].reset(new CompactPlan());
                    build_compact_plan(*qfilt_[k][t], d.filt, g_.n, k, g_.periodic[k] != 0, h_[k], CLES_F64, lo, hi);
                }
                dset_[k][t] = deriv_[k][t].get();
                fset_[k][t] = filt_[k][t].get();
                qset_[k][t] = qfilt_[k][t] ? qfilt_[k][t].get() : filt_[k][t].get();
                if (fold_[k].paired) {
                    // the same plan over the lines of one half of the pairing
                    // dimension: each parity then runs over its own half only
                    int nh[3] = {g_.n[0], g_.n[1], g_.n[2]};
                    nh[fold_[k].pp.sd] /= 2;
                    hderiv_[k][t].reset(new CompactPlan());
                    build_compact_plan(*hderiv_[k][t], d.deriv, nh, k, false, h_[k], dt, lo, hi);
                    hfilt_[k][t].reset(new CompactPlan());
                    build_compact_plan(*hfilt_[k][t], d.filt, nh, k, false, h_[k], dt, lo, hi);
                    if (dt != CLES_F64) {
                        hqfilt_[k][t].reset(new CompactPlan());
                        build_compact_plan(*hqfilt_[k][t], d.filt, nh, k, false, h_[k], CLES_F64, lo, hi);
                    }
                    hdset_[k][t] = hderiv_[k][t].get();
                    hfset_[k][t] = hfilt_[k][t].get();
                    hqset_[k][t] = hqfilt_[k][t] ? hqfilt_[k][t].get() : hfilt_[k][t].get();
                }
            }
        }
        const size_t c = (size_t)cells_;
        Q_.alloc(ctx, sizeof(double) * c * ncons_);
        du_.alloc(ctx, sizeof(double) * c * ncons_);
        dQ_.alloc(ctx, sizeof(F) * c * ncons_);
        prim_.alloc(ctx, sizeof(F) * c * (P_Y0 + Ns_ + 1));  // + the kappa*-sensor input
        g_u_.alloc(ctx, sizeof(F) * c * 9);
        gty_.alloc(ctx, sizeof(F) * c * 3 * (1 + Ns_));
        art_.alloc(ctx, sizeof(F) * c * (A_D0 + Ns_));
        scratch_.alloc(ctx, sizeof(F) * c * 5);
        flux_.alloc(ctx, sizeof(F) * c * 3 * ncons_);
        part_.alloc(ctx, sizeof(double) * 2 * (size_t)(rate_partials(cells_) + 1));
        res_.alloc(ctx, sizeof(double) * 4);
        CLES_CUDA(cudaMallocHost(&host_res_, sizeof(double) * 4));
        // du, gradients of collapsed dims and the artificial properties start
        // at zero, as after allocation in the reference
        CLES_CUDA(cudaMemsetAsync(Q_.p, 0, Q_.bytes, st_));
        CLES_CUDA(cudaMemsetAsync(du_.p, 0, du_.bytes, st_));
        CLES_CUDA(cudaMemsetAsync(dQ_.p, 0, dQ_.bytes, st_));
        CLES_CUDA(cudaMemsetAsync(prim_.p, 0, prim_.bytes, st_));
        CLES_CUDA(cudaMemsetAsync(g_u_.p, 0, g_u_.bytes, st_));
        CLES_CUDA(cudaMemsetAsync(gty_.p, 0, gty_.bytes, st_));
        CLES_CUDA(cudaMemsetAsync(art_.p, 0, art_.bytes, st_));
        CLES_CUDA(cudaMemsetAsync(scratch_.p, 0, scratch_.bytes, st_));
        CLES_CUDA(cudaMemsetAsync(flux_.p, 0, flux_.bytes, st_));
        if (d.control.retries > 0) save_.alloc(ctx, sizeof(double) * c * ncons_);
        if (decomposed_) alloc_split_buffers();
        if (geo_) build_geometry_tables(d);
        // the Stretch samples are read at create time only (kept in stretch_x_)
        for (int k = 0; k < 3; ++k) desc.stretch_x[k] = desc.stretch_dxdxi[k] = nullptr;
        CLES_CUDA(cudaStreamSynchronize(st_));
    }

    ~Solver() override {
        graph_free();
        if (cap_st_) cudaStreamDestroy(cap_st_);
        if (host_res_) cudaFreeHost(host_res_);
        if (host_clk_) cudaFreeHost(host_clk_);
    }

    // ------------------------------------------------------ decomposition --
    // Decomp(n_global, periodic; dims) on this rank (src/decomposition.jl:80-122):
    // the local extents and offsets by local_range, before any plan is built.
    void decompose(const cles_solver_desc& d, const cles_decomp& dc, const cles_exchange* ex) {
        if (!ex || !ex->halo || !ex->gather || !ex->allreduce)
            throw Error(CLES_EINVAL, "a decomposed solver needs halo, gather and allreduce callbacks");
        ex_ = *ex;
        dc_ = dc;
        for (int k = 0; k < 3; ++k) {
            if (dc.dims[k] < 1) throw Error(CLES_EINVAL, "process grid dims must be >= 1");
            if (!g_.active[k] && dc.dims[k] != 1)
                throw Error(CLES_EINVAL, "collapsed dimensions must not be decomposed: dims=(" +
                                             std::to_string(dc.dims[0]) + ", " + std::to_string(dc.dims[1]) + ", " +
                                             std::to_string(dc.dims[2]) + ")");
            if (dc.coords[k] < 0 || dc.coords[k] >= dc.dims[k])
                throw Error(CLES_EINVAL, "rank coordinates must lie in [0, dims)");
            const int N = d.n_global[k], P = dc.dims[k], r = dc.coords[k];
            const int base = N / P, rem = N % P;
            g_.n[k] = base + (r < rem ? 1 : 0);
            off_[k] = r * base + std::min(r, rem);
            if (g_.n[k] < 1) throw Error(CLES_EINVAL, "a rank's local extent is empty");
            split_[k].on = P > 1;
            if (split_[k].on) decomposed_ = true;
        }
        // a process grid of one rank is the ordinary solver
    }

    void check_decomposable(const cles_solver_desc& d) {
        if (geo_)
            throw Error(CLES_EINVAL, "a decomposed solver needs a uniform Cartesian grid (no metric, stretching or folds)");
        for (int k = 0; k < 3; ++k) {
            if (!split_[k].on) continue;
            for (int s = 0; s < 2; ++s)
                for (int w = 0; w < 2; ++w) {
                    const int bc = w == 0 ? d.bc[k][s] : (d.bc_switchable[k][s] ? d.bc_after[k][s] : -1);
                    if (bc == CLES_BC_NSCBC_OUTFLOW || bc == CLES_BC_NSCBC_INFLOW)
                        throw Error(CLES_EINVAL, "characteristic (NSCBC) faces on a decomposed dimension are not "
                                                 "supported");
                }
        }
    }

    // LineSolver / BandLineSolver with P > 1 (src/tridiag.jl:85-170,
    // src/banded.jl:108-214) for the derivative and the filter along a split
    // dim; their local plans stand in the plan sets.
    void build_split_plans(const cles_solver_desc& d, int k, int dt) {
        Split& S = split_[k];
        const bool per = g_.periodic[k] != 0;
        S.deriv.reset(new SplitPlan());
        build_split_plan(*S.deriv, d.deriv, g_.n, k, per, d.n_global[k], dc_.dims[k], dc_.coords[k], h_[k], dt);
        S.filt.reset(new SplitPlan());
        build_split_plan(*S.filt, d.filt, g_.n, k, per, d.n_global[k], dc_.dims[k], dc_.coords[k], h_[k], dt);
        if (dt != CLES_F64) {
            S.qfilt.reset(new SplitPlan());
            build_split_plan(*S.qfilt, d.filt, g_.n, k, per, d.n_global[k], dc_.dims[k], dc_.coords[k], h_[k],
                             CLES_F64);
        }
        dset_[k][0] = &S.deriv->local;
        fset_[k][0] = &S.filt->local;
        qset_[k][0] = S.qfilt ? &S.qfilt->local : &S.filt->local;
        S.lines = S.deriv->lines;
        S.prev = S.deriv->prev;
        S.next = S.deriv->next;
        S.lo_open = S.deriv->lo_open;
        S.hi_open = S.deriv->hi_open;
        hpad_ = std::max({hpad_, S.deriv->M, S.filt->M, 2});
    }

    // Padded copy of the fields of one split application and the exchange
    // buffers of every split dim (8-byte elements: the FP64 state filter).
    void alloc_split_buffers() {
        int64_t padded = 0;
        for (int k = 0; k < 3; ++k) {
            Split& S = split_[k];
            if (!S.on) continue;
            padded = std::max(padded, cells_ / g_.n[k] * (g_.n[k] + 2 * hpad_));
            const size_t halo = sizeof(double) * (size_t)ncons_ * hpad_ * (size_t)S.lines;
            const size_t iface = sizeof(double) * (size_t)ncons_ * 2 * CLES_MAX_Q * (size_t)S.lines;
            S.send_lo.alloc(ctx_, halo);
            S.send_hi.alloc(ctx_, halo);
            S.recv_lo.alloc(ctx_, halo);
            S.recv_hi.alloc(ctx_, halo);
            S.iface.alloc(ctx_, iface);
            S.zbuf.alloc(ctx_, iface);
            S.iface_all.alloc(ctx_, iface * (size_t)dc_.dims[k]);
        }
        padbuf_.alloc(ctx_, sizeof(double) * (size_t)ncons_ * (size_t)padded);
    }

    // The fields of one application along split dim k, with hpad_ halo planes
    // beyond each end of the dim (element size esz).
    FieldView padded_view(int k, size_t esz) const {
        int np[3] = {g_.n[0], g_.n[1], g_.n[2]};
        np[k] += 2 * hpad_;
        const int64_t sy = np[0], sz = (int64_t)np[0] * np[1];
        const int64_t lead = (int64_t)hpad_ * (k == 0 ? 1 : k == 1 ? sy : sz);
        return FieldView{static_cast<char*>(padbuf_.p) + esz * (size_t)lead, sz * np[2], sy, sz};
    }

    void exchange_halo(int k, int64_t bytes) {
        Split& S = split_[k];
        if (ex_.halo(ex_.user, k, S.prev, S.next, S.send_lo.p, S.send_hi.p, S.recv_lo.p, S.recv_hi.p, bytes,
                     reinterpret_cast<void*>(st_)) != 0)
            throw Error(CLES_EXCHANGE, "halo exchange along dim " + std::to_string(k + 1) + " failed");
    }

    void allreduce(int op, double* v, int n) {
        if (ex_.allreduce(ex_.user, op, v, n) != 0) throw Error(CLES_EXCHANGE, "allreduce failed");
    }

    // apply_along! on split dim k (src/operators.jl:118-131 with P > 1 ranks):
    // the fields are copied into the padded buffer, the M planes next to each
    // rank interface are exchanged into its halo, the local solve with open
    // ends writes `loc` and every line's heads and tails, which are gathered
    // along the dim; the correction then writes `out` by mode (OUT_STORE,
    // OUT_NEGATE, or OUT_SUBTRACT with loc distinct from out).
    void split_apply(const SplitPlan& P, int k, const void* in, void* loc, void* out, int count, int mode) {
        Split& S = split_[k];
        const size_t esz = P.dtype == CLES_F64 ? sizeof(double) : sizeof(float);
        if (count > ncons_) throw Error(CLES_EINVAL, "internal: too many fields for a split application");
        const FieldView vin = view(const_cast<void*>(in));
        const FieldView pv = padded_view(k, esz);
        copy_view(vin, pv, g_.n, count, P.dtype, st_);
        split_halo(P, vin, S.send_lo.p, S.send_hi.p, count, true, st_);
        exchange_halo(k, (int64_t)(esz * (size_t)count * P.M * (size_t)P.lines));
        split_halo(P, pv, S.recv_lo.p, S.recv_hi.p, count, false, st_);
        launch_compact_split(P.local, pv, view(loc), count, S.iface.p, st_);
        const int64_t ib = (int64_t)(esz * (size_t)count * 2 * P.q * (size_t)P.lines);
        if (ex_.gather(ex_.user, k, S.iface.p, S.iface_all.p, ib, reinterpret_cast<void*>(st_)) != 0)
            throw Error(CLES_EXCHANGE, "interface gather along dim " + std::to_string(k + 1) + " failed");
        split_correct(P, S.iface_all.p, S.zbuf.p, view(loc), view(out), count, mode, st_);
    }

    const SplitPlan& split_plan_of(const CompactPlan* const* ps, int k) const {
        const Split& S = split_[k];
        if (ps == dset_[k]) return *S.deriv;
        if (ps == fset_[k]) return *S.filt;
        if (ps == qset_[k]) return S.qfilt ? *S.qfilt : *S.filt;
        throw Error(CLES_EINVAL, "internal: no split plan for this operator");
    }

    // delta4_sum! of one or two fields (src/artificial.jl:67-94); on a
    // decomposed grid the two planes beyond each rank interface of every split
    // dim are exchanged first (the reference's exchange_halos! before it).
    void delta4(const F* f0, const F* f1, F* o0, F* o1, const double w0[3], const double w1[3]) {
        if (!decomposed_) {
            Pointwise<F>::delta4_tiled(f0, f1, o0, o1, g_, w0, w1, st_);
            return;
        }
        Halo4 h{};
        Grid3 gl = g_;
        const int dt = sizeof(F) == 8 ? CLES_F64 : CLES_F32;
        for (int k = 0; k < 3; ++k) {
            Split& S = split_[k];
            if (!S.on) continue;
            gl.periodic[k] = 0;
            HaloSpec hs;
            hs.dim = k;
            for (int e = 0; e < 3; ++e) hs.n3[e] = g_.n[e];
            hs.M = 2;
            hs.lines = S.lines;
            hs.lo_open = S.lo_open;
            hs.hi_open = S.hi_open;
            const size_t fb = sizeof(F) * 2 * (size_t)S.lines;
            halo_planes(hs, view(const_cast<F*>(f0)), S.send_lo.p, S.send_hi.p, 1, true, dt, st_);
            if (f1)
                halo_planes(hs, view(const_cast<F*>(f1)), static_cast<char*>(S.send_lo.p) + fb,
                            static_cast<char*>(S.send_hi.p) + fb, 1, true, dt, st_);
            exchange_halo(k, (int64_t)(fb * (f1 ? 2 : 1)));
            h.lo[k] = S.recv_lo.p;
            h.hi[k] = S.recv_hi.p;
            h.open_lo[k] = S.lo_open ? 1 : 0;
            h.open_hi[k] = S.hi_open ? 1 : 0;
        }
        Pointwise<F>::delta4_halo(f0, f1, o0, o1, gl, w0, w1, h, st_);
    }

    // at_lo_edge / at_hi_edge (src/decomposition.jl:137-140): the faces of a
    // split dim belong to the first and the last rank along it
    bool owns_face(int k, int s) const {
        if (!split_[k].on) return true;
        return s == 0 ? dc_.coords[k] == 0 : dc_.coords[k] == dc_.dims[k] - 1;
    }

    const cles_decomp* decomposition() const override { return decomposed_ ? &dc_ : nullptr; }

    // ----------------------------------------------------------- geometry --
    static bool is_fold_bc(int bc) { return bc == CLES_BC_AXIS || bc == CLES_BC_ORIGIN || bc == CLES_BC_POLE; }
    static bool unit_scalefactor(int metric, int k) {
        // unit_scalefactor (src/metric.jl:91-93)
        if (metric == CLES_METRIC_CYLINDRICAL) return k != 1;
        if (metric == CLES_METRIC_SPHERICAL) return k == 0;
        return true;
    }

    // The geometry part of Solver(...) (src/rhs.jl:143-311): validation of the
    // metric, stretching and folds, grid spacing with half-offset folded
    // dims, the fold specs with their velocity and flux parities.
    void setup_geometry(const cles_solver_desc& d) {
        if (d.metric < CLES_METRIC_CARTESIAN || d.metric > CLES_METRIC_SPHERICAL)
            throw Error(CLES_EINVAL, "unknown metric");
        bool str[3];
        for (int k = 0; k < 3; ++k) {
            str[k] = d.stretch_x[k] != nullptr;
            if (str[k] != (d.stretch_dxdxi[k] != nullptr))
                throw Error(CLES_EINVAL, "a Stretch needs both x and dx/dxi samples");
            stretched_[k] = str[k];
            if (str[k]) stretch_x_[k].assign(d.stretch_x[k], d.stretch_x[k] + d.n_global[k]);
        }
        geo_ = d.metric != CLES_METRIC_CARTESIAN || str[0] || str[1] || str[2];
        for (int k = 0; k < 3; ++k)
            for (int s = 0; s < 2; ++s)
                for (int w = 0; w < 2; ++w) {
                    const int bc = w == 0 ? d.bc[k][s] : (d.bc_switchable[k][s] ? d.bc_after[k][s] : -1);
                    if (bc != CLES_BC_NSCBC_OUTFLOW && bc != CLES_BC_NSCBC_INFLOW) continue;
                    if (!unit_scalefactor(d.metric, k))
                        throw Error(CLES_EINVAL, "characteristic boundary conditions need a face whose normal metric "
                                                 "scale factor is one");
                }
        const bool axis = d.bc[0][0] == CLES_BC_AXIS, orig1 = d.bc[0][0] == CLES_BC_ORIGIN;
        const bool pole_l = d.bc[1][0] == CLES_BC_POLE, pole_h = d.bc[1][1] == CLES_BC_POLE;
        if (pole_l != pole_h) throw Error(CLES_EINVAL, "PoleBC must be applied at both ends of θ");
        const bool poles = pole_l;
        const double PI = 3.14159265358979323846;
        if (axis) {
            if (d.metric != CLES_METRIC_CYLINDRICAL) throw Error(CLES_EINVAL, "AxisBC requires CylindricalMetric");
            if (str[0]) throw Error(CLES_EINVAL, "folded dimensions cannot be stretched");
            if (!(std::fabs(d.origin[0]) < 1e-14)) throw Error(CLES_EINVAL, "AxisBC requires origin[1] = 0");
            if (!(d.n_global[1] == 1 || d.n_global[1] % 2 == 0))
                throw Error(CLES_EINVAL, "resolved-θ AxisBC requires an even θ point count over 2π");
        }
        if (orig1) {
            if (d.metric != CLES_METRIC_SPHERICAL) throw Error(CLES_EINVAL, "OriginBC requires SphericalMetric");
            if (str[0]) throw Error(CLES_EINVAL, "folded dimensions cannot be stretched");
            if (!(std::fabs(d.origin[0]) < 1e-14)) throw Error(CLES_EINVAL, "OriginBC requires origin[1] = 0");
            if (!(d.n_global[2] == 1 || d.n_global[2] % 2 == 0))
                throw Error(CLES_EINVAL, "resolved-φ OriginBC requires an even φ point count over 2π");
            if (!(d.n_global[1] == 1 || std::fabs(2 * d.origin[1] + d.L[1] - PI) <= 1e-10))
                throw Error(CLES_EINVAL, "OriginBC requires a θ range symmetric about π/2");
            if (d.n_global[2] == 1 && d.n_global[1] > 1 && d.n_global[1] % 2 != 0)
                throw Error(CLES_EINVAL, "OriginBC pairs θ with π - θ: the θ point count must be even");
        }
        if (poles) {
            if (d.metric != CLES_METRIC_SPHERICAL) throw Error(CLES_EINVAL, "PoleBC requires SphericalMetric");
            if (str[1]) throw Error(CLES_EINVAL, "folded dimensions cannot be stretched");
            if (!(std::fabs(d.origin[1]) < 1e-14 && std::fabs(d.L[1] - PI) <= 1e-10))
                throw Error(CLES_EINVAL, "PoleBC requires the θ domain (0, π)");
            if (!(d.n_global[2] == 1 || d.n_global[2] % 2 == 0))
                throw Error(CLES_EINVAL, "resolved-φ PoleBC requires an even φ point count over 2π");
        }
        if (axis || orig1) g_.periodic[0] = 0;
        if (poles) g_.periodic[1] = 0;
        for (int k = 0; k < 3; ++k)
            if (str[k] && g_.periodic[k])
                throw Error(CLES_EINVAL, "dimension " + std::to_string(k + 1) + ": stretched dimensions must be non-periodic");
        if (d.metric != CLES_METRIC_CARTESIAN &&
            ((g_.active[0] && g_.periodic[0]) || (d.metric == CLES_METRIC_SPHERICAL && g_.active[1] && g_.periodic[1])))
            throw Error(CLES_EINVAL, "a periodic radial (or spherical polar) dimension is not supported");
        // grid spacing (src/rhs.jl:191-205)
        const bool flo[3] = {axis || orig1, poles, false}, fhi[3] = {false, poles, false};
        for (int k = 0; k < 3; ++k) {
            const int n = d.n_global[k];
            if (!g_.active[k]) h_[k] = 1.0;
            else if (str[k]) h_[k] = 1.0 / (n - 1);
            else if (flo[k] && fhi[k]) h_[k] = d.L[k] / n;
            else if (flo[k]) h_[k] = d.L[k] / (n - 0.5);
            else h_[k] = g_.periodic[k] ? d.L[k] / n : d.L[k] / (n - 1);
            shift_[k] = flo[k] ? h_[k] / 2 : 0.0;
            orig_[k] = str[k] ? 0.0 : d.origin[k];
        }
        // fold specs (src/rhs.jl:216-280, src/equations.jl:56-67)
        auto foldspec = [&](int k, bool lo, bool hi, int pdim, int revdim, const int sv[3], int area_parity) {
            Fold& f = fold_[k];
            f.on = true; f.lo = lo; f.hi = hi;
            for (int j = 0; j < 3; ++j) f.sigvel[j] = sv[j];
            for (int c = 0; c < ncons_; ++c) {
                const int cp = (c < Ns_ || c == Ns_ + 3) ? 1 : sv[c - Ns_];
                f.sigflux[c] = cp * sv[k] * area_parity;
                f.sigcons[c] = cp;
            }
            const bool shift = pdim >= 0 && g_.active[pdim], rev = revdim >= 0 && g_.active[revdim];
            f.paired = shift || rev;
            for (int j = 0; j < 3; ++j) f.pp.n[j] = g_.n[j];
            f.pp.pdim = shift ? pdim : -1;
            f.pp.revdim = rev ? revdim : -1;
            f.pp.sd = shift ? pdim : revdim;
            if (shift && g_.n[pdim] % 2 != 0)
                throw Error(CLES_EINVAL, "pairing dim " + std::to_string(pdim + 1) + " local extent must be even");
        };
        if (axis) {
            const int sv[3] = {-1, -1, 1};
            foldspec(0, true, false, 1, -1, sv, -1);   // A_1 = r is odd
        } else if (orig1) {
            const int sv[3] = {-1, 1, -1};
            foldspec(0, true, false, 2, 1, sv, 1);     // A_1 = r^2 sin(theta) is even
        }
        if (poles) {
            const int sv[3] = {1, -1, -1};
            foldspec(1, true, true, 2, -1, sv, -1);    // A_2 = r sin(theta) is odd in theta
        }
        for (int k = 0; k < 3; ++k)
            if (fold_[k].on) folded_ = true;
    }

    // Node tables of Geom (x, dx/dxi per dimension, sin/cos of theta) and the
    // GCL-corrected cot(theta)/r of a resolved spherical theta.
    void build_geometry_tables(const cles_solver_desc& d) {
        std::vector<double> tab;
        size_t off[8];
        for (int k = 0; k < 3; ++k) {
            const int n = g_.n[k];
            off[k] = tab.size();
            for (int i = 0; i < n; ++i)
                tab.push_back(stretched_[k] ? d.stretch_x[k][i] : orig_[k] + shift_[k] + (double)i * h_[k]);
            off[3 + k] = tab.size();
            for (int i = 0; i < n; ++i) tab.push_back(stretched_[k] ? d.stretch_dxdxi[k][i] : 1.0);
        }
        off[6] = tab.size();
        for (int j = 0; j < g_.n[1]; ++j) tab.push_back(std::sin(tab[off[1] + j]));
        off[7] = tab.size();
        for (int j = 0; j < g_.n[1]; ++j) tab.push_back(std::cos(tab[off[1] + j]));
        geo_tab_.alloc(ctx_, sizeof(double) * tab.size());
        CLES_CUDA(cudaMemcpy(geo_tab_.p, tab.data(), sizeof(double) * tab.size(), cudaMemcpyHostToDevice));
        const double* b = geo_tab_.as<double>();
        G_.metric = d.metric;
        for (int k = 0; k < 3; ++k) {
            G_.n[k] = g_.n[k];
            G_.x[k] = b + off[k];
            G_.m[k] = b + off[3 + k];
        }
        G_.sn = b + off[6];
        G_.cs = b + off[7];
        G_.cotr = nullptr;
        if (folded_) pairbuf_.alloc(ctx_, sizeof(double) * (size_t)cells_ * std::max(ncons_, 3 + Ns_));
        if (d.metric == CLES_METRIC_SPHERICAL && g_.active[1]) {
            // gcl_cotr! (src/metric.jl:154-170) in FP64 in every precision mode:
            // D_theta(A_theta) with the theta-momentum flux's fold sign
            DevBuf a2, da;
            a2.alloc(ctx_, sizeof(double) * (size_t)cells_);
            da.alloc(ctx_, sizeof(double) * (size_t)cells_);
            cotr_.alloc(ctx_, sizeof(double) * (size_t)cells_);
            geo_area(a2.as<double>(), 1, G_, st_);
            const int sig = fold_[1].on ? fold_[1].sigflux[Ns_ + 1] : 1;
            std::unique_ptr<CompactPlan> tmp[2], htmp[2];
            const CompactPlan* ps[2] = {dset_[1][0], dset_[1][1]};
            const CompactPlan* hs[2] = {hdset_[1][0], hdset_[1][1]};
            if (sizeof(F) != 8) {
                const int nt = fold_[1].on ? 2 : 1;
                for (int t = 0; t < nt; ++t) {
                    const int sg = t == 0 ? 1 : -1;
                    const int lo = fold_[1].on && fold_[1].lo ? sg : 0, hi = fold_[1].on && fold_[1].hi ? sg : 0;
                    tmp[t].reset(new CompactPlan());
                    build_compact_plan(*tmp[t], d.deriv, g_.n, 1, g_.periodic[1] != 0, h_[1], CLES_F64, lo, hi);
                    ps[t] = tmp[t].get();
                    if (fold_[1].paired) {
                        int nh[3] = {g_.n[0], g_.n[1], g_.n[2]};
                        nh[fold_[1].pp.sd] /= 2;
                        htmp[t].reset(new CompactPlan());
                        build_compact_plan(*htmp[t], d.deriv, nh, 1, false, h_[1], CLES_F64, lo, hi);
                        hs[t] = htmp[t].get();
                    }
                }
            }
            const int sgs[1] = {sig};
            along_set(ps, 1, a2.p, da.p, 1, OUT_STORE, sgs, hs);
            geo_gcl(cotr_.as<double>(), da.as<double>(), G_, st_);
            CLES_CUDA(cudaStreamSynchronize(st_));
            G_.cotr = cotr_.as<double>();
        }
    }

    // deriv_along! / filt_along! routing (src/rhs.jl:452-475, src/folds.jl:
    // 276-322) over `count` adjacent fields with antipodal parities sig[c]
    // (nullptr = all +1).  ps[0] is the plan of parity +1 (the only one off a
    // fold), ps[1] that of parity -1.  Off a fold or on a self-paired fold the
    // parity is inside the plan's mirror rows (one launch per run of equal
    // parity).  A paired fold runs the even/odd butterfly: the even
    // combination with the field's parity over the canonical half of the
    // pairing dimension and the odd one with parity -1 over the partner half
    // (hs: the same plans over half the lines), then the inverse butterfly in
    // place.  The reference applies both parities to every line and keeps
    // one half of each result; the halves kept are the same.
    const CompactPlan* const* half_of(const CompactPlan* const* ps, int k) const {
        if (ps == dset_[k]) return hdset_[k];
        if (ps == fset_[k]) return hfset_[k];
        if (ps == qset_[k]) return hqset_[k];
        return nullptr;
    }
    void along_set(const CompactPlan* const* ps, int k, const void* in, void* out, int count, int mode,
                   const int* sig, const CompactPlan* const* hs = nullptr) {
        const size_t esz = ps[0]->dtype == CLES_F64 ? sizeof(double) : sizeof(float);
        auto at = [&](const void* base, int c) {
            return reinterpret_cast<void*>(const_cast<char*>(static_cast<const char*>(base)) + esz * (size_t)cells_ * c);
        };
        if (split_[k].on) {
            if (mode != OUT_STORE && mode != OUT_NEGATE)
                throw Error(CLES_EINVAL, "internal: a split application stores or negates");
            split_apply(split_plan_of(ps, k), k, in, out, out, count, mode);
            return;
        }
        const Fold& f = fold_[k];
        if (!f.on) {
            launch_compact(*ps[0], view(const_cast<void*>(in)), view(out), count, mode, st_);
            return;
        }
        auto sg = [&](int c) { return sig ? sig[c] : 1; };
        if (!f.paired) {
            for (int c0 = 0; c0 < count;) {
                int c1 = c0 + 1;
                while (c1 < count && sg(c1) == sg(c0)) ++c1;
                launch_compact(*ps[sg(c0) > 0 ? 0 : 1], view(at(in, c0)), view(at(out, c0)), c1 - c0, mode, st_);
                c0 = c1;
            }
            return;
        }
        if (mode != OUT_STORE) throw Error(CLES_EINVAL, "a paired fold stores its result");
        if (!hs) hs = half_of(ps, k);
        if (!hs || !hs[0] || !hs[1]) throw Error(CLES_EINVAL, "internal: no half-grid plans for a paired fold");
        const int64_t sd_stride = f.pp.sd == 0 ? 1 : f.pp.sd == 1 ? (int64_t)g_.n[0] : (int64_t)g_.n[0] * g_.n[1];
        const int64_t upper = sd_stride * (g_.n[f.pp.sd] / 2);
        auto half_view = [&](void* base, bool up) {
            FieldView v = view(base);
            v.base = static_cast<char*>(base) + (up ? esz * (size_t)upper : 0);
            return v;
        };
        void* w = pairbuf_.p;
        for (int c0 = 0; c0 < count;) {
            int c1 = c0 + 1;
            while (c1 < count && sg(c1) == sg(c0)) ++c1;
            const int s = sg(c0), run = c1 - c0;
            if (esz == sizeof(double))
                pair_forward<double>(static_cast<const double*>(at(in, c0)), static_cast<double*>(at(w, c0)), run,
                                     cells_, f.pp, s, st_);
            else
                pair_forward<float>(static_cast<const float*>(at(in, c0)), static_cast<float*>(at(w, c0)), run, cells_,
                                    f.pp, s, st_);
            // even combination, folded with the field's parity (src/folds.jl:296-299)
            launch_compact(*hs[s > 0 ? 0 : 1], half_view(at(w, c0), false), half_view(at(out, c0), false), run,
                           OUT_STORE, st_);
            c0 = c1;
        }
        // odd combination, always folded as odd (src/folds.jl:300-301)
        launch_compact(*hs[1], half_view(w, true), half_view(out, true), count, OUT_STORE, st_);
        for (int c0 = 0; c0 < count;) {
            int c1 = c0 + 1;
            while (c1 < count && sg(c1) == sg(c0)) ++c1;
            if (esz == sizeof(double))
                pair_backward<double>(static_cast<double*>(at(out, c0)), c1 - c0, cells_, f.pp, sg(c0), st_);
            else
                pair_backward<float>(static_cast<float*>(at(out, c0)), c1 - c0, cells_, f.pp, sg(c0), st_);
            c0 = c1;
        }
    }

    // ------------------------------------------------------------- views --
    FieldView view(void* p) const { return FieldView{p, cells_, g_.n[0], (int64_t)g_.n[0] * g_.n[1]}; }
    F* prim(int slot) const { return prim_.as<F>() + (size_t)cells_ * slot; }
    F* scratch(int k) const { return scratch_.as<F>() + (size_t)cells_ * k; }

    // --------------------------------------------------------- operators --
    void smooth(F* f, int count) {
        // smooth! (src/artificial.jl:98-111): one filter pass per active dim, in
        // place, over `count` adjacent fields
        for (int k = 0; k < 3; ++k)
            if (g_.active[k]) along_set(fset_[k], k, f, f, count, OUT_STORE, nullptr);
    }

    // The condition face (k, s) acts as now: a switchable face forwards to its
    // `after` condition once switched (src/boundary.jl:170-183).
    int face_kind(int k, int s) const {
        return desc.bc_switchable[k][s] && switched_[k][s] ? desc.bc_after[k][s] : desc.bc[k][s];
    }
    const cles_bc_params& face_params(int k, int s) const {
        return desc.bc_switchable[k][s] && switched_[k][s] ? desc.bc_after_params[k][s] : desc.bc_params[k][s];
    }
    const double* face_state(int k, int s) const {
        return desc.bc_switchable[k][s] && switched_[k][s] ? desc.bc_after_state[k][s] : desc.bc_state[k][s];
    }
    // a DirichletBC(fun) / NSCBCInflowBC(target = fun) face function and the
    // face's node coordinates
    struct FaceFn {
        cles_face_fn fn = nullptr;
        void* user = nullptr;
        std::vector<double> x[3];
    };
    // the face function of the condition face (k, s) acts as now, if any
    const FaceFn& face_fn(int k, int s) const {
        return face_fn_[k][s][desc.bc_switchable[k][s] && switched_[k][s] ? 1 : 0];
    }
    void set_face_fn(int k, int s, int which, cles_face_fn fn, void* user) override {
        if (k < 0 || k > 2 || s < 0 || s > 1 || which < 0 || which > 1) throw Error(CLES_EINVAL, "no such face");
        if (which == 1 && !desc.bc_switchable[k][s]) throw Error(CLES_EINVAL, "face is not a SwitchableBC");
        const int bc = which == 0 ? desc.bc[k][s] : desc.bc_after[k][s];
        if (fn && bc != CLES_BC_DIRICHLET && bc != CLES_BC_NSCBC_INFLOW)
            throw Error(CLES_EINVAL, "only DirichletBC and NSCBCInflowBC faces take a function");
        FaceFn& f = face_fn_[k][s][which];
        f.fn = fn;
        f.user = user;
        if (fn && f.x[0].empty()) {
            // node coordinates of the face in plane order (xcoord, src/rhs.jl:320-335)
            const int o1 = k == 0 ? 1 : 0, o2 = k == 2 ? 1 : 2;
            const int64_t np = (int64_t)g_.n[o1] * g_.n[o2];
            for (int e = 0; e < 3; ++e) f.x[e].resize((size_t)np);
            for (int64_t t = 0; t < np; ++t) {
                int c[3];
                c[o1] = (int)(t % g_.n[o1]);
                c[o2] = (int)(t / g_.n[o1]);
                c[k] = s == 0 ? 0 : g_.n[k] - 1;
                for (int e = 0; e < 3; ++e) f.x[e][(size_t)t] = node_coord(e, off_[e] + c[e]);
            }
        }
    }
    // physical coordinate of interior node i along e (global_xcoord, src/rhs.jl:331-335)
    double node_coord(int e, int i) const {
        return stretched_[e] ? stretch_x_[e][(size_t)i] : orig_[e] + shift_[e] + (double)i * h_[e];
    }
    // Evaluate a face function at the stage time into the device face buffer;
    // returns the device pointer ([values][plane]).
    const double* eval_face_fn(int k, int s, int nvals) {
        const FaceFn& f = face_fn(k, s);
        const int64_t np = (int64_t)f.x[0].size();
        face_host_.assign((size_t)(np * nvals), std::numeric_limits<double>::quiet_NaN());
        f.fn(f.user, k, s, tstage, np, f.x[0].data(), f.x[1].data(), f.x[2].data(), face_host_.data());
        const size_t bytes = sizeof(double) * face_host_.size();
        if (face_dev_.bytes < bytes) {
            CLES_CUDA(cudaStreamSynchronize(st_));
            face_dev_.release();
            face_dev_.alloc(ctx_, bytes);
        }
        // pageable source: the call returns once the data is staged, so the
        // host buffer may be refilled by the next evaluation
        CLES_CUDA(cudaMemcpyAsync(face_dev_.p, face_host_.data(), bytes, cudaMemcpyHostToDevice, st_));
        return face_dev_.as<double>();
    }
    bool any_nscbc() const {
        for (int k = 0; k < 3; ++k)
            for (int s = 0; s < 2; ++s)
                if (g_.active[k] && (face_kind(k, s) == CLES_BC_NSCBC_OUTFLOW || face_kind(k, s) == CLES_BC_NSCBC_INFLOW))
                    return true;
        return false;
    }
    void switch_bc(int k, int s) override {
        if (k < 0 || k > 2 || s < 0 || s > 1 || !desc.bc_switchable[k][s])
            throw Error(CLES_EINVAL, "face is not a SwitchableBC");
        switched_[k][s] = true;
    }
    bool bc_switched(int k, int s) const override {
        if (k < 0 || k > 2 || s < 0 || s > 1) throw Error(CLES_EINVAL, "no such face");
        return switched_[k][s];
    }

    void apply_bcs() override {
        // apply_bcs! (src/boundary.jl:280-286): active dims, low then high face
        for (int k = 0; k < 3; ++k) {
            if (!g_.active[k]) continue;
            for (int s = 0; s < 2; ++s) {
                const int bc = face_kind(k, s);
                if (bc == CLES_BC_PERIODIC || bc == CLES_BC_NSCBC_OUTFLOW || bc == CLES_BC_NSCBC_INFLOW) continue;
                if (is_fold_bc(bc)) continue;   // enforce! is a no-op on folds (src/boundary.jl:173-175)
                if (!owns_face(k, s)) continue;
                BcState bs;
                std::memset(&bs, 0, sizeof(bs));
                const double* q = face_state(k, s);
                for (int c = 0; c < ncons_; ++c) bs.q[c] = q[c];
                if (bc == CLES_BC_NOSLIP_WALL) {
                    const double Tw = face_params(k, s).Twall;
                    bs.iso = std::isnan(Tw) ? 0 : 1;
                    bs.Twall = Tw;
                    bs.ew_times_T = desc.eos == CLES_EOS_IDEAL ? 1 : 0;
                    if (bs.iso)
                        for (int sp = 0; sp < Ns_; ++sp)
                            bs.ew[sp] = desc.eos == CLES_EOS_IDEAL ? pc_.cvk[sp] : nasa9_species_energy(desc, sp, Tw);
                }
                const double* qface = nullptr;
                if (bc == CLES_BC_DIRICHLET && face_fn(k, s).fn) qface = eval_face_fn(k, s, ncons_);
                bc_plane(Q_.as<double>(), g_, k, s, Ns_, bc, bs, st_, qface);
            }
        }
    }

    // correct_rhs! of the characteristic faces (src/rhs.jl:688-691), after the
    // flux divergence and before any RK update
    void correct_rhs_nscbc() {
        for (int k = 0; k < 3; ++k) {
            if (!g_.active[k]) continue;
            for (int s = 0; s < 2; ++s) {
                const int bc = face_kind(k, s);
                if (bc != CLES_BC_NSCBC_OUTFLOW && bc != CLES_BC_NSCBC_INFLOW) continue;
                const cles_bc_params& bp = face_params(k, s);
                NscbcParams np;
                std::memset(&np, 0, sizeof(np));
                np.kind = bc;
                for (int j = 0; j < 3; ++j) np.act[j] = g_.active[j];
                np.Lref = bp.Lref > 0 ? bp.Lref : desc.L[k];
                np.pinf = bp.pinf; np.sigma = bp.sigma; np.beta_t = bp.beta_t;
                for (int j = 0; j < 3; ++j) np.u[j] = bp.u[j];
                np.T = bp.T_ion;
                for (int sp = 0; sp < Ns_; ++sp) np.Y[sp] = bp.Y[sp];
                np.eta_u = bp.eta_u; np.eta_T = bp.eta_T; np.eta_t = bp.eta_t; np.eta_Y = bp.eta_Y;
                // one-sided derivatives from the closure rows (full-field applications);
                // scratch 0, 3, 4 are free once the fluxes are assembled (2 holds the
                // last sensor, which get_field exposes)
                F* dpd = scratch(0);
                F* dt0 = scratch(3);
                F* dt1 = scratch(4);
                along_set(dset_[k], k, prim(P_P), dpd, 1, OUT_STORE, nullptr);
                const int t1 = k == 0 ? 1 : 0, t2 = k == 2 ? 1 : 2;
                F* drd = nullptr;
                if (bc == CLES_BC_NSCBC_OUTFLOW) {
                    if (g_.active[t1]) along_set(dset_[t1], t1, prim(P_P), dt0, 1, OUT_STORE, nullptr);
                    if (g_.active[t2]) along_set(dset_[t2], t2, prim(P_P), dt1, 1, OUT_STORE, nullptr);
                } else {
                    drd = dt0;
                    along_set(dset_[k], k, prim(P_RHO), drd, 1, OUT_STORE, nullptr);
                }
                const double* tgt = nullptr;
                if (bc == CLES_BC_NSCBC_INFLOW && face_fn(k, s).fn) tgt = eval_face_fn(k, s, 4 + Ns_);
                Pointwise<F>::nscbc(dQ_.as<F>(), prim_.as<F>(), g_u_.as<F>(), gty_.as<F>(), Ns_ == 1 ? 1 : 1 + Ns_, dpd,
                                    dt0, dt1, drd, g_, k, s, Ns_, pc_, np, st_, tgt, geo_ ? &G_ : nullptr);
            }
        }
    }

    void compute_artificial() {
        // compute_artificial! (src/artificial.jl:261-359).  The strain and the
        // internal-energy sensor chains are independent, so their fourth
        // differences are one tiled pass, their smoothing one batched filter
        // launch per direction, and mu*, beta*, kappa* one pointwise pass; each
        // field sees the reference's operations in the reference's order.
        if (!desc.art_enabled) return;
        using PW = Pointwise<F>;
        F* strain = scratch(0);
        F* sensor = scratch(1);     // smoothed strain sensor
        F* sensor_e = scratch(2);   // smoothed internal-energy sensor (adjacent: batched smoothing)
        F* tmp_a = scratch(3);
        F* tmp_b = scratch(4);
        const double w2[3] = {h_[0] * h_[0], h_[1] * h_[1], h_[2] * h_[2]};
        const double w1[3] = {h_[0], h_[1], h_[2]};
        PW::strain(g_u_.as<F>(), strain, cells_, st_);
        delta4(strain, prim(P_Y0 + Ns_), sensor, sensor_e, w2, w1);
        smooth(sensor, 2);
        PW::art_coef(sensor, sensor_e, prim_.as<F>(), g_u_.as<F>(), art_.as<F>(), cells_, desc.C_mu, desc.C_beta,
                     desc.C_kappa, desc.beta_sensor == CLES_BETA_GATED_STRAIN, st_);
        if (desc.beta_sensor == CLES_BETA_DILATATION) {
            PW::dilatation(g_u_.as<F>(), tmp_a, tmp_b, cells_, st_);
            delta4(tmp_a, nullptr, sensor, nullptr, w2, w2);
            smooth(sensor, 1);
            PW::beta_dilatation(sensor, prim_.as<F>(), tmp_b, art_.as<F>(), cells_, desc.C_beta, st_);
        }
        if (Ns_ > 1) {
            for (int sp = 0; sp < Ns_; ++sp) {
                delta4(prim(P_Y0 + sp), nullptr, tmp_a, nullptr, w1, w1);
                smooth(tmp_a, 1);
                PW::dart(tmp_a, prim_.as<F>(), art_.as<F>(), cells_, desc.C_D, sp, st_);
            }
        }
    }

    void compute_rhs(bool primitives_current) override { compute_rhs_impl(primitives_current, nullptr); }

    // Returns true when `rk` was applied inside the last divergence launch.
    bool compute_rhs_impl(bool primitives_current, const RkEpilogue* rk) {
        using PW = Pointwise<F>;
        const bool nscbc = any_nscbc();
        const bool sources = desc.n_body_forces > 0;
        // the boundary correction and the sources come between the divergence and the update
        if (nscbc || sources) rk = nullptr;
        if (!primitives_current) PW::primitives(Q_.as<double>(), prim_.as<F>(), cells_, Ns_, pc_, st_, desc.art_enabled);
        velocity_gradients();
        compute_artificial();
        // temperature and mass-fraction gradients (src/rhs.jl:628-636); with one
        // species only dT (the species diffusion flux vanishes, see k_fluxes)
        const int ngty = Ns_ == 1 ? 1 : 1 + Ns_;
        for (int k = 0; k < 3; ++k)
            if (g_.active[k])
                along_set(dset_[k], k, prim(P_T), gty_.as<F>() + (size_t)cells_ * ngty * k, ngty, OUT_STORE, nullptr);
        if (geo_) {
            MetricOps<F>::scale_grad(gty_.as<F>(), ngty, G_, g_, st_);
            PW::fluxes_geo(Q_.as<double>(), prim_.as<F>(), g_u_.as<F>(), gty_.as<F>(), art_.as<F>(), flux_.as<F>(),
                           cells_, Ns_, pc_, desc.mu0, desc.Pr, desc.Sc, G_, st_);
            // general path (src/rhs.jl:669-687): D_d(A_d F_d) in place over the
            // flux block, then dQ = -sum_d inv_J D_d(A_d F_d) + metric sources
            for (int k = 0; k < 3; ++k) {
                if (!g_.active[k]) continue;
                F* fk = flux_.as<F>() + (size_t)cells_ * ncons_ * k;
                along_set(dset_[k], k, fk, fk, ncons_, OUT_STORE, fold_[k].on ? fold_[k].sigflux : nullptr);
            }
            MetricOps<F>::metric_div(dQ_.as<F>(), flux_.as<F>(), ncons_, Ns_, prim_.as<F>(), g_u_.as<F>(), art_.as<F>(),
                                     desc.mu0, G_, g_, st_);
            if (nscbc) correct_rhs_nscbc();
            if (sources) add_sources();
            return false;
        }
        PW::fluxes(Q_.as<double>(), prim_.as<F>(), g_u_.as<F>(), gty_.as<F>(), art_.as<F>(), flux_.as<F>(), cells_, Ns_,
                   pc_, desc.mu0, desc.Pr, desc.Sc, st_);
        // flux divergence dQ[c] = -sum_d D_d(F_dc) (src/rhs.jl:650-668), accumulated in the store.
        // With all three dims active the order is y, x, z: the first direction only
        // stores (no read of dQ), the x kernel reads dQ with vector loads, and z,
        // last, carries the RK update.  The sum differs from x, y, z by rounding.
        // On a decomposed grid the split dims come first, each corrected
        // straight into dQ (negated or subtracted) from its local solution
        // written over its own flux block; the last unsplit dim may carry the
        // RK update.
        int order[3] = {0, 1, 2};
        if (decomposed_) {
            int no = 0;
            for (int k = 0; k < 3; ++k)
                if (split_[k].on) order[no++] = k;
            for (int k = 0; k < 3; ++k)
                if (!split_[k].on) order[no++] = k;
        } else if (g_.active[0] && g_.active[1] && g_.active[2]) {
            order[0] = 1;
            order[1] = 0;
        }
        int last = -1;
        for (int o = 0; o < 3; ++o)
            if (g_.active[order[o]]) last = order[o];
        bool first = true, fused = false;
        for (int o = 0; o < 3; ++o) {
            const int k = order[o];
            if (!g_.active[k]) continue;
            F* fk = flux_.as<F>() + (size_t)cells_ * ncons_ * k;
            const FieldView fin = view(fk);
            if (split_[k].on) {
                split_apply(*split_[k].deriv, k, fk, fk, dQ_.p, ncons_, first ? OUT_NEGATE : OUT_SUBTRACT);
            } else if (k == last && !first && rk &&
                       launch_compact_rk(*dset_[k][0], fin, view(dQ_.as<F>()), ncons_, *rk, st_)) {
                fused = true;
            } else {
                launch_compact(*dset_[k][0], fin, view(dQ_.as<F>()), ncons_, first ? OUT_NEGATE : OUT_SUBTRACT, st_);
            }
            first = false;
        }
        if (first) CLES_CUDA(cudaMemsetAsync(dQ_.p, 0, dQ_.bytes, st_));
        if (nscbc) correct_rhs_nscbc();
        if (sources) add_sources();
        return fused;
    }

    void step(double dt, bool prepared) override {
        for (int stage = 0; stage < 5; ++stage) {
            tstage = t + RKC[stage] * dt;
            const bool first_prepared = prepared && stage == 0;
            if (!first_prepared) apply_bcs();
            // the last flux-divergence direction applies the RK update in its
            // store when its plan takes the TMA path; otherwise a separate pass
            const RkEpilogue rk{Q_.as<double>(), du_.as<double>(), RKA[stage], RKB[stage], dt};
            if (!compute_rhs_impl(first_prepared, &rk))
                Pointwise<F>::lsrk(Q_.as<double>(), du_.as<double>(), dQ_.as<F>(), cells_ * ncons_, RKA[stage],
                                   RKB[stage], dt, st_);
        }
        tstage = t + dt;
        apply_bcs();
    }

    // add_sources! (src/rhs.jl:692, src/sources.jl:42-82)
    void add_sources() {
        BodyForces bf{};
        bf.n = desc.n_body_forces;
        for (int f = 0; f < bf.n; ++f)
            for (int a = 0; a < 3; ++a) bf.g[f][a] = desc.body_force[f][a];
        Pointwise<F>::body_forces(dQ_.as<F>(), Q_.as<double>(), cells_, Ns_, bf, st_);
    }

    // velocity gradients grad_u[d][j] (src/rhs.jl:596-604): one launch per dim
    // for u, v, w (per parity on a fold), then on curvilinear / stretched grids
    // the 1/h_d scaling and the curvature terms
    void velocity_gradients() {
        for (int k = 0; k < 3; ++k)
            if (g_.active[k])
                along_set(dset_[k], k, prim(P_U), g_u_.as<F>() + (size_t)cells_ * 3 * k, 3, OUT_STORE,
                          fold_[k].on ? fold_[k].sigvel : nullptr);
        if (geo_) MetricOps<F>::metric_grad(g_u_.as<F>(), prim_.as<F>(), G_, g_, st_);
    }

    // the rate reduction of max_rate on the refreshed primitives
    void rate_pass() {
        if (geo_) {
            MetricOps<F>::rate_geo(Q_.as<double>(), prim_.as<F>(), art_.as<F>(), part_.as<double>(), res_.as<double>(),
                                   Ns_, h_, desc.mu0, desc.Pr, desc.Sc, G_, g_, st_);
            return;
        }
        double idx[3];
        int act[3];
        for (int k = 0; k < 3; ++k) { idx[k] = 1.0 / h_[k]; act[k] = g_.active[k]; }
        Pointwise<F>::rate(Q_.as<double>(), prim_.as<F>(), art_.as<F>(), part_.as<double>(), res_.as<double>(), cells_,
                           Ns_, idx, act, desc.mu0, desc.Pr, desc.Sc, st_);
    }

    void max_rate(double* rate, double* rho_min) override {
        Pointwise<F>::primitives(Q_.as<double>(), prim_.as<F>(), cells_, Ns_, pc_, st_, desc.art_enabled);
        rate_pass();
        CLES_CUDA(cudaMemcpyAsync(host_res_, res_.p, 2 * sizeof(double), cudaMemcpyDeviceToHost, st_));
        CLES_CUDA(cudaStreamSynchronize(st_));
        if (take_device_timeouts(st_))
            throw Error(CLES_ETIMEOUT, "a bounded device wait expired in a compact-operator kernel");
        *rate = host_res_[0];
        *rho_min = host_res_[1];
        if (decomposed_) {
            // one collective: both reduced with max by negating the density (src/timestep.jl:170-173)
            double v[2] = {*rate, -*rho_min};
            allreduce(CLES_REDUCE_MAX, v, 2);
            *rate = v[0];
            *rho_min = -v[1];
        }
    }

    void filter_state() override {
        // filter_state! (src/timestep.jl:414-426): every conserved component
        // along every active dim in turn, in place (FP64 state in every mode)
        for (int k = 0; k < 3; ++k) {
            if (!g_.active[k]) continue;
            along_set(qset_[k], k, Q_.p, Q_.p, ncons_, OUT_STORE, fold_[k].on ? fold_[k].sigcons : nullptr);
        }
    }

    double predicted_dt(double rate) {
        const cles_step_control& c = desc.control;
        double r = rate;
        if (c.predict > 0 && rate_prev > 0) r = jmax(r, r + c.predict * (r - rate_prev));
        double dt = cfl / r;
        if (c.max_growth > 0 && dt_prev > 0) dt = jmin(dt, c.max_growth * dt_prev);
        return dt;
    }

    int run(double tfinal, int64_t nmax, cles_run_result* res) override {
        const cles_step_control& ctl = desc.control;
        const bool have_save = ctl.retries > 0;
        double save_t = t;
        int64_t save_step = step_count;
        if (have_save) {
            if (!save_.p) save_.alloc(ctx_, sizeof(double) * (size_t)cells_ * ncons_);
            CLES_CUDA(cudaMemcpyAsync(save_.p, Q_.p, Q_.bytes, cudaMemcpyDeviceToDevice, st_));
        }
        int attempts = 0;
        double dt_seen = 0.0, last_dt = 0.0;
        int64_t guard_step = -1, done = 0;
        int failure = CLES_FAIL_NONE;
        while (t < tfinal && step_count < nmax) {
            tstage = t;
            apply_bcs();
            double rate, rmin;
            max_rate(&rate, &rmin);
            double dt = predicted_dt(rate);
            const int f = check_step(ctl, dt, rmin, dt_seen);
            if (f != CLES_FAIL_NONE) {
                if (!have_save || attempts >= ctl.retries) { failure = f; break; }
                attempts += 1;
                const int64_t fail_step = step_count;
                CLES_CUDA(cudaMemcpyAsync(Q_.p, save_.p, Q_.bytes, cudaMemcpyDeviceToDevice, st_));
                t = save_t;
                step_count = save_step;
                cfl *= ctl.cfl_backoff;
                guard_step = fail_step;
                dt_prev = 0.0;
                rate_prev = 0.0;
                dt_seen = 0.0;
                continue;
            }
            if (have_save && ctl.savepoint_interval > 0 && step_count > guard_step &&
                step_count % ctl.savepoint_interval == 0) {
                CLES_CUDA(cudaMemcpyAsync(save_.p, Q_.p, Q_.bytes, cudaMemcpyDeviceToDevice, st_));
                save_t = t;
                save_step = step_count;
            }
            dt_seen = jmax(dt_seen, dt);
            dt = jmin(dt, tfinal - t);
            step(dt, true);
            t += dt;
            step_count += 1;
            dt_prev = dt;
            rate_prev = rate;
            last_dt = dt;
            ++done;
            if (desc.filter_interval > 0 && step_count % desc.filter_interval == 0) filter_state();
        }
        CLES_CUDA(cudaStreamSynchronize(st_));
        if (res) {
            res->steps = done;
            res->t = t;
            res->last_dt = last_dt;
            res->cfl = cfl;
            res->failure = failure;
            res->retries_used = attempts;
        }
        return failure == CLES_FAIL_NONE ? CLES_OK : CLES_EFAILURE;
    }

    // ---------------------------------------------------------- transfers --
    void set_state(const double* Q, int layout) override {
        const int64_t fcells = (int64_t)(g_.n[0] + 2 * pad_[0]) * (g_.n[1] + 2 * pad_[1]) * (g_.n[2] + 2 * pad_[2]);
        if (layout == CLES_LAYOUT_PADDED && fcells != cells_ && (size_t)fcells * sizeof(double) <= flux_.bytes) {
            // A pitched host-to-device copy of the interior moves 2 KB rows at
            // about half the link rate; each component's whole padded block goes
            // over contiguously instead, into the flux buffer (dead between RHS
            // evaluations), and a kernel gathers the interior.
            double* stage = flux_.as<double>();
            for (int c = 0; c < ncons_; ++c) {
                CLES_CUDA(cudaMemcpyAsync(stage, Q + fcells * c, sizeof(double) * fcells, cudaMemcpyHostToDevice, st_));
                gather_interior(stage, Q_.as<double>() + cells_ * c, g_.n, pad_, st_);
            }
        } else {
            copy_state_h2d(Q_.as<double>(), Q, g_.n, pad_, ncons_, layout, st_);
        }
        CLES_CUDA(cudaStreamSynchronize(st_));
    }
    void get_state(double* Q, int layout) override {
        copy_state_d2h(Q, Q_.as<double>(), g_.n, pad_, ncons_, layout, st_);
        CLES_CUDA(cudaStreamSynchronize(st_));
    }
    void get_double(const F* src, int ncomp, double* host, int layout) {
        if (sizeof(F) == sizeof(double)) {
            copy_state_d2h(host, reinterpret_cast<const double*>(src), g_.n, pad_, ncomp, layout, st_);
        } else {
            DevBuf tmp;
            tmp.alloc(ctx_, sizeof(double) * (size_t)cells_ * ncomp);
            Pointwise<F>::to_double(src, tmp.as<double>(), cells_ * ncomp, st_);
            copy_state_d2h(host, tmp.as<double>(), g_.n, pad_, ncomp, layout, st_);
            CLES_CUDA(cudaStreamSynchronize(st_));
        }
        CLES_CUDA(cudaStreamSynchronize(st_));
    }
    void get_rhs(double* dQ, int layout) override { get_double(dQ_.as<F>(), ncons_, dQ, layout); }
    void get_field(int which, double* host, int layout) override {
        const F* src = nullptr;
        switch (which) {
            case CLES_FIELD_RHO: src = prim(P_RHO); break;
            case CLES_FIELD_U: src = prim(P_U); break;
            case CLES_FIELD_V: src = prim(P_V); break;
            case CLES_FIELD_W: src = prim(P_W); break;
            case CLES_FIELD_P: src = prim(P_P); break;
            case CLES_FIELD_T: src = prim(P_T); break;
            case CLES_FIELD_C: src = prim(P_C); break;
            case CLES_FIELD_CP: src = prim(P_CP); break;
            case CLES_FIELD_MU_ART: src = art_.as<F>() + (size_t)cells_ * A_MU; break;
            case CLES_FIELD_BETA_ART: src = art_.as<F>() + (size_t)cells_ * A_BETA; break;
            case CLES_FIELD_KAPPA_ART: src = art_.as<F>() + (size_t)cells_ * A_KAPPA; break;
            case CLES_FIELD_SENSOR: src = scratch(2); break;  // the last sensor built: internal energy
            default:
                if (which >= CLES_FIELD_Y0 && which < CLES_FIELD_Y0 + Ns_) src = prim(P_Y0 + which - CLES_FIELD_Y0);
                else if (which >= CLES_FIELD_D_ART0 && which < CLES_FIELD_D_ART0 + Ns_)
                    src = art_.as<F>() + (size_t)cells_ * (A_D0 + which - CLES_FIELD_D_ART0);
                else if (which >= CLES_FIELD_GRAD_U0 && which < CLES_FIELD_GRAD_U0 + 9)
                    src = g_u_.as<F>() + (size_t)cells_ * (which - CLES_FIELD_GRAD_U0);
        }
        if (!src) throw Error(CLES_EINVAL, "unknown field");
        get_double(src, 1, host, layout);
    }

    double kinetic_energy() override {
        if (geo_) throw Error(CLES_EINVAL, "the kinetic-energy diagnostic is built for uniform Cartesian grids only");
        Pointwise<F>::kinetic(Q_.as<double>(), part_.as<double>(), res_.as<double>(), cells_, Ns_, st_);
        CLES_CUDA(cudaMemcpyAsync(host_res_, res_.p, sizeof(double), cudaMemcpyDeviceToHost, st_));
        CLES_CUDA(cudaStreamSynchronize(st_));
        double cellvol = 1.0, vol = 1.0;
        for (int k = 0; k < 3; ++k) {
            cellvol *= g_.active[k] ? h_[k] : 1.0;
            vol *= g_.active[k] ? desc.L[k] : 1.0;
        }
        double sum = host_res_[0];
        if (decomposed_) allreduce(CLES_REDUCE_SUM, &sum, 1);
        return sum * cellvol / vol;
    }

    double dissipation_rate() override {
        // dissipation_rate (src/diagnostics.jl:354-378): refreshes primitives,
        // gradients and artificial properties from the resident state
        using PW = Pointwise<F>;
        PW::primitives(Q_.as<double>(), prim_.as<F>(), cells_, Ns_, pc_, st_, desc.art_enabled);
        velocity_gradients();
        compute_artificial();
        unsigned foldmask = 0u;
        for (int k = 0; k < 3; ++k) {
            if (fold_[k].on && fold_[k].lo) foldmask |= 1u << (2 * k);
            if (fold_[k].on && fold_[k].hi) foldmask |= 1u << (2 * k + 1);
        }
        PW::dissipation(prim_.as<F>(), g_u_.as<F>(), art_.as<F>(), part_.as<double>(), res_.as<double>(), g_, desc.mu0,
                        st_, geo_ ? &G_ : nullptr, foldmask);
        CLES_CUDA(cudaMemcpyAsync(host_res_, res_.p, 2 * sizeof(double), cudaMemcpyDeviceToHost, st_));
        CLES_CUDA(cudaStreamSynchronize(st_));
        double v[2] = {host_res_[0], host_res_[1]};
        if (decomposed_) allreduce(CLES_REDUCE_SUM, v, 2);
        return v[0] / v[1];
    }

    double* state_device() override { return Q_.as<double>(); }
    cudaStream_t stream() const override { return st_; }

    // ------------------------------------------------------------ graph mode --
    // Captures on a private non-blocking stream (the legacy default stream,
    // which a context may use, cannot be captured); the graph is launched on
    // the context's stream.
    void capture_step(bool with_filter, cudaGraphExec_t* exec) {
        cudaGraph_t g = nullptr;
        if (!cap_st_) CLES_CUDA(cudaStreamCreateWithFlags(&cap_st_, cudaStreamNonBlocking));
        const cudaStream_t user = st_;
        st_ = cap_st_;
        const cudaError_t eb = cudaStreamBeginCapture(st_, cudaStreamCaptureModeRelaxed);
        if (eb != cudaSuccess) {
            st_ = user;
            throw Error(CLES_ECUDA, std::string("cudaStreamBeginCapture: ") + cudaGetErrorString(eb));
        }
        try {
            double* clk = clk_.as<double>();
            apply_bcs();
            Pointwise<F>::primitives(Q_.as<double>(), prim_.as<F>(), cells_, Ns_, pc_, st_, desc.art_enabled);
            rate_pass();
            clock_before(clk, res_.as<double>(), cc_, st_);
            for (int stage = 0; stage < 5; ++stage) {
                if (stage > 0) apply_bcs();
                const RkEpilogue rk{Q_.as<double>(), du_.as<double>(), RKA[stage], RKB[stage], 0.0, clk + DC_DT};
                if (!compute_rhs_impl(stage == 0, &rk))
                    Pointwise<F>::lsrk(Q_.as<double>(), du_.as<double>(), dQ_.as<F>(), cells_ * ncons_, RKA[stage],
                                       RKB[stage], 0.0, st_, clk + DC_DT);
            }
            apply_bcs();
            clock_after(clk, cc_, st_);
            if (with_filter) filter_state();
            CLES_CUDA(cudaMemcpyAsync(host_clk_, clk_.p, 8 * sizeof(double), cudaMemcpyDeviceToHost, st_));
        } catch (...) {
            cudaStreamEndCapture(st_, &g);
            st_ = user;
            if (g) cudaGraphDestroy(g);
            cudaGetLastError();
            throw;
        }
        const cudaError_t ee = cudaStreamEndCapture(st_, &g);
        st_ = user;
        if (ee != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            throw Error(CLES_ECUDA, std::string("cudaStreamEndCapture: ") + cudaGetErrorString(ee));
        }
        const cudaError_t e = cudaGraphInstantiate(exec, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) throw Error(CLES_ECUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
    }

    void graph_begin(double tfinal, int64_t nmax) override {
        if (decomposed_) throw Error(CLES_EINVAL, "graph mode does not run a decomposed solver (its exchanges are host calls)");
        for (int k = 0; k < 3; ++k)
            for (int s = 0; s < 2; ++s)
                for (int w = 0; w < 2; ++w)
                    if (face_fn_[k][s][w].fn)
                        throw Error(CLES_EINVAL, "graph mode cannot call a boundary face function at the stage times");
        const cles_step_control& c = desc.control;
        if (c.predict > 0 || c.max_growth > 0)
            throw Error(CLES_EINVAL, "graph mode supports neither rate prediction nor growth capping");
        cc_ = ClockConst{cfl, tfinal, (double)nmax, c.dt_min, c.dt_min_ratio};
        if (!clk_.p) clk_.alloc(ctx_, 16 * sizeof(double));
        if (!host_clk_) CLES_CUDA(cudaMallocHost(&host_clk_, 16 * sizeof(double)));
        double h[16] = {0};
        h[DC_T] = t;
        h[DC_STEP] = (double)step_count;
        h[DC_DONE] = (t < tfinal && step_count < nmax) ? 0.0 : 1.0;
        std::memcpy(host_clk_, h, sizeof(h));
        CLES_CUDA(cudaMemcpyAsync(clk_.p, host_clk_, sizeof(h), cudaMemcpyHostToDevice, st_));
        CLES_CUDA(cudaStreamSynchronize(st_));
        graph_free();
        capture_step(true, &gexec_filter_);
        if (desc.filter_interval != 1) capture_step(false, &gexec_plain_);
        CLES_CUDA(cudaStreamSynchronize(st_));
    }

    void graph_launch() override {
        const int64_t next = (int64_t)host_clk_[DC_STEP] + 1;
        const bool filt = desc.filter_interval > 0 && next % desc.filter_interval == 0;
        CLES_CUDA(cudaGraphLaunch(filt || !gexec_plain_ ? gexec_filter_ : gexec_plain_, st_));
    }

    const double* graph_clock() const override { return host_clk_; }

    void graph_end() override {
        CLES_CUDA(cudaStreamSynchronize(st_));
        t = host_clk_[DC_T];
        step_count = (int64_t)host_clk_[DC_STEP];
        dt_prev = host_clk_[DC_DT];
        rate_prev = host_clk_[DC_RATE];
    }

    void graph_free() {
        if (gexec_filter_) cudaGraphExecDestroy(gexec_filter_);
        if (gexec_plain_) cudaGraphExecDestroy(gexec_plain_);
        gexec_filter_ = gexec_plain_ = nullptr;
    }

    cles_solver_info info() const override {
        cles_solver_info I;
        std::memset(&I, 0, sizeof(I));
        for (int k = 0; k < 3; ++k) {
            I.n_local[k] = g_.n[k];
            I.active[k] = g_.active[k];
            I.h[k] = h_[k];
        }
        I.n_cons = ncons_;
        I.n_species = Ns_;
        I.cells = cells_;
        I.padded_cells = (int64_t)(g_.n[0] + 2 * pad_[0]) * (g_.n[1] + 2 * pad_[1]) * (g_.n[2] + 2 * pad_[2]);
        I.device_bytes = ctx_->allocated;
        return I;
    }

private:
    cles_ctx* ctx_;
    cudaStream_t st_;
    Grid3 g_{};
    int pad_[3]{};
    double h_[3]{};
    int Ns_ = 1, ncons_ = 5;
    int64_t cells_ = 0;
    PhysConst pc_{};
    std::unique_ptr<CompactPlan> deriv_[3][2], filt_[3][2], qfilt_[3][2];
    const CompactPlan* dset_[3][2] = {};
    const CompactPlan* fset_[3][2] = {};
    const CompactPlan* qset_[3][2] = {};
    // geometry: curvilinear metric or stretching, node tables, folds
    struct Fold {
        bool on = false, lo = false, hi = false, paired = false;
        PairParams pp{};
        int sigvel[3] = {1, 1, 1};
        int sigflux[CLES_MAX_SPECIES + 4] = {};
        int sigcons[CLES_MAX_SPECIES + 4] = {};
    };
    FaceFn face_fn_[3][2][2];
    std::vector<double> face_host_;
    DevBuf face_dev_;
    std::vector<double> stretch_x_[3];
    bool geo_ = false, folded_ = false;
    bool stretched_[3] = {false, false, false};
    double shift_[3]{}, orig_[3]{};
    Fold fold_[3];
    Geom G_{};
    std::unique_ptr<CompactPlan> hderiv_[3][2], hfilt_[3][2], hqfilt_[3][2];
    const CompactPlan* hdset_[3][2] = {};
    const CompactPlan* hfset_[3][2] = {};
    const CompactPlan* hqset_[3][2] = {};
    DevBuf geo_tab_, cotr_, pairbuf_;
    DevBuf Q_, du_, dQ_, prim_, g_u_, gty_, art_, scratch_, flux_, part_, res_, save_, clk_;
    double* host_res_ = nullptr;
    double* host_clk_ = nullptr;
    ClockConst cc_{};
    cudaGraphExec_t gexec_filter_ = nullptr, gexec_plain_ = nullptr;
    cudaStream_t cap_st_ = nullptr;
    bool switched_[3][2] = {{false, false}, {false, false}, {false, false}};
    // decomposition: this rank's offsets, the split dims' plans and buffers
    struct Split {
        bool on = false;
        std::unique_ptr<SplitPlan> deriv, filt, qfilt;
        int64_t lines = 0;
        int prev = -1, next = -1;
        bool lo_open = false, hi_open = false;
        DevBuf send_lo, send_hi, recv_lo, recv_hi, iface, iface_all, zbuf;
    };
    bool decomposed_ = false;
    cles_decomp dc_{};
    cles_exchange ex_{};
    int off_[3] = {0, 0, 0};
    int hpad_ = 0;
    Split split_[3];
    DevBuf padbuf_;
};

}  // namespace

double nasa9_cp_over_R(const cles_nasa9_interval& iv, double T) {
    const double* a = iv.a;
    const double T2 = T * T;
    return a[0] / T2 + a[1] / T + a[2] + a[3] * T + a[4] * T2 + a[5] * (T2 * T) + a[6] * (T2 * T2);
}

double nasa9_h_over_R(const cles_nasa9_interval& iv, double T) {
    const double* a = iv.a;
    const double T2 = T * T;
    return -a[0] / T + a[1] * std::log(T) + a[2] * T + a[3] * T2 / 2 + a[4] * (T2 * T) / 3 + a[5] * (T2 * T2) / 4 +
           a[6] * (T2 * T2 * T) / 5 + iv.b1;
}

double nasa9_species_energy(const cles_solver_desc& d, int k, double T) {
    const int n = d.n_intervals[k];
    int i = n - 1;
    for (int j = 0; j < n - 1; ++j)
        if (T <= d.nasa9[k][j].Tmax) { i = j; break; }
    return d.R[k] * nasa9_h_over_R(d.nasa9[k][i], T) - d.R[k] * T;
}

void nasa9_setup(PhysConst& pc, const cles_solver_desc& d) {
    pc.eos = d.eos;
    pc.T_guess = d.T_guess;
    if (d.eos != CLES_EOS_NASA9) return;
    if (!(d.T_guess > 0)) throw Error(CLES_EINVAL, "Nasa9Mixture T_guess must be positive");
    for (int k = 0; k < d.n_species; ++k) {
        const int n = d.n_intervals[k];
        if (n < 1 || n > CLES_MAX_NASA9_INTERVALS) throw Error(CLES_EINVAL, "NASA-9 species needs 1..4 intervals");
        if (!(d.R[k] > 0)) throw Error(CLES_EINVAL, "NASA-9 species has non-positive R");
        const cles_nasa9_interval* iv = d.nasa9[k];
        for (int i = 0; i < n; ++i)
            if (!(iv[i].Tmin > 0 && iv[i].Tmin < iv[i].Tmax)) throw Error(CLES_EINVAL, "invalid NASA-9 interval");
        // contiguity and continuity of cp and h at the joins
        // (_validate_nasa9_intervals, src/physics.jl:322-345; relative tolerance 2e-3)
        for (int i = 0; i + 1 < n; ++i) {
            const cles_nasa9_interval &lo = iv[i], &hi = iv[i + 1];
            const double sT = std::max({std::fabs(lo.Tmax), std::fabs(hi.Tmin), 1.0});
            if (!(std::fabs(lo.Tmax - hi.Tmin) <= 1e-10 * sT)) throw Error(CLES_EINVAL, "non-contiguous NASA-9 intervals");
            const double Tj = (lo.Tmax + hi.Tmin) / 2;
            const double cl = nasa9_cp_over_R(lo, Tj), ch = nasa9_cp_over_R(hi, Tj);
            if (!(std::fabs(cl - ch) <= 2e-3 * std::max({std::fabs(cl), std::fabs(ch), 1.0})))
                throw Error(CLES_EINVAL, "discontinuous NASA-9 cp at an interval join");
            const double hl = nasa9_h_over_R(lo, Tj), hh = nasa9_h_over_R(hi, Tj);
            if (!(std::fabs(hl - hh) <= 2e-3 * std::max({std::fabs(hl), std::fabs(hh), Tj})))
                throw Error(CLES_EINVAL, "discontinuous NASA-9 h at an interval join");
        }
        pc.nint[k] = n;
        for (int i = 0; i < n; ++i) {
            pc.Tmax[k][i] = iv[i].Tmax;
            for (int j = 0; j < 7; ++j) pc.a[k][i][j] = iv[i].a[j];
            pc.b1[k][i] = iv[i].b1;
        }
        // species energy and cv at T_guess: the state-independent part of the
        // Newton seed (src/physics.jl:475-482)
        int ig = n - 1;
        for (int i = 0; i < n - 1; ++i)
            if (d.T_guess <= iv[i].Tmax) { ig = i; break; }
        pc.e_ref[k] = d.R[k] * nasa9_h_over_R(iv[ig], d.T_guess) - d.R[k] * d.T_guess;
        pc.cv_ref[k] = d.R[k] * nasa9_cp_over_R(iv[ig], d.T_guess) - d.R[k];
    }
}

int check_step(const cles_step_control& c, double dt, double rho_min, double dt_seen) {
    // check_step (src/stepcontrol.jl:184-204)
    if (!std::isfinite(dt)) return CLES_FAIL_NONFINITE;
    if (!(rho_min > 0)) return CLES_FAIL_NEGATIVE_DENSITY;
    if (!(dt > PLANCK_TIME)) return CLES_FAIL_PLANCK;
    if (!(dt >= c.dt_min)) return CLES_FAIL_DT_MIN;
    if (c.dt_min_ratio > 0 && dt_seen > 0)
        if (!(dt >= c.dt_min_ratio * dt_seen)) return CLES_FAIL_DT_COLLAPSE;
    return CLES_FAIL_NONE;
}

size_t solver_bytes_estimate(const cles_solver_desc& d) {
    int64_t cells = 1;
    for (int k = 0; k < 3; ++k) cells *= d.n_global[k] < 1 ? 1 : d.n_global[k];
    const int Ns = d.n_species, nc = Ns + 4;
    const size_t F = d.precision == CLES_PREC_MIXED ? sizeof(float) : sizeof(double);
    const size_t per_cell = 2 * nc * sizeof(double)                     // Q, du
                            + F * (nc + (P_Y0 + Ns + 1) + 9 + 3 * (1 + Ns) + (A_D0 + Ns) + 5 + 3 * nc) +
                            (d.control.retries > 0 ? nc * sizeof(double) : 0);
    return (size_t)cells * per_cell + ((size_t)4 << 20);  // + plan tables and reduction scratch
}

int run_graph(SolverBase& s, double tfinal, int64_t nmax, cles_run_result* res) {
    const double t0 = s.t;
    const int64_t s0 = s.step_count;
    s.graph_begin(tfinal, nmax);
    const double* clk = s.graph_clock();
    while (clk[DC_DONE] == 0.0 && clk[DC_FAILURE] == 0.0) {
        s.graph_launch();
        CLES_CUDA(cudaStreamSynchronize(s.stream()));
    }
    s.graph_end();
    const int failure = (int)clk[DC_FAILURE];
    if (res) {
        res->steps = s.step_count - s0;
        res->t = s.t;
        res->last_dt = clk[DC_DT];
        res->cfl = s.cfl;
        res->failure = failure;
        res->retries_used = 0;
    }
    (void)t0;
    return failure == CLES_FAIL_NONE ? CLES_OK : CLES_EFAILURE;
}

std::unique_ptr<SolverBase> make_solver(cles_ctx* ctx, const cles_solver_desc& desc, const cles_decomp* dc,
                                        const cles_exchange* ex) {
    if (desc.precision == CLES_PREC_MIXED) return std::unique_ptr<SolverBase>(new Solver<float>(ctx, desc, dc, ex));
    if (desc.precision != CLES_PREC_FP64) throw Error(CLES_EINVAL, "unknown precision mode");
    return std::unique_ptr<SolverBase>(new Solver<double>(ctx, desc, dc, ex));
}

namespace {
void copy3d(double* dst, const double* src, const int n[3], const int pad[3], int ncomp, int layout, bool h2d,
            cudaStream_t st) {
    const int64_t cells = (int64_t)n[0] * n[1] * n[2];
    if (layout == CLES_LAYOUT_INTERIOR) {
        CLES_CUDA(cudaMemcpyAsync(dst, src, sizeof(double) * cells * ncomp,
                                  h2d ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToHost, st));
        return;
    }
    if (layout != CLES_LAYOUT_PADDED) throw Error(CLES_EINVAL, "unknown layout");
    const int F0 = n[0] + 2 * pad[0], F1 = n[1] + 2 * pad[1], F2 = n[2] + 2 * pad[2];
    const int64_t fcells = (int64_t)F0 * F1 * F2;
    for (int c = 0; c < ncomp; ++c) {
        cudaMemcpy3DParms p;
        std::memset(&p, 0, sizeof(p));
        if (h2d) {
            p.srcPtr = make_cudaPitchedPtr(const_cast<double*>(src) + fcells * c, sizeof(double) * F0, F0, F1);
            p.srcPos = make_cudaPos(sizeof(double) * pad[0], pad[1], pad[2]);
            p.dstPtr = make_cudaPitchedPtr(dst + cells * c, sizeof(double) * n[0], n[0], n[1]);
            p.kind = cudaMemcpyHostToDevice;
        } else {
            p.srcPtr = make_cudaPitchedPtr(const_cast<double*>(src) + cells * c, sizeof(double) * n[0], n[0], n[1]);
            p.dstPtr = make_cudaPitchedPtr(dst + fcells * c, sizeof(double) * F0, F0, F1);
            p.dstPos = make_cudaPos(sizeof(double) * pad[0], pad[1], pad[2]);
            p.kind = cudaMemcpyDeviceToHost;
        }
        p.extent = make_cudaExtent(sizeof(double) * n[0], n[1], n[2]);
        CLES_CUDA(cudaMemcpy3DAsync(&p, st));
    }
}
}  // namespace

void copy_state_h2d(double* dev, const double* host, const int n[3], const int pad[3], int ncomp, int layout,
                    cudaStream_t st) {
    copy3d(dev, host, n, pad, ncomp, layout, true, st);
}
void copy_state_d2h(double* host, const double* dev, const int n[3], const int pad[3], int ncomp, int layout,
                    cudaStream_t st) {
    copy3d(host, dev, n, pad, ncomp, layout, false, st);
}

}  // namespace cles
