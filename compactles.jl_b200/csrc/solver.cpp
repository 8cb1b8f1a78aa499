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

namespace {

const double RKA[5] = {0.0, -567301805773.0 / 1357537059087.0, -2404267990393.0 / 2016746695238.0,
                       -3550918686646.0 / 2091501179385.0, -1275806237668.0 / 842570457699.0};
const double RKB[5] = {1432997174477.0 / 9575080441755.0, 5161836677717.0 / 13612068292357.0,
                       1720146321549.0 / 2090206949498.0, 3134564353537.0 / 4481467310338.0,
                       2277821191437.0 / 14882151754819.0};
const double RKC[5] = {0.0, 1432997174477.0 / 9575080441755.0, 2526269341429.0 / 6820363962896.0,
                       2006345519317.0 / 3224310063776.0, 2802321613138.0 / 2924317926251.0};
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
    Solver(cles_ctx* ctx, const cles_solver_desc& d) : ctx_(ctx) {
        desc = d;
        st_ = ctx->stream;
        for (int k = 0; k < 3; ++k) {
            const bool p0 = d.bc[k][0] == CLES_BC_PERIODIC, p1 = d.bc[k][1] == CLES_BC_PERIODIC;
            if (p0 != p1) throw Error(CLES_EINVAL, "dimension " + std::to_string(k + 1) + " mixes periodic and non-periodic conditions");
            if (d.n_global[k] < 1) throw Error(CLES_EINVAL, "n_global must be >= 1");
            if (d.n_global[k] == 1 && !p0) throw Error(CLES_EINVAL, "collapsed dimension must use (PeriodicBC(), PeriodicBC())");
            for (int s = 0; s < 2; ++s) {
                if (d.bc[k][s] < CLES_BC_PERIODIC || d.bc[k][s] > CLES_BC_NSCBC_INFLOW)
                    throw Error(CLES_EINVAL, "unknown boundary condition");
                if (d.bc_switchable[k][s]) {
                    // SwitchableBC(before, after) (src/boundary.jl:137-148)
                    if (d.bc_after[k][s] < CLES_BC_PERIODIC || d.bc_after[k][s] > CLES_BC_NSCBC_INFLOW)
                        throw Error(CLES_EINVAL, "unknown boundary condition");
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
        if (d.n_species < 1 || d.n_species > CLES_MAX_SPECIES) throw Error(CLES_EINVAL, "bad species count");
        if (d.beta_sensor < 0 || d.beta_sensor > 2) throw Error(CLES_EINVAL, "unknown beta sensor");
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
        const int dt = sizeof(F) == 8 ? CLES_F64 : CLES_F32;
        for (int k = 0; k < 3; ++k) {
            if (!g_.active[k]) continue;
            deriv_[k].reset(new CompactPlan());
            build_compact_plan(*deriv_[k], d.deriv, g_.n, k, g_.periodic[k] != 0, h_[k], dt);
            filt_[k].reset(new CompactPlan());
            build_compact_plan(*filt_[k], d.filt, g_.n, k, g_.periodic[k] != 0, h_[k], dt);
            if (dt != CLES_F64) {
                qfilt_[k].reset(new CompactPlan());
                build_compact_plan(*qfilt_[k], d.filt, g_.n, k, g_.periodic[k] != 0, h_[k], CLES_F64);
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
        CLES_CUDA(cudaStreamSynchronize(st_));
    }

    ~Solver() override {
        graph_free();
        if (host_res_) cudaFreeHost(host_res_);
        if (host_clk_) cudaFreeHost(host_clk_);
        if (cap_st_) cudaStreamDestroy(cap_st_);
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
            if (g_.active[k]) launch_compact(*filt_[k], view(f), view(f), count, OUT_STORE, st_);
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
                bc_plane(Q_.as<double>(), g_, k, s, Ns_, bc, bs, st_);
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
                launch_compact(*deriv_[k], view(prim(P_P)), view(dpd), 1, OUT_STORE, st_);
                const int t1 = k == 0 ? 1 : 0, t2 = k == 2 ? 1 : 2;
                F* drd = nullptr;
                if (bc == CLES_BC_NSCBC_OUTFLOW) {
                    if (g_.active[t1]) launch_compact(*deriv_[t1], view(prim(P_P)), view(dt0), 1, OUT_STORE, st_);
                    if (g_.active[t2]) launch_compact(*deriv_[t2], view(prim(P_P)), view(dt1), 1, OUT_STORE, st_);
                } else {
                    drd = dt0;
                    launch_compact(*deriv_[k], view(prim(P_RHO)), view(drd), 1, OUT_STORE, st_);
                }
                Pointwise<F>::nscbc(dQ_.as<F>(), prim_.as<F>(), g_u_.as<F>(), gty_.as<F>(), Ns_ == 1 ? 1 : 1 + Ns_, dpd,
                                    dt0, dt1, drd, g_, k, s, Ns_, pc_, np, st_);
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
        PW::delta4_tiled(strain, prim(P_Y0 + Ns_), sensor, sensor_e, g_, w2, w1, st_);
        smooth(sensor, 2);
        PW::art_coef(sensor, sensor_e, prim_.as<F>(), g_u_.as<F>(), art_.as<F>(), cells_, desc.C_mu, desc.C_beta,
                     desc.C_kappa, desc.beta_sensor == CLES_BETA_GATED_STRAIN, st_);
        if (desc.beta_sensor == CLES_BETA_DILATATION) {
            PW::dilatation(g_u_.as<F>(), tmp_a, tmp_b, cells_, st_);
            PW::delta4_tiled(tmp_a, nullptr, sensor, nullptr, g_, w2, w2, st_);
            smooth(sensor, 1);
            PW::beta_dilatation(sensor, prim_.as<F>(), tmp_b, art_.as<F>(), cells_, desc.C_beta, st_);
        }
        if (Ns_ > 1) {
            for (int sp = 0; sp < Ns_; ++sp) {
                PW::delta4_tiled(prim(P_Y0 + sp), nullptr, tmp_a, nullptr, g_, w1, w1, st_);
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
        if (nscbc) rk = nullptr;   // the boundary correction comes between the divergence and the update
        if (!primitives_current) PW::primitives(Q_.as<double>(), prim_.as<F>(), cells_, Ns_, pc_, st_, desc.art_enabled);
        // velocity gradients grad_u[d][j] (src/rhs.jl:596-603), one launch per dim for u, v, w
        for (int k = 0; k < 3; ++k)
            if (g_.active[k])
                launch_compact(*deriv_[k], view(prim(P_U)), view(g_u_.as<F>() + (size_t)cells_ * 3 * k), 3, OUT_STORE, st_);
        compute_artificial();
        // temperature and mass-fraction gradients (src/rhs.jl:628-636); with one
        // species only dT (the species diffusion flux vanishes, see k_fluxes)
        const int ngty = Ns_ == 1 ? 1 : 1 + Ns_;
        for (int k = 0; k < 3; ++k)
            if (g_.active[k])
                launch_compact(*deriv_[k], view(prim(P_T)), view(gty_.as<F>() + (size_t)cells_ * ngty * k), ngty,
                               OUT_STORE, st_);
        PW::fluxes(Q_.as<double>(), prim_.as<F>(), g_u_.as<F>(), gty_.as<F>(), art_.as<F>(), flux_.as<F>(), cells_, Ns_,
                   pc_, desc.mu0, desc.Pr, desc.Sc, st_);
        // flux divergence dQ[c] = -sum_d D_d(F_dc) (src/rhs.jl:650-668), accumulated in the store.
        // With all three dims active the order is y, x, z: the first direction only
        // stores (no read of dQ), the x kernel reads dQ with vector loads, and z,
        // last, carries the RK update.  The sum differs from x, y, z by rounding.
        int order[3] = {0, 1, 2};
        if (g_.active[0] && g_.active[1] && g_.active[2]) { order[0] = 1; order[1] = 0; }
        int last = -1;
        for (int k = 0; k < 3; ++k)
            if (g_.active[k]) last = k;
        bool first = true, fused = false;
        for (int o = 0; o < 3; ++o) {
            const int k = order[o];
            if (!g_.active[k]) continue;
            const FieldView fin = view(flux_.as<F>() + (size_t)cells_ * ncons_ * k);
            if (k == last && !first && rk && launch_compact_rk(*deriv_[k], fin, view(dQ_.as<F>()), ncons_, *rk, st_)) {
                fused = true;
            } else {
                launch_compact(*deriv_[k], fin, view(dQ_.as<F>()), ncons_, first ? OUT_NEGATE : OUT_SUBTRACT, st_);
            }
            first = false;
        }
        if (first) CLES_CUDA(cudaMemsetAsync(dQ_.p, 0, dQ_.bytes, st_));
        if (nscbc) correct_rhs_nscbc();
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

    void max_rate(double* rate, double* rho_min) override {
        Pointwise<F>::primitives(Q_.as<double>(), prim_.as<F>(), cells_, Ns_, pc_, st_, desc.art_enabled);
        double idx[3];
        int act[3];
        for (int k = 0; k < 3; ++k) { idx[k] = 1.0 / h_[k]; act[k] = g_.active[k]; }
        Pointwise<F>::rate(Q_.as<double>(), prim_.as<F>(), art_.as<F>(), part_.as<double>(), res_.as<double>(), cells_,
                           Ns_, idx, act, desc.mu0, desc.Pr, desc.Sc, st_);
        CLES_CUDA(cudaMemcpyAsync(host_res_, res_.p, 2 * sizeof(double), cudaMemcpyDeviceToHost, st_));
        CLES_CUDA(cudaStreamSynchronize(st_));
        if (take_device_timeouts(st_))
            throw Error(CLES_ETIMEOUT, "a bounded device wait expired in a compact-operator kernel");
        *rate = host_res_[0];
        *rho_min = host_res_[1];
    }

    void filter_state() override {
        // filter_state! (src/timestep.jl:414-426): every conserved component
        // along every active dim in turn, in place (FP64 state in every mode)
        for (int k = 0; k < 3; ++k) {
            if (!g_.active[k]) continue;
            const CompactPlan& p = qfilt_[k] ? *qfilt_[k] : *filt_[k];
            launch_compact(p, view(Q_.p), view(Q_.p), ncons_, OUT_STORE, st_);
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
        Pointwise<F>::kinetic(Q_.as<double>(), part_.as<double>(), res_.as<double>(), cells_, Ns_, st_);
        CLES_CUDA(cudaMemcpyAsync(host_res_, res_.p, sizeof(double), cudaMemcpyDeviceToHost, st_));
        CLES_CUDA(cudaStreamSynchronize(st_));
        double cellvol = 1.0, vol = 1.0;
        for (int k = 0; k < 3; ++k) {
            cellvol *= g_.active[k] ? h_[k] : 1.0;
            vol *= g_.active[k] ? desc.L[k] : 1.0;
        }
        return host_res_[0] * cellvol / vol;
    }

    double dissipation_rate() override {
        // dissipation_rate (src/diagnostics.jl:354-378): refreshes primitives,
        // gradients and artificial properties from the resident state
        using PW = Pointwise<F>;
        PW::primitives(Q_.as<double>(), prim_.as<F>(), cells_, Ns_, pc_, st_, desc.art_enabled);
        for (int k = 0; k < 3; ++k)
            if (g_.active[k])
                launch_compact(*deriv_[k], view(prim(P_U)), view(g_u_.as<F>() + (size_t)cells_ * 3 * k), 3, OUT_STORE, st_);
        compute_artificial();
        PW::dissipation(prim_.as<F>(), g_u_.as<F>(), art_.as<F>(), part_.as<double>(), res_.as<double>(), g_, desc.mu0,
                        st_);
        CLES_CUDA(cudaMemcpyAsync(host_res_, res_.p, 2 * sizeof(double), cudaMemcpyDeviceToHost, st_));
        CLES_CUDA(cudaStreamSynchronize(st_));
        return host_res_[0] / host_res_[1];
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
            double idx[3];
            int act[3];
            for (int k = 0; k < 3; ++k) { idx[k] = 1.0 / h_[k]; act[k] = g_.active[k]; }
            Pointwise<F>::rate(Q_.as<double>(), prim_.as<F>(), art_.as<F>(), part_.as<double>(), res_.as<double>(),
                               cells_, Ns_, idx, act, desc.mu0, desc.Pr, desc.Sc, st_);
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
    std::unique_ptr<CompactPlan> deriv_[3], filt_[3], qfilt_[3];
    DevBuf Q_, du_, dQ_, prim_, g_u_, gty_, art_, scratch_, flux_, part_, res_, save_, clk_;
    double* host_res_ = nullptr;
    double* host_clk_ = nullptr;
    ClockConst cc_{};
    cudaGraphExec_t gexec_filter_ = nullptr, gexec_plain_ = nullptr;
    cudaStream_t cap_st_ = nullptr;
    bool switched_[3][2] = {{false, false}, {false, false}, {false, false}};
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

std::unique_ptr<SolverBase> make_solver(cles_ctx* ctx, const cles_solver_desc& desc) {
    if (desc.precision == CLES_PREC_MIXED) return std::unique_ptr<SolverBase>(new Solver<float>(ctx, desc));
    if (desc.precision != CLES_PREC_FP64) throw Error(CLES_EINVAL, "unknown precision mode");
    return std::unique_ptr<SolverBase>(new Solver<double>(ctx, desc));
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
