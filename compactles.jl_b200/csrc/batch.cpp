// Many independent solves of one physics class advanced together: run! in
// graph mode over a batch of grids of different sizes (no counterpart in the
// reference, which runs one problem per process).
//
// Layout.  The fields of every member live in shared arena blocks: field f of
// member g starts at element f * cells_total + off_g, with off_g a multiple of
// 64 cells.  The per-cell kernels of the step (primitives, strain, the
// artificial coefficients, fluxes) run unchanged over all cells_total
// elements, so one launch serves every member.  The padding cells between
// members hold a quiet uniform gas that no line solve, stencil or reduction
// reads.  Everything that depends on a grid's shape or spacing takes a table:
//   * line solves: a launch table of per-grid plans (power-of-two segments)
//     and a CTA table (launch_compact_batch);
//   * delta4_sum!: a table of 32 x 16 x 32 tiles;
//   * boundary planes: a table of faces;
//   * max_rate + the graph-mode clock: a table of 2048-cell chunks, then one
//     block per grid; every grid keeps its own dt, clock and stop condition.
// So one step of the whole batch is O(stages) launches, independent of the
// number of members, and it is captured once as a CUDA graph per batch
// composition.  The composition changes when a member is added or finishes;
// the arena is then rebuilt (state, artificial properties and clocks carried
// over), the tables rebuilt and the step re-captured.
//
// Autotuning.  Each batched line-solve launch has one free knob: the threads
// per CTA, which fixes the lines per CTA (LB = threads / S) for y/z lines and
// the depth of the transposed shared-memory tile for x lines.  The first time
// a launch of a given shape is built (operator, direction, element type, the
// largest segment count and the total line count to within a factor of two),
// every candidate (128, 256, 512 threads that fit the segments and shared
// memory) is timed with CUDA events on the batch's own fields and the fastest
// is kept for that shape.
//
// Arithmetic per grid does not depend on the composition (segmentation is a
// function of the line length alone, reductions are max / min), so a member's
// results are the same alone and in any mix, bitwise.

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "solver.h"

namespace cles {

namespace {

constexpr int64_t kAlignCells = 64;   // = the cell tile of the per-member constant map (cell / 64)

// Segment length of a batched plan: the fewest power-of-two segments of at
// most 32 points.  Fixed by the line length alone, so a member's arithmetic
// never depends on the other members; long segments keep the interface
// system (whose cost per point grows as n / m^2) small.
int batch_seg_max(int, int64_t) { return 32; }

__global__ void k_fill_const(double* __restrict__ a, int64_t n, double v) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        a[i] = v;
}

void fill_const(double* a, int64_t n, double v, cudaStream_t st) {
    if (n <= 0) return;
    int64_t b = (n + 255) / 256;
    if (b > 148 * 16) b = 148 * 16;
    k_fill_const<<<(unsigned)b, 256, 0, st>>>(a, n, v);
    count_launch();
    check_launch("k_fill_const");
}

bool face_supported(int bc) {
    return bc == CLES_BC_PERIODIC || bc == CLES_BC_SLIPWALL || bc == CLES_BC_NOSLIP_WALL ||
           bc == CLES_BC_EXTRAPOLATION || bc == CLES_BC_DIRICHLET;
}

// The fields every member of a batch must share (everything but the grid
// extents, the domain, the boundary states and the species gas constants and
// heat-capacity ratios), checked field by field.
void check_class(const cles_solver_desc& c, const cles_solver_desc& d) {
    auto bad = [](const std::string& what) {
        throw Error(CLES_EINVAL, "batch member differs from the batch's class in " + what);
    };
    if (d.n_species != c.n_species) bad("n_species");
    if (d.mu0 != c.mu0 || d.Pr != c.Pr || d.Sc != c.Sc) bad("transport");
    if (d.art_enabled != c.art_enabled || d.C_mu != c.C_mu || d.C_beta != c.C_beta || d.C_kappa != c.C_kappa ||
        d.C_D != c.C_D || d.beta_sensor != c.beta_sensor)
        bad("artificial-property parameters");
    if (std::memcmp(&d.deriv, &c.deriv, sizeof(cles_scheme)) != 0) bad("derivative scheme");
    if (std::memcmp(&d.filt, &c.filt, sizeof(cles_scheme)) != 0) bad("filter scheme");
    if (d.cfl != c.cfl || d.filter_interval != c.filter_interval) bad("cfl / filter_interval");
    if (d.control.dt_min != c.control.dt_min || d.control.dt_min_ratio != c.control.dt_min_ratio) bad("step control");
    if (d.precision != c.precision) bad("precision");
    for (int k = 0; k < 3; ++k) {
        if ((d.n_global[k] > 1) != (c.n_global[k] > 1)) bad("active dimensions");
        for (int s = 0; s < 2; ++s)
            if (d.bc[k][s] != c.bc[k][s]) bad("boundary condition kinds");
    }
}

// What the batch path supports (checked on every member).
void check_supported(const cles_solver_desc& d) {
    auto no = [](const std::string& what) { throw Error(CLES_EINVAL, "batched solves do not support " + what); };
    if (d.eos != CLES_EOS_IDEAL) no("NASA-9 mixtures");
    if (d.metric != CLES_METRIC_CARTESIAN) no("curvilinear metrics");
    for (int k = 0; k < 3; ++k)
        if (d.stretch_x[k] || d.stretch_dxdxi[k]) no("stretched grids");
    if (d.n_body_forces) no("source terms");
    if (d.control.retries > 0 || d.control.predict > 0 || d.control.max_growth > 0)
        no("rollback retries, rate prediction or growth capping");
    if (d.filter_interval < 0) no("a negative filter interval");
    if (d.n_species < 1 || d.n_species > CLES_MAX_SPECIES) no("this species count");
    if (d.beta_sensor < 0 || d.beta_sensor > 2) no("this beta sensor");
    if (d.precision != CLES_PREC_FP64 && d.precision != CLES_PREC_MIXED) no("this precision mode");
    bool any = false;
    for (int k = 0; k < 3; ++k) {
        if (d.n_global[k] < 1) throw Error(CLES_EINVAL, "n_global must be >= 1");
        const bool p0 = d.bc[k][0] == CLES_BC_PERIODIC, p1 = d.bc[k][1] == CLES_BC_PERIODIC;
        if (p0 != p1) throw Error(CLES_EINVAL, "dimension " + std::to_string(k + 1) + " mixes periodic and non-periodic conditions");
        if (d.n_global[k] == 1 && !p0) throw Error(CLES_EINVAL, "collapsed dimension must use (PeriodicBC(), PeriodicBC())");
        any = any || d.n_global[k] > 1;
        for (int s = 0; s < 2; ++s) {
            if (!face_supported(d.bc[k][s])) no("this boundary condition (periodic, slip and no-slip walls, extrapolation and constant Dirichlet only)");
            if (d.bc_switchable[k][s]) no("switchable faces");
        }
    }
    if (!any) throw Error(CLES_EINVAL, "a batched solve needs at least one active dimension");
}

struct Member {
    int64_t id = 0;
    cles_solver_desc desc{};
    double tfinal = 0.0;
    int64_t nmax = 0;
    int layout = CLES_LAYOUT_PADDED;
    int n[3] = {1, 1, 1};
    int pad[3] = {0, 0, 0};
    bool active[3] = {false, false, false};
    bool periodic[3] = {true, true, true};
    double h[3] = {1, 1, 1};
    int64_t cells = 0;
    std::unique_ptr<CompactPlan> deriv[3], filt[3], qfilt[3];      // batched segmentation
    std::unique_ptr<CompactPlan> sderiv[3], sfilt[3], sqfilt[3];   // the one-grid solver's plans
    std::vector<double> Qhost;     // interior layout: initial state until placed, final state once retired
    bool placed = false;           // its state lives in the arena
    bool retired = false;          // finished, failed or removed; Qhost holds the last state
    int state = CLES_REQ_QUEUED;
    int failure = CLES_FAIL_NONE;
    double clk[16] = {0};
    double mc[24] = {0};           // R_k, cv_k, cp_k of its ideal mixture
    int64_t off = 0;               // arena offset while placed
    double admit_s = -1, done_s = -1;
};

// One batched line-solve launch: the plans of every member along one
// direction for one operator, with its tuned thread count.
struct Role {
    BatchLaunchKind kind{};
    DevBuf plans, blocks;
    int nblocks = 0;
    bool per_member = false;   // launch each member's one-grid kernel instead of the batched one
};

constexpr int kAuxStreams = 8;   // streams the per-member launches of one role spread over

enum { R_DERIV = 0, R_FILT = 1, R_QFILT = 2 };

}  // namespace

std::map<std::string, int>& batch_tuning_cache() {
    static std::map<std::string, int> m;
    return m;
}

template <typename F>
class Batch final : public BatchBase {
public:
    explicit Batch(cles_ctx* ctx, const cles_solver_desc& cls) : ctx_(ctx), cls_(cls) {
        st_ = ctx->stream;
        Ns_ = cls.n_species;
        ncons_ = Ns_ + 4;
        for (int k = 0; k < Ns_; ++k) {
            pc_.Rk[k] = cls.R[k];
            pc_.cvk[k] = cls.R[k] / (cls.gamma[k] - 1);
            pc_.cpk[k] = pc_.Rk[k] + pc_.cvk[k];
        }
        pc_.eos = CLES_EOS_IDEAL;
        for (int k = 0; k < 3; ++k) act_[k] = cls.n_global[k] > 1;
        CLES_CUDA(cudaStreamCreateWithFlags(&cap_st_, cudaStreamNonBlocking));
        CLES_CUDA(cudaEventCreate(&ev0_));
        CLES_CUDA(cudaEventCreate(&ev1_));
        for (int i = 0; i < kAuxStreams; ++i) {
            CLES_CUDA(cudaStreamCreateWithFlags(&aux_[i], cudaStreamNonBlocking));
            CLES_CUDA(cudaEventCreateWithFlags(&aux_ev_[i], cudaEventDisableTiming));
        }
        CLES_CUDA(cudaEventCreateWithFlags(&fork_ev_, cudaEventDisableTiming));
    }
    ~Batch() override {
        if (exec_) cudaGraphExecDestroy(exec_);
        if (host_clk_) cudaFreeHost(host_clk_);
        if (cap_st_) cudaStreamDestroy(cap_st_);
        cudaEventDestroy(ev0_);
        cudaEventDestroy(ev1_);
        for (int i = 0; i < kAuxStreams; ++i) {
            cudaStreamDestroy(aux_[i]);
            cudaEventDestroy(aux_ev_[i]);
        }
        cudaEventDestroy(fork_ev_);
    }

    int64_t add(const cles_solver_desc& d, const double* Q0, int layout, double tfinal, int64_t nmax,
                double now) override {
        check_supported(d);
        check_class(cls_, d);
        if (layout != CLES_LAYOUT_PADDED && layout != CLES_LAYOUT_INTERIOR) throw Error(CLES_EINVAL, "unknown layout");
        if (!Q0) throw Error(CLES_EINVAL, "null initial state");
        auto m = std::make_unique<Member>();
        m->id = next_id_++;
        m->desc = d;
        m->tfinal = tfinal;
        m->nmax = nmax;
        m->layout = layout;
        m->cells = 1;
        for (int k = 0; k < 3; ++k) {
            m->n[k] = d.n_global[k];
            m->active[k] = d.n_global[k] > 1;
            m->periodic[k] = m->active[k] ? d.bc[k][0] == CLES_BC_PERIODIC : true;
            m->pad[k] = m->active[k] ? d.n_halo : 0;
            m->h[k] = !m->active[k] ? 1.0 : (m->periodic[k] ? d.L[k] / d.n_global[k] : d.L[k] / (d.n_global[k] - 1));
            m->cells *= m->n[k];
        }
        const int dtF = sizeof(F) == 8 ? CLES_F64 : CLES_F32;
        for (int k = 0; k < 3; ++k) {
            if (!m->active[k]) continue;
            const int sm = batch_seg_max(m->n[k], m->cells / m->n[k]);
            m->deriv[k].reset(new CompactPlan());
            build_compact_plan(*m->deriv[k], d.deriv, m->n, k, m->periodic[k], m->h[k], dtF, 0, 0, false, false, sm);
            m->filt[k].reset(new CompactPlan());
            build_compact_plan(*m->filt[k], d.filt, m->n, k, m->periodic[k], m->h[k], dtF, 0, 0, false, false, sm);
            if (dtF != CLES_F64) {
                m->qfilt[k].reset(new CompactPlan());
                build_compact_plan(*m->qfilt[k], d.filt, m->n, k, m->periodic[k], m->h[k], CLES_F64, 0, 0, false,
                                   false, sm);
            }
            m->sderiv[k].reset(new CompactPlan());
            build_compact_plan(*m->sderiv[k], d.deriv, m->n, k, m->periodic[k], m->h[k], dtF);
            m->sfilt[k].reset(new CompactPlan());
            build_compact_plan(*m->sfilt[k], d.filt, m->n, k, m->periodic[k], m->h[k], dtF);
            if (dtF != CLES_F64) {
                m->sqfilt[k].reset(new CompactPlan());
                build_compact_plan(*m->sqfilt[k], d.filt, m->n, k, m->periodic[k], m->h[k], CLES_F64);
            }
        }
        for (int sp = 0; sp < Ns_; ++sp) {
            m->mc[sp] = d.R[sp];
            m->mc[8 + sp] = d.R[sp] / (d.gamma[sp] - 1);
            m->mc[16 + sp] = m->mc[sp] + m->mc[8 + sp];
        }
        // initial state to the interior layout on the host
        m->Qhost.assign((size_t)(m->cells * ncons_), 0.0);
        const int64_t F0 = m->n[0] + 2 * m->pad[0], F1 = m->n[1] + 2 * m->pad[1], F2 = m->n[2] + 2 * m->pad[2];
        const int64_t fe = layout == CLES_LAYOUT_PADDED ? F0 * F1 * F2 : m->cells;
        for (int c = 0; c < ncons_; ++c)
            for (int kk = 0; kk < m->n[2]; ++kk)
                for (int j = 0; j < m->n[1]; ++j) {
                    const double* src = Q0 + c * fe;
                    const int64_t so = layout == CLES_LAYOUT_PADDED
                                           ? (m->pad[0] + (j + m->pad[1]) * F0 + (kk + m->pad[2]) * F0 * F1)
                                           : ((int64_t)j * m->n[0] + (int64_t)kk * m->n[0] * m->n[1]);
                    std::memcpy(&m->Qhost[(size_t)(c * m->cells + (int64_t)j * m->n[0] + (int64_t)kk * m->n[0] * m->n[1])],
                                src + so, sizeof(double) * m->n[0]);
                }
        m->clk[DC_T] = 0.0;
        m->clk[DC_STEP] = 0.0;
        m->clk[DC_DONE] = (0.0 < tfinal && 0 < nmax) ? 0.0 : 1.0;
        m->state = CLES_REQ_RUNNING;
        m->admit_s = now;
        if (m->clk[DC_DONE] != 0.0) {
            m->retired = true;
            m->state = CLES_REQ_DONE;
            m->done_s = now;
        } else {
            dirty_ = true;
        }
        const int64_t id = m->id;
        members_.push_back(std::move(m));
        return id;
    }

    int n_active() const override {
        int n = 0;
        for (auto& m : members_)
            if (!m->retired) ++n;
        return n;
    }

    int step(double now) override {
        launch(now);
        return collect(now);
    }

    void launch(double now) override {
        if (dirty_) compose(now);
        if (order_.empty()) return;
        CLES_CUDA(cudaGraphLaunch(exec_, st_));
        launched_ = true;
    }

    int collect(double now) override {
        if (!launched_) return n_active_after_step();
        launched_ = false;
        CLES_CUDA(cudaStreamSynchronize(st_));
        ++steps_;
        for (size_t g = 0; g < order_.size(); ++g) {
            Member& m = *order_[g];
            std::memcpy(m.clk, host_clk_ + 16 * g, sizeof(m.clk));
            if (m.clk[DC_DONE] != 0.0 || m.clk[DC_FAILURE] != 0.0) {
                m.failure = (int)m.clk[DC_FAILURE];
                m.state = m.failure ? CLES_REQ_FAILED : CLES_REQ_DONE;
                m.done_s = now;
                dirty_ = true;   // retired at the next composition
            }
        }
        return n_active_after_step();
    }

    void remove(int64_t id, double now) override {
        Member& m = find(id);
        if (m.retired) return;
        if (m.placed) {
            dirty_ = true;
            m.state = CLES_REQ_CANCELLED;
            m.done_s = now;
            // the state is saved when the arena is rebuilt
            cancelled_.push_back(id);
        } else {
            m.retired = true;
            m.state = CLES_REQ_CANCELLED;
            m.done_s = now;
        }
    }

    void status(int64_t id, cles_request_status* out) const override {
        const Member& m = find(id);
        std::memset(out, 0, sizeof(*out));
        out->state = m.state;
        out->failure = m.failure;
        out->steps = (int64_t)m.clk[DC_STEP];
        out->t = m.clk[DC_T];
        out->admit_s = m.admit_s;
        out->done_s = m.done_s;
        out->device_bytes = member_bytes(m);
    }

    void fetch(int64_t id, double* Q, int layout) override {
        Member& m = find(id);
        if (m.placed) save_member(m);
        const int64_t F0 = m.n[0] + 2 * m.pad[0], F1 = m.n[1] + 2 * m.pad[1], F2 = m.n[2] + 2 * m.pad[2];
        const int64_t fe = layout == CLES_LAYOUT_PADDED ? F0 * F1 * F2 : m.cells;
        for (int c = 0; c < ncons_; ++c)
            for (int kk = 0; kk < m.n[2]; ++kk)
                for (int j = 0; j < m.n[1]; ++j) {
                    const int64_t so = layout == CLES_LAYOUT_PADDED
                                           ? (m.pad[0] + (j + m.pad[1]) * F0 + (kk + m.pad[2]) * F0 * F1)
                                           : ((int64_t)j * m.n[0] + (int64_t)kk * m.n[0] * m.n[1]);
                    std::memcpy(Q + c * fe + so,
                                &m.Qhost[(size_t)(c * m.cells + (int64_t)j * m.n[0] + (int64_t)kk * m.n[0] * m.n[1])],
                                sizeof(double) * m.n[0]);
                }
    }

    void set_strategy(int st) override {
        if (st != CLES_BATCH_AUTO && st != CLES_BATCH_BATCHED && st != CLES_BATCH_PER_MEMBER)
            throw Error(CLES_EINVAL, "unknown batch strategy");
        strategy_ = st;
        dirty_ = true;   // re-tune and re-capture at the next step
    }

    void stats(cles_batch_stats* s) const override {
        std::memset(s, 0, sizeof(*s));
        s->members = (int)members_.size();
        s->active = n_active();
        s->compositions = compositions_;
        s->steps = steps_;
        s->launches_per_step = launches_per_step_;
        s->cells_total = ct_;
        s->n_roles = 0;
        for (int r = 0; r < 3; ++r)
            for (int k = 0; k < 3; ++k)
                if (roles_[r][k].nblocks > 0 && s->n_roles < 9) {
                    cles_batch_tuning& t = s->tuning[s->n_roles++];
                    t.op = r;
                    t.dim = k + 1;
                    t.threads = roles_[r][k].kind.threads;
                    t.smem = (int64_t)roles_[r][k].kind.smem;
                    t.ctas = roles_[r][k].nblocks;
                    t.tuned_ms = tuned_ms_[r][k];
                }
    }

    static size_t member_bytes(const Member& m) {
        cles_solver_desc d = m.desc;
        return solver_bytes_estimate(d);
    }

private:
    Member& find(int64_t id) const {
        for (auto& m : members_)
            if (m->id == id) return *m;
        throw Error(CLES_EINVAL, "no batch member with this id");
    }

    int n_active_after_step() const {
        int n = 0;
        for (Member* m : order_)
            if (m->state == CLES_REQ_RUNNING) ++n;
        for (auto& m : members_)
            if (!m->placed && !m->retired) ++n;
        return n;
    }

    // copy a placed member's state from the arena to its host buffer
    void save_member(Member& m) {
        CLES_CUDA(cudaStreamSynchronize(st_));
        for (int c = 0; c < ncons_; ++c)
            CLES_CUDA(cudaMemcpyAsync(&m.Qhost[(size_t)(c * m.cells)], Q_.as<double>() + c * ct_ + m.off,
                                      sizeof(double) * m.cells, cudaMemcpyDeviceToHost, st_));
        CLES_CUDA(cudaStreamSynchronize(st_));
    }

    F* field(const DevBuf& b, int slot) const { return b.as<F>() + (size_t)ct_ * slot; }

    // ------------------------------------------------------------ compose --
    void compose(double now) {
        CLES_CUDA(cudaStreamSynchronize(st_));
        // retire members that finished, failed or were cancelled (their state to the host)
        for (auto& mp : members_) {
            Member& m = *mp;
            if (m.placed && m.state != CLES_REQ_RUNNING) {
                save_member(m);
                m.placed = false;
                m.retired = true;
            }
        }
        cancelled_.clear();
        std::vector<Member*> keep;
        for (auto& mp : members_)
            if (!mp->retired) keep.push_back(mp.get());
        // new offsets
        int64_t ct = 0;
        std::vector<int64_t> off(keep.size());
        for (size_t g = 0; g < keep.size(); ++g) {
            off[g] = ct;
            ct += (keep[g]->cells + kAlignCells - 1) / kAlignCells * kAlignCells;
        }
        const int G = (int)keep.size();
        // new arena; the persistent fields move over from the old one
        DevBuf Qn, artn, clkn;
        const size_t Fs = sizeof(F);
        if (G > 0) {
            Qn.alloc(ctx_, sizeof(double) * (size_t)ct * ncons_);
            artn.alloc(ctx_, Fs * (size_t)ct * (A_D0 + Ns_));
            clkn.alloc(ctx_, sizeof(double) * 16 * (size_t)G);
            // quiet uniform gas in the padding: rho_1 = 1, no momentum, E = 1
            CLES_CUDA(cudaMemsetAsync(Qn.p, 0, Qn.bytes, st_));
            fill_const(Qn.as<double>(), ct, 1.0, st_);
            fill_const(Qn.as<double>() + (size_t)ct * (Ns_ + 3), ct, 1.0, st_);
            CLES_CUDA(cudaMemsetAsync(artn.p, 0, artn.bytes, st_));
            std::vector<double> clk_h(16 * (size_t)G, 0.0);
            for (int g = 0; g < G; ++g) {
                Member& m = *keep[g];
                for (int c = 0; c < ncons_; ++c) {
                    double* dst = Qn.as<double>() + (size_t)c * ct + off[g];
                    if (m.placed)
                        CLES_CUDA(cudaMemcpyAsync(dst, Q_.as<double>() + (size_t)c * ct_ + m.off,
                                                  sizeof(double) * m.cells, cudaMemcpyDeviceToDevice, st_));
                    else
                        CLES_CUDA(cudaMemcpyAsync(dst, &m.Qhost[(size_t)(c * m.cells)], sizeof(double) * m.cells,
                                                  cudaMemcpyHostToDevice, st_));
                }
                if (m.placed)
                    for (int a = 0; a < A_D0 + Ns_; ++a)
                        CLES_CUDA(cudaMemcpyAsync(artn.as<F>() + (size_t)a * ct + off[g], art_.as<F>() + (size_t)a * ct_ + m.off,
                                                  Fs * m.cells, cudaMemcpyDeviceToDevice, st_));
                std::memcpy(&clk_h[16 * (size_t)g], m.clk, sizeof(m.clk));
            }
            CLES_CUDA(cudaMemcpyAsync(clkn.p, clk_h.data(), sizeof(double) * clk_h.size(), cudaMemcpyHostToDevice, st_));
            CLES_CUDA(cudaStreamSynchronize(st_));   // pageable sources above
        }
        for (int g = 0; g < G; ++g) {
            keep[g]->placed = true;
            keep[g]->off = off[g];
            if (keep[g]->admit_s < 0) keep[g]->admit_s = now;
        }
        std::swap(Q_.p, Qn.p); std::swap(Q_.bytes, Qn.bytes); std::swap(Q_.ctx, Qn.ctx);
        std::swap(art_.p, artn.p); std::swap(art_.bytes, artn.bytes); std::swap(art_.ctx, artn.ctx);
        std::swap(clk_.p, clkn.p); std::swap(clk_.bytes, clkn.bytes); std::swap(clk_.ctx, clkn.ctx);
        Qn.release(); artn.release(); clkn.release();
        ct_ = ct;
        order_ = keep;
        dirty_ = false;
        ++compositions_;
        if (exec_) { cudaGraphExecDestroy(exec_); exec_ = nullptr; }
        if (G == 0) {
            release_derived();
            return;
        }
        alloc_derived();
        build_tables();
        tune_roles();
        capture();
    }

    void release_derived() {
        for (DevBuf* b : {&du_, &dQ_, &prim_, &g_u_, &gty_, &scratch_, &flux_, &part_, &grids_, &tiles_, &faces_,
                          &chunks_, &chunk_first_, &mc_, &tmap_})
            b->release();
        for (auto& rr : roles_)
            for (auto& r : rr) { r.plans.release(); r.blocks.release(); r.nblocks = 0; }
    }

    void alloc_derived() {
        release_derived();
        const size_t c = (size_t)ct_, Fs = sizeof(F);
        du_.alloc(ctx_, sizeof(double) * c * ncons_);
        dQ_.alloc(ctx_, Fs * c * ncons_);
        prim_.alloc(ctx_, Fs * c * (P_Y0 + Ns_ + 1));
        g_u_.alloc(ctx_, Fs * c * 9);
        gty_.alloc(ctx_, Fs * c * 3 * (1 + Ns_));
        scratch_.alloc(ctx_, Fs * c * 5);
        flux_.alloc(ctx_, Fs * c * 3 * ncons_);
        for (DevBuf* b : {&du_, &dQ_, &prim_, &g_u_, &gty_, &scratch_, &flux_})
            CLES_CUDA(cudaMemsetAsync(b->p, 0, b->bytes, st_));
        if (host_clk_cap_ < order_.size()) {
            if (host_clk_) cudaFreeHost(host_clk_);
            host_clk_cap_ = std::max<size_t>(order_.size(), 2 * host_clk_cap_);
            CLES_CUDA(cudaMallocHost(&host_clk_, sizeof(double) * 16 * host_clk_cap_));
        }
    }

    template <typename T>
    static void upload(DevBuf& b, cles_ctx* ctx, const std::vector<T>& v, cudaStream_t st) {
        b.release();
        if (v.empty()) return;
        b.alloc(ctx, sizeof(T) * v.size());
        CLES_CUDA(cudaMemcpyAsync(b.p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, st));
    }

    void build_tables() {
        const int G = (int)order_.size();
        std::vector<BatchGrid> grids(G);
        std::vector<BatchTile> tiles;
        std::vector<BatchFace> faces;
        std::vector<BatchChunk> chunks;
        std::vector<int> first(G + 1, 0);
        std::vector<double> mc(24 * (size_t)G);
        std::vector<int> tmap((size_t)(ct_ / kAlignCells), 0);
        for (int g = 0; g < G; ++g) {
            const Member& m = *order_[g];
            std::memcpy(&mc[24 * (size_t)g], m.mc, sizeof(m.mc));
            const int64_t t1 = (g + 1 < G ? order_[g + 1]->off : ct_) / kAlignCells;
            for (int64_t t = m.off / kAlignCells; t < t1; ++t) tmap[(size_t)t] = g;
            BatchGrid& B = grids[g];
            std::memset(&B, 0, sizeof(B));
            for (int k = 0; k < 3; ++k) {
                B.g.n[k] = m.n[k];
                B.g.active[k] = m.active[k];
                B.g.periodic[k] = m.periodic[k];
                B.h[k] = m.h[k];
            }
            B.off = m.off;
            B.cells = m.cells;
            B.clk = clk_.as<double>() + 16 * (size_t)g;
            B.cc = ClockConst{cls_.cfl, m.tfinal, (double)m.nmax, cls_.control.dt_min, cls_.control.dt_min_ratio};
            // delta4 tiles
            const int tx = (m.n[0] + kD4X - 1) / kD4X, ty = (m.n[1] + kD4Y - 1) / kD4Y,
                      tz = (m.n[2] + kD4Z - 1) / kD4Z;
            for (int z = 0; z < tz; ++z)
                for (int y = 0; y < ty; ++y)
                    for (int x = 0; x < tx; ++x) tiles.push_back(BatchTile{g, kD4X * x, kD4Y * y, kD4Z * z});
            // faces (apply_bcs! order: dims, low then high)
            for (int k = 0; k < 3; ++k) {
                if (!m.active[k]) continue;
                for (int s = 0; s < 2; ++s) {
                    const int bc = m.desc.bc[k][s];
                    if (bc == CLES_BC_PERIODIC) continue;
                    BatchFace f;
                    std::memset(&f, 0, sizeof(f));
                    f.grid = g; f.d = k; f.side = s; f.kind = bc;
                    for (int c = 0; c < ncons_; ++c) f.st.q[c] = m.desc.bc_state[k][s][c];
                    if (bc == CLES_BC_NOSLIP_WALL) {
                        const double Tw = m.desc.bc_params[k][s].Twall;
                        f.st.iso = std::isnan(Tw) ? 0 : 1;
                        f.st.Twall = Tw;
                        f.st.ew_times_T = 1;
                        for (int sp = 0; sp < Ns_; ++sp) f.st.ew[sp] = m.mc[8 + sp];
                    }
                    faces.push_back(f);
                }
            }
            first[g] = (int)chunks.size();
            for (int64_t c0 = 0; c0 < m.cells; c0 += kBatchChunk) chunks.push_back(BatchChunk{g, c0});
        }
        first[G] = (int)chunks.size();
        upload(grids_, ctx_, grids, st_);
        upload(tiles_, ctx_, tiles, st_);
        upload(faces_, ctx_, faces, st_);
        upload(chunks_, ctx_, chunks, st_);
        upload(chunk_first_, ctx_, first, st_);
        upload(mc_, ctx_, mc, st_);
        upload(tmap_, ctx_, tmap, st_);
        part_.release();
        part_.alloc(ctx_, sizeof(double) * 2 * std::max<size_t>(chunks.size(), 1));
        ntiles_ = (int)tiles.size();
        nfaces_ = (int)faces.size();
        nchunks_ = (int)chunks.size();
        CLES_CUDA(cudaStreamSynchronize(st_));
    }

    const CompactPlan* plan_of(const Member& m, int role, int k) const {
        if (role == R_DERIV) return m.deriv[k].get();
        if (role == R_FILT) return m.filt[k].get();
        return m.qfilt[k] ? m.qfilt[k].get() : m.filt[k].get();
    }

    // Tables of one role with `threads` per CTA; false if a plan does not fit.
    bool role_tables(int role, int k, int threads, Role& R) {
        const int G = (int)order_.size();
        std::vector<BatchLinePlan> plans(G);
        std::vector<int2> blocks;
        const int dtype = role == R_QFILT ? CLES_F64 : (sizeof(F) == 8 ? CLES_F64 : CLES_F32);
        size_t smem = 0;
        int ms = 8;
        for (int g = 0; g < G; ++g) {
            const Member& m = *order_[g];
            const CompactPlan* p = plan_of(m, role, k);
            if (p->P.S > threads) return false;
            const int LB = threads / p->P.S;
            BatchLinePlan& bp = plans[g];
            std::memset(&bp, 0, sizeof(bp));
            bp.P = p->P;
            bp.P.LB = LB;
            bp.tab = dtype == CLES_F64 ? static_cast<const void*>(p->tab64) : static_cast<const void*>(p->tab32);
            bp.off = m.off;
            bp.sy = m.n[0];
            bp.sz = (int64_t)m.n[0] * m.n[1];
            bp.clk = clk_.as<double>() + 16 * (size_t)g;
            smem = std::max(smem, batch_plan_smem(p->P, LB, dtype));
            const int mlen = p->P.seg_base + (p->P.seg_rem ? 1 : 0);
            ms = std::max(ms, mlen <= 8 ? 8 : (mlen <= 16 ? 16 : 32));
            for (int64_t l = 0; l < p->P.lines; l += LB) blocks.push_back(make_int2(g, (int)l));
        }
        if (smem > 200 * 1024) return false;
        R.kind.dtype = dtype;
        R.kind.q = cls_.deriv.q;
        if (role != R_DERIV) R.kind.q = cls_.filt.q;
        R.kind.M = role == R_DERIV ? cls_.deriv.M : cls_.filt.M;
        R.kind.xmode = k == 0 ? 1 : 0;
        R.kind.threads = threads;
        R.kind.smem = smem;
        R.kind.ms = ms;
        R.per_member = false;
        upload(R.plans, ctx_, plans, st_);
        upload(R.blocks, ctx_, blocks, st_);
        R.nblocks = (int)blocks.size();
        CLES_CUDA(cudaStreamSynchronize(st_));
        return true;
    }

    // The launch shape the tuned choice is kept for: operator, direction,
    // element type, bandwidth, periodicity, the largest segment count and the
    // total line count to within a factor of two (so compositions that differ
    // by a few members reuse the choice instead of timing again).
    std::string role_key(int role, int k) const {
        int smax = 0;
        int64_t lines = 0;
        for (Member* m : order_) {
            smax = std::max(smax, plan_of(*m, role, k)->P.S);
            lines += m->cells / m->n[k];
        }
        int lg = 0;
        while ((int64_t)1 << (lg + 1) <= lines) ++lg;
        return std::to_string(role) + "/" + std::to_string(k) + "/" + std::to_string(sizeof(F)) + "/" +
               std::to_string(cls_.deriv.q) + std::to_string(cls_.filt.q) + "/" + std::to_string(periodic_of(k)) +
               "/S" + std::to_string(smax) + "/L" + std::to_string(lg);
    }
    int periodic_of(int k) const { return cls_.bc[k][0] == CLES_BC_PERIODIC ? 1 : 0; }

    // the autotuner: time every candidate thread count on this batch's fields
    void tune_roles() {
        for (int r = 0; r < 3; ++r)
            for (int k = 0; k < 3; ++k) {
                roles_[r][k].nblocks = 0;
                tuned_ms_[r][k] = 0.0;
                if (!act_[k]) continue;
                if (r == R_QFILT && cls_.filter_interval == 0) continue;
                if (strategy_ == CLES_BATCH_PER_MEMBER) { set_role(r, k, 0); continue; }
                const std::string key = role_key(r, k);
                auto& cache = batch_tuning_cache();
                auto it = strategy_ == CLES_BATCH_AUTO ? cache.find(key) : cache.end();
                if (it != cache.end() && (it->second == 0 || role_tables(r, k, it->second, roles_[r][k]))) {
                    set_role(r, k, it->second);
                    continue;
                }
                roles_[r][k].per_member = false;
                int best = -1;
                float best_ms = 1e30f;
                for (int th : {128, 256, 512}) {
                    Role R;
                    if (!role_tables(r, k, th, R)) continue;
                    const bool f64 = R.kind.dtype == CLES_F64;
                    const void* in = f64 && r == R_QFILT ? static_cast<const void*>(Q_.p) : static_cast<const void*>(prim_.p);
                    void* out = r == R_QFILT ? flux_.p : scratch_.p;
                    launch_compact_batch(R.kind, R.plans.as<BatchLinePlan>(), R.blocks.as<int2>(), R.nblocks, in, out,
                                         ct_, 1, OUT_STORE, nullptr, nullptr, 0, 0, 0, st_);
                    CLES_CUDA(cudaEventRecord(ev0_, st_));
                    const int reps = 3;
                    for (int i = 0; i < reps; ++i)
                        launch_compact_batch(R.kind, R.plans.as<BatchLinePlan>(), R.blocks.as<int2>(), R.nblocks, in,
                                             out, ct_, 1, OUT_STORE, nullptr, nullptr, 0, 0, 0, st_);
                    CLES_CUDA(cudaEventRecord(ev1_, st_));
                    CLES_CUDA(cudaEventSynchronize(ev1_));
                    float ms = 0;
                    CLES_CUDA(cudaEventElapsedTime(&ms, ev0_, ev1_));
                    ms /= reps;
                    if (ms < best_ms) { best_ms = ms; best = th; }
                }
                // the other strategy: every member's one-grid kernel, on the auxiliary streams
                if (strategy_ == CLES_BATCH_AUTO) {
                    const bool f64 = (r == R_QFILT) || sizeof(F) == 8;
                    const void* in = f64 && r == R_QFILT ? static_cast<const void*>(Q_.p) : static_cast<const void*>(prim_.p);
                    void* out = r == R_QFILT ? flux_.p : scratch_.p;
                    along_members(r, k, in, out, 1, OUT_STORE, 0);
                    CLES_CUDA(cudaEventRecord(ev0_, st_));
                    const int reps = 3;
                    for (int i = 0; i < reps; ++i) along_members(r, k, in, out, 1, OUT_STORE, 0);
                    CLES_CUDA(cudaEventRecord(ev1_, st_));
                    CLES_CUDA(cudaEventSynchronize(ev1_));
                    float ms = 0;
                    CLES_CUDA(cudaEventElapsedTime(&ms, ev0_, ev1_));
                    ms /= reps;
                    if (ms < best_ms) { best_ms = ms; best = 0; }   // 0 threads: per-member launches
                }
                if (best < 0) throw Error(CLES_EINVAL, "no batched launch shape fits the lines of this batch");
                if (strategy_ == CLES_BATCH_AUTO) cache[key] = best;
                tuned_ms_[r][k] = best_ms;
                set_role(r, k, best);
            }
    }
    void set_role(int r, int k, int choice) {
        if (choice == 0) {
            Role& R = roles_[r][k];
            R.plans.release();
            R.blocks.release();
            R.nblocks = (int)order_.size();   // members, for the statistics
            R.kind = BatchLaunchKind{};
            R.per_member = true;
        } else {
            roles_[r][k].per_member = false;
            role_tables(r, k, choice, roles_[r][k]);
        }
    }

    // ------------------------------------------------------------ the step --
    const CompactPlan* solo_plan_of(const Member& m, int role, int k) const {
        if (role == R_DERIV) return m.sderiv[k].get();
        if (role == R_FILT) return m.sfilt[k].get();
        return m.sqfilt[k] ? m.sqfilt[k].get() : m.sfilt[k].get();
    }

    // Each member's one-grid kernel (the solver's own choice of tile, warp or
    // generic kernel) on its views of the arena, spread over the auxiliary
    // streams between a fork and a join on the batch stream.  OUT_RK tries the
    // fused update; a member whose kernel cannot fuse it gets a subtracting
    // store, and its `rk_fused_` entry says so for the separate RK pass.
    void along_members(int role, int k, const void* in, void* out, int count, int mode, int stage) {
        const size_t el = (role == R_QFILT || sizeof(F) == 8) ? sizeof(double) : sizeof(float);
        CLES_CUDA(cudaEventRecord(fork_ev_, st_));
        const int ns = std::min<int>(kAuxStreams, (int)order_.size());
        for (int i = 0; i < ns; ++i) CLES_CUDA(cudaStreamWaitEvent(aux_[i], fork_ev_, 0));
        for (size_t g = 0; g < order_.size(); ++g) {
            const Member& m = *order_[g];
            const CompactPlan* p = solo_plan_of(m, role, k);
            cudaStream_t st = aux_[g % ns];
            const int64_t sy = m.n[0], sz = (int64_t)m.n[0] * m.n[1];
            const FieldView vin{const_cast<char*>(static_cast<const char*>(in)) + el * (size_t)m.off, ct_, sy, sz};
            const FieldView vout{static_cast<char*>(out) + el * (size_t)m.off, ct_, sy, sz};
            if (mode == OUT_RK) {
                const RkEpilogue rk{Q_.as<double>() + m.off, du_.as<double>() + m.off, kLsrkA[stage], kLsrkB[stage],
                                    0.0, clk_.as<double>() + 16 * g + DC_DT};
                const bool fused = launch_compact_rk(*p, vin, vout, count, rk, st);
                if (!fused) launch_compact(*p, vin, vout, count, OUT_SUBTRACT, st);
                rk_fused_[g] = fused ? 1 : 0;
            } else {
                launch_compact(*p, vin, vout, count, mode, st);
            }
        }
        for (int i = 0; i < ns; ++i) {
            CLES_CUDA(cudaEventRecord(aux_ev_[i], aux_[i]));
            CLES_CUDA(cudaStreamWaitEvent(st_, aux_ev_[i], 0));
        }
    }

    void along(int role, int k, const void* in, void* out, int count, int mode, int stage = 0, int skip = 0) {
        Role& R = roles_[role][k];
        if (R.per_member) {
            along_members(role, k, in, out, count, mode, stage);
            return;
        }
        launch_compact_batch(R.kind, R.plans.as<BatchLinePlan>(), R.blocks.as<int2>(), R.nblocks, in, out, ct_, count,
                             mode, Q_.as<double>(), du_.as<double>(), kLsrkA[stage], kLsrkB[stage], skip, st_);
        if (mode == OUT_RK) std::fill(rk_fused_.begin(), rk_fused_.end(), 1);
    }
    void smooth(F* f, int count) {
        for (int k = 0; k < 3; ++k)
            if (act_[k]) along(R_FILT, k, f, f, count, OUT_STORE);
    }
    void primitives() {
        BatchOps<F>::primitives(Q_.as<double>(), prim_.as<F>(), ct_, Ns_, pc_, cls_.art_enabled, mc_.as<double>(),
                                tmap_.as<int>(), st_);
    }
    void bcs() {
        batch_bc(Q_.as<double>(), grids_.as<BatchGrid>(), faces_.as<BatchFace>(), nfaces_, ct_, Ns_, st_);
    }
    void delta4(const F* f0, const F* f1, F* o0, F* o1, int p0, int p1) {
        BatchOps<F>::delta4(f0, f1, o0, o1, p0, p1, grids_.as<BatchGrid>(), tiles_.as<BatchTile>(), ntiles_, ct_, st_);
    }

    void artificial() {
        // compute_artificial! (src/artificial.jl:261-359), the batched form of
        // the solver's: the same passes in the same order
        if (!cls_.art_enabled) return;
        using PW = Pointwise<F>;
        F* strain = field(scratch_, 0);
        F* sensor = field(scratch_, 1);
        F* sensor_e = field(scratch_, 2);
        F* tmp_a = field(scratch_, 3);
        F* tmp_b = field(scratch_, 4);
        PW::strain(g_u_.as<F>(), strain, ct_, st_);
        delta4(strain, field(prim_, P_Y0 + Ns_), sensor, sensor_e, 2, 1);
        smooth(sensor, 2);
        PW::art_coef(sensor, sensor_e, prim_.as<F>(), g_u_.as<F>(), art_.as<F>(), ct_, cls_.C_mu, cls_.C_beta,
                     cls_.C_kappa, cls_.beta_sensor == CLES_BETA_GATED_STRAIN, st_);
        if (cls_.beta_sensor == CLES_BETA_DILATATION) {
            PW::dilatation(g_u_.as<F>(), tmp_a, tmp_b, ct_, st_);
            delta4(tmp_a, nullptr, sensor, nullptr, 2, 2);
            smooth(sensor, 1);
            PW::beta_dilatation(sensor, prim_.as<F>(), tmp_b, art_.as<F>(), ct_, cls_.C_beta, st_);
        }
        if (Ns_ > 1) {
            for (int sp = 0; sp < Ns_; ++sp) {
                delta4(field(prim_, P_Y0 + sp), nullptr, tmp_a, nullptr, 1, 1);
                smooth(tmp_a, 1);
                PW::dart(tmp_a, prim_.as<F>(), art_.as<F>(), ct_, cls_.C_D, sp, st_);
            }
        }
    }

    void rhs_and_update(bool primitives_current, int stage) {
        using PW = Pointwise<F>;
        if (!primitives_current) primitives();
        for (int k = 0; k < 3; ++k)
            if (act_[k]) along(R_DERIV, k, field(prim_, P_U), g_u_.as<F>() + (size_t)ct_ * 3 * k, 3, OUT_STORE);
        artificial();
        const int ngty = Ns_ == 1 ? 1 : 1 + Ns_;
        for (int k = 0; k < 3; ++k)
            if (act_[k]) along(R_DERIV, k, field(prim_, P_T), gty_.as<F>() + (size_t)ct_ * ngty * k, ngty, OUT_STORE);
        BatchOps<F>::fluxes(Q_.as<double>(), prim_.as<F>(), g_u_.as<F>(), gty_.as<F>(), art_.as<F>(), flux_.as<F>(),
                            ct_, Ns_, pc_, cls_.mu0, cls_.Pr, cls_.Sc, mc_.as<double>(), tmap_.as<int>(), st_);
        // dQ = -sum_d D_d(F_d) with the RK update in the last direction's store
        // (y, x, z on 3-D grids, as the solver orders them)
        int order[3] = {0, 1, 2};
        if (act_[0] && act_[1] && act_[2]) { order[0] = 1; order[1] = 0; }
        int nact = 0, seen = 0;
        for (int k = 0; k < 3; ++k) nact += act_[k] ? 1 : 0;
        if (nact == 1) CLES_CUDA(cudaMemsetAsync(dQ_.p, 0, dQ_.bytes, st_));
        for (int o = 0; o < 3; ++o) {
            const int k = order[o];
            if (!act_[k]) continue;
            ++seen;
            const F* fin = flux_.as<F>() + (size_t)ct_ * ncons_ * k;
            const int mode = seen == nact ? OUT_RK : (seen == 1 ? OUT_NEGATE : OUT_SUBTRACT);
            along(R_DERIV, k, fin, dQ_.p, ncons_, mode, stage);
        }
        // members whose last divergence could not apply the update (per-member
        // kernels without the fused store): one batched RK pass, each with its dt
        if (roles_[R_DERIV][last_dim()].per_member)
            BatchOps<F>::lsrk(Q_.as<double>(), du_.as<double>(), dQ_.as<F>(), ct_, ncons_, tmap_.as<int>(),
                              grids_.as<BatchGrid>(), need_lsrk_.as<int>(), kLsrkA[stage], kLsrkB[stage], st_);
    }
    int last_dim() const {
        int l = 0;
        for (int k = 0; k < 3; ++k)
            if (act_[k]) l = k;
        return l;
    }

    void capture() {
        rk_fused_.assign(order_.size(), 1);
        need_lsrk_.release();
        need_lsrk_.alloc(ctx_, sizeof(int) * order_.size());
        cudaGraph_t g = nullptr;
        const cudaStream_t user = st_;
        st_ = cap_st_;
        const int64_t l0 = launch_count();
        CLES_CUDA(cudaStreamBeginCapture(st_, cudaStreamCaptureModeRelaxed));
        try {
            using PW = Pointwise<F>;
            bcs();
            primitives();
            BatchOps<F>::rate_clock(Q_.as<double>(), prim_.as<F>(), art_.as<F>(), grids_.as<BatchGrid>(),
                                    (int)order_.size(), chunks_.as<BatchChunk>(), nchunks_, chunk_first_.as<int>(),
                                    part_.as<double>(), ct_, Ns_, cls_.mu0, cls_.Pr, cls_.Sc, st_);
            for (int stage = 0; stage < 5; ++stage) {
                if (stage > 0) bcs();
                rhs_and_update(stage == 0, stage);
            }
            bcs();
            batch_clock_after(grids_.as<BatchGrid>(), (int)order_.size(), st_);
            if (cls_.filter_interval > 0)
                for (int k = 0; k < 3; ++k)
                    if (act_[k]) along(R_QFILT, k, Q_.p, Q_.p, ncons_, OUT_STORE, 0, cls_.filter_interval);
            CLES_CUDA(cudaMemcpyAsync(host_clk_, clk_.p, sizeof(double) * 16 * order_.size(), cudaMemcpyDeviceToHost,
                                      st_));
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
        launches_per_step_ = (int)(launch_count() - l0);
        // which members the separate RK pass updates (read by the graph when it runs)
        std::vector<int> need(order_.size());
        for (size_t i = 0; i < order_.size(); ++i) need[i] = rk_fused_[i] ? 0 : 1;
        CLES_CUDA(cudaMemcpy(need_lsrk_.p, need.data(), sizeof(int) * need.size(), cudaMemcpyHostToDevice));
        const cudaError_t e = cudaGraphInstantiate(&exec_, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) throw Error(CLES_ECUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
    }

    cles_ctx* ctx_;
    cudaStream_t st_ = nullptr, cap_st_ = nullptr;
    cudaEvent_t ev0_ = nullptr, ev1_ = nullptr;
    cudaStream_t aux_[kAuxStreams] = {};
    cudaEvent_t aux_ev_[kAuxStreams] = {}, fork_ev_ = nullptr;
    std::vector<int> rk_fused_;   // per member: its RK update ran inside the last divergence
    DevBuf need_lsrk_;            // per member: 1 when the separate batched RK pass must update it
    cles_solver_desc cls_;
    int Ns_ = 1, ncons_ = 5;
    bool act_[3] = {false, false, false};
    PhysConst pc_{};
    std::vector<std::unique_ptr<Member>> members_;
    std::vector<Member*> order_;
    std::vector<int64_t> cancelled_;
    int64_t next_id_ = 1;
    bool dirty_ = false, launched_ = false;
    int strategy_ = CLES_BATCH_AUTO;
    int64_t ct_ = 0;
    DevBuf Q_, art_, clk_;
    DevBuf du_, dQ_, prim_, g_u_, gty_, scratch_, flux_, part_;
    DevBuf grids_, tiles_, faces_, chunks_, chunk_first_, mc_, tmap_;
    int ntiles_ = 0, nfaces_ = 0, nchunks_ = 0;
    Role roles_[3][3];
    double tuned_ms_[3][3] = {};
    double* host_clk_ = nullptr;
    size_t host_clk_cap_ = 0;
    cudaGraphExec_t exec_ = nullptr;
    int compositions_ = 0;
    int64_t steps_ = 0;
    int launches_per_step_ = 0;
};

std::unique_ptr<BatchBase> make_batch(cles_ctx* ctx, const cles_solver_desc& cls) {
    check_supported(cls);
    if (cls.precision == CLES_PREC_MIXED) return std::unique_ptr<BatchBase>(new Batch<float>(ctx, cls));
    return std::unique_ptr<BatchBase>(new Batch<double>(ctx, cls));
}

bool batch_compatible(const cles_solver_desc& cls, const cles_solver_desc& d) {
    try {
        check_supported(d);
        check_class(cls, d);
        return true;
    } catch (const Error&) {
        return false;
    }
}

}  // namespace cles
