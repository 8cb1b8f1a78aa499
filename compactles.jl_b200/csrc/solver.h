// Device-resident solver runtime (the B200 counterpart of the reference's
// Solver + compute_rhs! + step! + max_rate + filter_state! + run!).
#pragma once

#include <atomic>
#include <memory>

#include "pointwise.h"

struct cles_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    size_t budget = 0;     // 0 = unlimited
    size_t allocated = 0;
    // the caller's handle plus one per live plan, solver or batch made with
    // it: cles_ctx_destroy only drops the caller's, so objects destroyed after
    // their context (in any order) still find it
    std::atomic<int> refs{1};
};

namespace cles {
inline cles_ctx* ctx_retain(cles_ctx* c) {
    c->refs.fetch_add(1);
    return c;
}
inline void ctx_release(cles_ctx* c) {
    if (c && c->refs.fetch_sub(1) == 1) delete c;
}
}  // namespace cles

namespace cles {

// Device allocation charged against the context's HBM budget.
struct DevBuf {
    cles_ctx* ctx = nullptr;
    void* p = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { release(); }
    void alloc(cles_ctx* c, size_t b);
    void release();
    template <typename T> T* as() const { return reinterpret_cast<T*>(p); }
};

class SolverBase {
public:
    virtual ~SolverBase() = default;
    virtual void apply_bcs() = 0;
    virtual void max_rate(double* rate, double* rho_min) = 0;
    virtual void compute_rhs(bool primitives_current) = 0;
    virtual void step(double dt, bool prepared) = 0;
    virtual void filter_state() = 0;
    virtual int run(double tfinal, int64_t nmax, cles_run_result* res) = 0;
    virtual void set_state(const double* Q, int layout) = 0;
    virtual void get_state(double* Q, int layout) = 0;
    virtual void get_rhs(double* dQ, int layout) = 0;
    virtual void get_field(int which, double* host, int layout) = 0;
    virtual double kinetic_energy() = 0;
    virtual double dissipation_rate() = 0;
    virtual double* state_device() = 0;
    virtual cles_solver_info info() const = 0;

    // Graph mode: one run! iteration per CUDA-graph launch, with the timestep,
    // the step-control floors and the clock kept on the device (no host read
    // inside a step).  graph_begin captures the graphs; graph_launch enqueues one
    // step and an asynchronous read of the clock into pinned memory, which
    // graph_clock returns once the stream has been synchronised; graph_end
    // copies the clock back into t / step.  No rate prediction, growth cap or
    // rollback in this mode.
    virtual void graph_begin(double tfinal, int64_t nmax) = 0;
    virtual void graph_launch() = 0;
    virtual const double* graph_clock() const = 0;
    virtual void graph_end() = 0;
    virtual cudaStream_t stream() const = 0;
    // switch!(::SwitchableBC) on face (dim, side)
    virtual void switch_bc(int dim, int side) = 0;
    virtual void set_face_fn(int dim, int side, int which, cles_face_fn fn, void* user) = 0;
    virtual bool bc_switched(int dim, int side) const = 0;
    // this rank's place in a decomposition (nullptr on an undecomposed solver)
    virtual const cles_decomp* decomposition() const { return nullptr; }

    cles_solver_desc desc{};
    double t = 0.0, tstage = 0.0, dt_prev = 0.0, rate_prev = 0.0, cfl = 0.5;
    int64_t step_count = 0;
};

std::unique_ptr<SolverBase> make_solver(cles_ctx* ctx, const cles_solver_desc& desc,
                                        const cles_decomp* decomp = nullptr, const cles_exchange* ex = nullptr);
// Device bytes a solver of `desc` allocates (fields and plan tables), for admission control.
size_t solver_bytes_estimate(const cles_solver_desc& desc);
// run! in graph mode on one solver (same contract as SolverBase::run without retries).
int run_graph(SolverBase& s, double tfinal, int64_t nmax, cles_run_result* res);

// Host layout transfer of a component-slowest state between a host array in
// `layout` and an interior device array (cudaMemcpy3DAsync per component).
void copy_state_h2d(double* dev, const double* host, const int n[3], const int pad[3], int ncomp, int layout,
                    cudaStream_t st);
void copy_state_d2h(double* host, const double* dev, const int n[3], const int pad[3], int ncomp, int layout,
                    cudaStream_t st);

int check_step(const cles_step_control& c, double dt, double rho_min, double dt_seen);

// Many solves of one physics class advanced together (batch.cpp).
class BatchBase {
public:
    virtual ~BatchBase() = default;
    virtual int64_t add(const cles_solver_desc& d, const double* Q0, int layout, double tfinal, int64_t nmax,
                        double now) = 0;
    virtual int step(double now) = 0;          // launch + collect; returns the members still running
    virtual void launch(double now) = 0;       // (re)compose if needed and enqueue one step on the batch's stream
    virtual int collect(double now) = 0;       // wait for it and update the members' clocks
    virtual int n_active() const = 0;
    virtual void remove(int64_t id, double now) = 0;
    virtual void status(int64_t id, cles_request_status* out) const = 0;
    virtual void fetch(int64_t id, double* Q, int layout) = 0;
    virtual void stats(cles_batch_stats* s) const = 0;
    virtual void set_strategy(int strategy) = 0;
};
std::unique_ptr<BatchBase> make_batch(cles_ctx* ctx, const cles_solver_desc& cls);
// d fits a batch of class cls (supported and equal in every class field)
bool batch_compatible(const cles_solver_desc& cls, const cles_solver_desc& d);

// LSRK(5,4) coefficients A, B, C per stage (src/timestep.jl:5-21)
extern const double kLsrkA[5], kLsrkB[5], kLsrkC[5];

}  // namespace cles
