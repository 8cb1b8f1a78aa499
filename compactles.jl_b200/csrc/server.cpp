// Continuous-batching server of independent solves on one device (cles_server_*).
//
// A tick admits queued requests in arrival order while the active count and
// the HBM budget allow, enqueues one run! step for every running request,
// waits for them together, and retires finished or failed requests, returning
// their memory to the budget.  Two ways to hold a request:
//   * its own stream and device-resident solver, one CUDA-graph launch per
//     step (see SolverBase::graph_begin);
//   * with batching on (cles_server_set_batching), a request the batch path
//     supports joins a batch of its physics class (batch.cpp): the members'
//     fields share one arena and one captured step of O(stages) launches
//     advances them all, each with its own dt and end time.  Requests admitted
//     while others run join the running batch at its next step.  With a
//     member limit a class spreads over several batches, each on its own
//     stream, whose steps overlap on the device.
// Requests never share reductions or change each other's arithmetic, so a
// result does not depend on which other requests were in flight.

#include <chrono>
#include <cstring>
#include <deque>
#include <map>
#include <vector>

#include "solver.h"

using namespace cles;

namespace {

struct Request {
    int64_t id = 0;
    cles_solver_desc desc{};
    std::vector<double> stretch[3][2];   // owned copies of the descriptor's Stretch samples
    std::vector<double> Q0;
    int layout = CLES_LAYOUT_PADDED;
    double tfinal = 0.0;
    int64_t nmax = 0;
    int state = CLES_REQ_QUEUED;
    int failure = CLES_FAIL_NONE;
    int64_t steps = 0;
    double t = 0.0;
    double submit_s = 0.0, admit_s = -1.0, done_s = -1.0;
    size_t bytes = 0;
    bool graph = true;
    cles_ctx ctx{};
    std::unique_ptr<SolverBase> solver;
    int batch = -1;            // index of the batch slot holding it, or -1
    int64_t member = 0;        // its id in that batch
    std::vector<double> Qout;
};

// One batch of a physics class with its own stream.
struct BatchSlot {
    cles_ctx ctx{};
    cles_solver_desc cls{};
    std::unique_ptr<BatchBase> b;
    int members = 0;           // requests currently held
};

size_t state_elems(const cles_solver_desc& d, int layout) {
    size_t n = (size_t)(d.n_species + 4);
    for (int k = 0; k < 3; ++k) {
        const int pad = (layout == CLES_LAYOUT_PADDED && d.n_global[k] > 1) ? d.n_halo : 0;
        n *= (size_t)(d.n_global[k] + 2 * pad);
    }
    return n;
}

}  // namespace

struct cles_server {
    int device = 0;
    size_t budget = 0;
    int max_active = 0;
    size_t used = 0;
    int64_t next_id = 1;
    std::deque<int64_t> queue;
    std::vector<int64_t> running;
    std::map<int64_t, std::unique_ptr<Request>> reqs;
    bool batching = false;
    int batch_limit = 0;   // members per batch (0 = no limit)
    std::vector<std::unique_ptr<BatchSlot>> batches;
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
    double now() const {
        return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
    void release(Request& r) {
        r.solver.reset();
        if (r.ctx.stream) {
            cudaStreamDestroy(r.ctx.stream);
            r.ctx.stream = nullptr;
        }
        if (r.batch >= 0) {
            BatchSlot& b = *batches[r.batch];
            b.members -= 1;
            // an emptied batch is replaced by a fresh one, which frees its arena
            if (b.members == 0) b.b = make_batch(&b.ctx, b.cls);
            r.batch = -1;
        }
        used -= r.bytes;
    }
    // the batch slot of r's class, created on first use
    int batch_for(const cles_solver_desc& d) {
        for (size_t i = 0; i < batches.size(); ++i)
            if ((batch_limit <= 0 || batches[i]->members < batch_limit) && batch_compatible(batches[i]->cls, d))
                return (int)i;
        auto slot = std::make_unique<BatchSlot>();
        slot->ctx.device = device;
        CLES_CUDA(cudaStreamCreateWithFlags(&slot->ctx.stream, cudaStreamNonBlocking));
        slot->cls = d;
        try {
            slot->b = make_batch(&slot->ctx, d);
        } catch (...) {
            cudaStreamDestroy(slot->ctx.stream);
            throw;
        }
        batches.push_back(std::move(slot));
        return (int)batches.size() - 1;
    }
    ~cles_server() {
        for (auto& b : batches) {
            b->b.reset();
            if (b->ctx.stream) cudaStreamDestroy(b->ctx.stream);
        }
    }
};

#define SAPI_BEGIN try {
#define SAPI_END                                        \
    }                                                   \
    catch (const cles::Error& e) {                      \
        set_last_error(e.what());                       \
        return e.code;                                  \
    }                                                   \
    catch (const std::exception& e) {                   \
        set_last_error(e.what());                       \
        return CLES_EINVAL;                             \
    }                                                   \
    set_last_error("");                                 \
    return CLES_OK;

extern "C" {

int cles_run_graph(cles_solver* s, double tfinal, int64_t nmax, cles_run_result* out);

int cles_server_create(int device, size_t hbm_budget_bytes, int max_active, cles_server** out) {
    SAPI_BEGIN
    if (!out) throw Error(CLES_EINVAL, "null output pointer");
    if (max_active < 1) throw Error(CLES_EINVAL, "max_active must be >= 1");
    int count = 0;
    CLES_CUDA(cudaGetDeviceCount(&count));
    if (device < 0 || device >= count) throw Error(CLES_EINVAL, "no such CUDA device");
    auto* s = new cles_server();
    s->device = device;
    s->budget = hbm_budget_bytes;
    s->max_active = max_active;
    *out = s;
    SAPI_END
}

void cles_server_destroy(cles_server* s) {
    if (!s) return;
    cudaSetDevice(s->device);
    for (auto& kv : s->reqs) s->release(*kv.second);
    delete s;
}

int cles_server_submit(cles_server* s, const cles_solver_desc* desc, const double* Q0, int layout, double tfinal,
                       int64_t nmax, int64_t* id) {
    SAPI_BEGIN
    if (!s || !desc || !Q0 || !id) throw Error(CLES_EINVAL, "null argument");
    if (layout != CLES_LAYOUT_PADDED && layout != CLES_LAYOUT_INTERIOR) throw Error(CLES_EINVAL, "unknown layout");
    auto r = std::make_unique<Request>();
    r->id = s->next_id++;
    r->desc = *desc;
    // the solver is created at admission, after the caller's arrays may be gone
    for (int k = 0; k < 3; ++k)
        if (desc->stretch_x[k] && desc->stretch_dxdxi[k]) {
            const int n = desc->n_global[k];
            r->stretch[k][0].assign(desc->stretch_x[k], desc->stretch_x[k] + n);
            r->stretch[k][1].assign(desc->stretch_dxdxi[k], desc->stretch_dxdxi[k] + n);
            r->desc.stretch_x[k] = r->stretch[k][0].data();
            r->desc.stretch_dxdxi[k] = r->stretch[k][1].data();
        }
    r->layout = layout;
    r->tfinal = tfinal;
    r->nmax = nmax;
    r->Q0.assign(Q0, Q0 + state_elems(*desc, layout));
    r->bytes = solver_bytes_estimate(*desc);
    r->graph = desc->control.retries == 0 && desc->control.predict == 0 && desc->control.max_growth == 0;
    r->submit_s = s->now();
    if (s->budget && r->bytes > s->budget) throw Error(CLES_ENOMEM, "request needs more HBM than the server budget");
    *id = r->id;
    s->queue.push_back(r->id);
    s->reqs[r->id] = std::move(r);
    SAPI_END
}

int cles_server_tick(cles_server* s, int* n_running, int* n_queued) {
    SAPI_BEGIN
    if (!s) throw Error(CLES_EINVAL, "null server");
    CLES_CUDA(cudaSetDevice(s->device));
    // admit in arrival order while slots and memory allow
    while (!s->queue.empty() && (int)s->running.size() < s->max_active) {
        Request& r = *s->reqs[s->queue.front()];
        if (s->budget && s->used + r.bytes > s->budget) break;
        if (s->batching && r.graph && batch_compatible(r.desc, r.desc)) {
            s->used += r.bytes;
            try {
                const int bi = s->batch_for(r.desc);
                r.member = s->batches[bi]->b->add(r.desc, r.Q0.data(), r.layout, r.tfinal, r.nmax, s->now());
                r.batch = bi;
                s->batches[bi]->members += 1;
            } catch (const Error& e) {
                s->used -= r.bytes;
                if (e.code == CLES_ENOMEM) break;
                r.state = CLES_REQ_FAILED;
                r.done_s = s->now();
                s->queue.pop_front();
                continue;
            }
            r.Q0.clear();
            r.Q0.shrink_to_fit();
            r.state = CLES_REQ_RUNNING;
            r.admit_s = s->now();
            s->queue.pop_front();
            s->running.push_back(r.id);
            continue;
        }
        r.ctx.device = s->device;
        CLES_CUDA(cudaStreamCreateWithFlags(&r.ctx.stream, cudaStreamNonBlocking));
        s->used += r.bytes;
        try {
            r.solver = make_solver(&r.ctx, r.desc);
            r.solver->set_state(r.Q0.data(), r.layout);
            if (r.graph) r.solver->graph_begin(r.tfinal, r.nmax);
        } catch (const Error& e) {
            s->release(r);
            if (e.code == CLES_ENOMEM) break;  // stays queued until memory frees up
            r.state = CLES_REQ_FAILED;
            r.done_s = s->now();
            s->queue.pop_front();
            continue;
        }
        r.Q0.clear();
        r.Q0.shrink_to_fit();
        r.state = CLES_REQ_RUNNING;
        r.admit_s = s->now();
        s->queue.pop_front();
        s->running.push_back(r.id);
    }
    // one step for every running request (every batch one captured step);
    // host-stepped ones run synchronously
    const double tnow = s->now();
    for (auto& b : s->batches)
        if (b->members > 0) b->b->launch(tnow);
    for (int64_t id : s->running) {
        Request& r = *s->reqs[id];
        if (r.graph && r.batch < 0) r.solver->graph_launch();
    }
    for (int64_t id : s->running) {
        Request& r = *s->reqs[id];
        if (!r.graph) {
            cles_run_result res{};
            const int rc = r.solver->run(r.tfinal, r.solver->step_count + 1, &res);
            if (rc == CLES_EFAILURE) r.failure = res.failure;
        }
    }
    for (auto& b : s->batches)
        if (b->members > 0) b->b->collect(s->now());
    for (int64_t id : s->running)
        if (s->reqs[id]->batch < 0) CLES_CUDA(cudaStreamSynchronize(s->reqs[id]->ctx.stream));
    // retire finished and failed requests
    std::vector<int64_t> still;
    for (int64_t id : s->running) {
        Request& r = *s->reqs[id];
        bool done = false;
        if (r.batch >= 0) {
            BatchBase& B = *s->batches[r.batch]->b;
            cles_request_status bs{};
            B.status(r.member, &bs);
            r.t = bs.t;
            r.steps = bs.steps;
            r.failure = bs.failure;
            done = bs.state == CLES_REQ_DONE;
            if (done) {
                r.Qout.resize(state_elems(r.desc, r.layout));
                B.fetch(r.member, r.Qout.data(), r.layout);
                r.state = CLES_REQ_DONE;
                r.done_s = s->now();
                s->release(r);
            } else if (bs.state == CLES_REQ_FAILED) {
                r.state = CLES_REQ_FAILED;
                r.done_s = s->now();
                s->release(r);
            } else {
                still.push_back(id);
            }
            continue;
        }
        if (r.graph) {
            const double* clk = r.solver->graph_clock();
            r.t = clk[DC_T];
            r.steps = (int64_t)clk[DC_STEP];
            if (clk[DC_FAILURE] != 0.0) r.failure = (int)clk[DC_FAILURE];
            done = clk[DC_DONE] != 0.0;
        } else {
            r.t = r.solver->t;
            r.steps = r.solver->step_count;
            done = !(r.t < r.tfinal && r.steps < r.nmax);
        }
        if (r.failure != CLES_FAIL_NONE) {
            r.state = CLES_REQ_FAILED;
            r.done_s = s->now();
            s->release(r);
        } else if (done) {
            if (r.graph) r.solver->graph_end();
            r.Qout.resize(state_elems(r.desc, r.layout));
            r.solver->get_state(r.Qout.data(), r.layout);
            r.state = CLES_REQ_DONE;
            r.done_s = s->now();
            s->release(r);
        } else {
            still.push_back(id);
        }
    }
    s->running.swap(still);
    if (n_running) *n_running = (int)s->running.size();
    if (n_queued) *n_queued = (int)s->queue.size();
    SAPI_END
}

int cles_server_set_batching(cles_server* s, int on, int max_members) {
    SAPI_BEGIN
    if (!s) throw Error(CLES_EINVAL, "null server");
    if (max_members < 0) throw Error(CLES_EINVAL, "max_members must be >= 0");
    s->batching = on != 0;
    s->batch_limit = max_members;
    SAPI_END
}

int cles_server_status(cles_server* s, int64_t id, cles_request_status* out) {
    SAPI_BEGIN
    if (!s || !out) throw Error(CLES_EINVAL, "null argument");
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) throw Error(CLES_EINVAL, "unknown request id");
    const Request& r = *it->second;
    out->state = r.state;
    out->failure = r.failure;
    out->steps = r.steps;
    out->t = r.t;
    out->submit_s = r.submit_s;
    out->admit_s = r.admit_s;
    out->done_s = r.done_s;
    out->device_bytes = r.bytes;
    SAPI_END
}

int cles_server_fetch(cles_server* s, int64_t id, double* Q_host) {
    SAPI_BEGIN
    if (!s || !Q_host) throw Error(CLES_EINVAL, "null argument");
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) throw Error(CLES_EINVAL, "unknown request id");
    Request& r = *it->second;
    if (r.state != CLES_REQ_DONE) throw Error(CLES_EINVAL, "request has not finished successfully");
    std::memcpy(Q_host, r.Qout.data(), sizeof(double) * r.Qout.size());
    s->reqs.erase(it);
    SAPI_END
}

int cles_server_cancel(cles_server* s, int64_t id) {
    SAPI_BEGIN
    if (!s) throw Error(CLES_EINVAL, "null server");
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) throw Error(CLES_EINVAL, "unknown request id");
    Request& r = *it->second;
    if (r.state == CLES_REQ_QUEUED) {
        for (auto q = s->queue.begin(); q != s->queue.end(); ++q)
            if (*q == id) { s->queue.erase(q); break; }
    } else if (r.state == CLES_REQ_RUNNING) {
        if (r.batch >= 0) s->batches[r.batch]->b->remove(r.member, s->now());
        else CLES_CUDA(cudaStreamSynchronize(r.ctx.stream));
        s->release(r);
        for (auto q = s->running.begin(); q != s->running.end(); ++q)
            if (*q == id) { s->running.erase(q); break; }
    } else {
        return CLES_OK;
    }
    r.state = CLES_REQ_CANCELLED;
    r.done_s = s->now();
    SAPI_END
}

}  // extern "C"
