// In-process exchange among the ranks of a decomposed grid (cles_local_group_*).
//
// Every rank is one host thread of this process with its own solver and
// stream (on one GPU or several).  An exchange records a "sends ready" event
// on the caller's stream and publishes it with the caller's buffers; after a
// host barrier each rank's stream waits on its peers' ready events and copies
// what it receives with cudaMemcpyAsync, then records a "copied" event; after
// a second barrier each stream waits on the copied events of the peers that
// read its buffers, so nothing later on it overwrites them too early.  The
// host never waits for the device here, and no kernel waits on another rank:
// the ordering is stream-event dependencies.  The barriers are bounded by the
// group's timeout, after which (or after cles_local_group_abort) every
// barrier of the group fails and the callers return CLES_EXCHANGE.

#include <cuda_runtime.h>

#include <chrono>
#include <condition_variable>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "cles_internal.h"

namespace {

struct Post {
    const void* a = nullptr;   // halo: send_lo; gather: the local block
    const void* b = nullptr;   // halo: send_hi
    cudaEvent_t ready = nullptr, copied = nullptr;
    double vals[8] = {0};
    int count = 0;
};

struct Endpoint {
    cles_local_group* g = nullptr;
    int rank = 0;
    int coords[3] = {0, 0, 0};
    cudaEvent_t ready = nullptr, copied = nullptr;   // created on the caller's device at first use
};

}  // namespace

struct cles_local_group {
    int dims[3] = {1, 1, 1};
    int n = 1;
    std::chrono::duration<double> timeout{60.0};
    std::mutex m;
    std::condition_variable cv;
    int arrived = 0;
    unsigned long long gen = 0;
    bool aborted = false;
    std::vector<Post> post;
    std::vector<Endpoint> eps;

    ~cles_local_group() {
        for (Endpoint& e : eps) {
            if (e.ready) cudaEventDestroy(e.ready);
            if (e.copied) cudaEventDestroy(e.copied);
        }
    }

    int linear(const int c[3]) const { return c[0] + dims[0] * (c[1] + dims[1] * c[2]); }

    void abort() {
        std::lock_guard<std::mutex> lk(m);
        aborted = true;
        cv.notify_all();
    }

    // true once every rank has arrived; false on abort or timeout (which
    // aborts the group, so no other rank waits out the limit again)
    bool barrier() {
        std::unique_lock<std::mutex> lk(m);
        if (aborted) return false;
        const unsigned long long my = gen;
        if (++arrived == n) {
            arrived = 0;
            ++gen;
            cv.notify_all();
            return true;
        }
        cv.wait_for(lk, timeout, [&] { return gen != my || aborted; });
        if (gen != my) return true;
        aborted = true;
        cv.notify_all();
        return false;
    }
};

namespace {

int fail(cles_local_group* g) {
    g->abort();
    return 1;
}

bool events(Endpoint* e) {
    if (!e->ready && cudaEventCreateWithFlags(&e->ready, cudaEventDisableTiming) != cudaSuccess) return false;
    if (!e->copied && cudaEventCreateWithFlags(&e->copied, cudaEventDisableTiming) != cudaSuccess) return false;
    return true;
}

// first half: publish `a`, `b` with a ready event recorded on st
bool publish(Endpoint* e, cudaStream_t st, const void* a, const void* b) {
    cles_local_group* g = e->g;
    if (!events(e) || cudaEventRecord(e->ready, st) != cudaSuccess) return false;
    Post& me = g->post[e->rank];
    me.a = a;
    me.b = b;
    me.ready = e->ready;
    return true;
}

// after the copies from `peers`: record and publish the copied event, meet
// everyone, then order st after the copies of the ranks that read from us
bool finish(Endpoint* e, cudaStream_t st, const std::vector<int>& readers) {
    cles_local_group* g = e->g;
    if (cudaEventRecord(e->copied, st) != cudaSuccess) return false;
    g->post[e->rank].copied = e->copied;
    if (!g->barrier()) return false;
    for (int r : readers)
        if (r != e->rank && cudaStreamWaitEvent(st, g->post[r].copied, 0) != cudaSuccess) return false;
    return true;
}

int lg_halo(void* user, int dim, int prev, int next, const void* send_lo, const void* send_hi, void* recv_lo,
            void* recv_hi, int64_t bytes, void* stream) {
    auto* e = static_cast<Endpoint*>(user);
    cles_local_group* g = e->g;
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (dim < 0 || dim > 2) return fail(g);
    if (!publish(e, st, send_lo, send_hi)) return fail(g);
    if (!g->barrier()) return 1;
    bool ok = true;
    int c[3] = {e->coords[0], e->coords[1], e->coords[2]};
    std::vector<int> readers;
    if (prev >= 0) {
        c[dim] = prev;
        const Post& p = g->post[g->linear(c)];
        readers.push_back(g->linear(c));
        ok = ok && (g->linear(c) == e->rank || cudaStreamWaitEvent(st, p.ready, 0) == cudaSuccess) &&
             cudaMemcpyAsync(recv_lo, p.b, (size_t)bytes, cudaMemcpyDefault, st) == cudaSuccess;
    }
    if (next >= 0) {
        c[dim] = next;
        const Post& p = g->post[g->linear(c)];
        readers.push_back(g->linear(c));
        ok = ok && (g->linear(c) == e->rank || cudaStreamWaitEvent(st, p.ready, 0) == cudaSuccess) &&
             cudaMemcpyAsync(recv_hi, p.a, (size_t)bytes, cudaMemcpyDefault, st) == cudaSuccess;
    }
    // the neighbours that read our sends are the same two ranks
    if (!ok || !finish(e, st, readers)) return fail(g);
    return 0;
}

int lg_gather(void* user, int dim, const void* local, void* all, int64_t bytes, void* stream) {
    auto* e = static_cast<Endpoint*>(user);
    cles_local_group* g = e->g;
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (dim < 0 || dim > 2) return fail(g);
    if (!publish(e, st, local, nullptr)) return fail(g);
    if (!g->barrier()) return 1;
    bool ok = true;
    int c[3] = {e->coords[0], e->coords[1], e->coords[2]};
    std::vector<int> line;
    for (int r = 0; r < g->dims[dim]; ++r) {
        c[dim] = r;
        const int src = g->linear(c);
        line.push_back(src);
        ok = ok && (src == e->rank || cudaStreamWaitEvent(st, g->post[src].ready, 0) == cudaSuccess) &&
             cudaMemcpyAsync(static_cast<char*>(all) + (size_t)r * (size_t)bytes, g->post[src].a, (size_t)bytes,
                             cudaMemcpyDefault, st) == cudaSuccess;
    }
    // every rank of the line reads our block
    if (!ok || !finish(e, st, line)) return fail(g);
    return 0;
}

// Julia's max (NaN wins), as the reductions of max_rate see it
double jl_max(double x, double y) {
    if (x != x) return x;
    if (y != y) return y;
    return y > x ? y : x;
}

int lg_allreduce(void* user, int op, double* vals, int count) {
    auto* e = static_cast<Endpoint*>(user);
    cles_local_group* g = e->g;
    if (count < 0 || count > 8 || (op != CLES_REDUCE_MAX && op != CLES_REDUCE_SUM)) return fail(g);
    Post& me = g->post[e->rank];
    for (int i = 0; i < count; ++i) me.vals[i] = vals[i];
    me.count = count;
    if (!g->barrier()) return 1;
    // every rank reduces in rank order, so all of them get the same bits
    for (int i = 0; i < count; ++i) {
        double acc = g->post[0].vals[i];
        for (int r = 1; r < g->n; ++r)
            acc = op == CLES_REDUCE_MAX ? jl_max(acc, g->post[r].vals[i]) : acc + g->post[r].vals[i];
        vals[i] = acc;
    }
    return g->barrier() ? 0 : 1;
}

}  // namespace

extern "C" {

int cles_local_group_create(const int dims[3], double timeout_s, cles_local_group** out) {
    if (!dims || !out) {
        cles::set_last_error("null argument");
        return CLES_EINVAL;
    }
    int n = 1;
    for (int k = 0; k < 3; ++k) {
        if (dims[k] < 1 || dims[k] > 4096) {
            cles::set_last_error("process grid dims must lie in [1, 4096]");
            return CLES_EINVAL;
        }
        n *= dims[k];
    }
    if (n > 4096 || !(timeout_s > 0)) {
        cles::set_last_error("at most 4096 ranks and a positive timeout");
        return CLES_EINVAL;
    }
    auto* g = new cles_local_group();
    for (int k = 0; k < 3; ++k) g->dims[k] = dims[k];
    g->n = n;
    g->timeout = std::chrono::duration<double>(timeout_s);
    g->post.resize((size_t)n);
    g->eps.resize((size_t)n);
    for (int r = 0; r < n; ++r) {
        Endpoint& e = g->eps[(size_t)r];
        e.g = g;
        e.rank = r;
        e.coords[0] = r % dims[0];
        e.coords[1] = (r / dims[0]) % dims[1];
        e.coords[2] = r / (dims[0] * dims[1]);
    }
    *out = g;
    return CLES_OK;
}

void cles_local_group_destroy(cles_local_group* g) { delete g; }

int cles_local_group_exchange(cles_local_group* g, const int coords[3], cles_exchange* out) {
    if (!g || !coords || !out) {
        cles::set_last_error("null argument");
        return CLES_EINVAL;
    }
    for (int k = 0; k < 3; ++k)
        if (coords[k] < 0 || coords[k] >= g->dims[k]) {
            cles::set_last_error("rank coordinates must lie in [0, dims)");
            return CLES_EINVAL;
        }
    std::memset(out, 0, sizeof(*out));
    out->user = &g->eps[(size_t)g->linear(coords)];
    out->halo = lg_halo;
    out->gather = lg_gather;
    out->allreduce = lg_allreduce;
    return CLES_OK;
}

void cles_local_group_abort(cles_local_group* g) {
    if (g) g->abort();
}

}  // extern "C"
