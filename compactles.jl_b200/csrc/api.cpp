// C ABI of libcles.so (include/cles.h).  Every entry point catches every
// exception, records its text for cles_last_error() and returns a status.

#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <vector>
#include <string>

#include "solver.h"

namespace cles {

namespace {
thread_local std::string g_last_error;
std::atomic<int64_t> g_launches{0};
}  // namespace

namespace {
struct ProfRec {
    int family;
    double bytes;
    cudaEvent_t a, b;
};
bool g_prof_on = false;
std::vector<ProfRec> g_prof;
std::vector<cudaEvent_t> g_event_pool;
size_t g_event_next = 0;
cudaEvent_t next_event() {
    if (g_event_next == g_event_pool.size()) {
        cudaEvent_t e;
        CLES_CUDA(cudaEventCreate(&e));
        g_event_pool.push_back(e);
    }
    return g_event_pool[g_event_next++];
}
}  // namespace

bool profiling() { return g_prof_on; }
int prof_begin(cudaStream_t st, int family, double bytes) {
    ProfRec r{family, bytes, next_event(), next_event()};
    CLES_CUDA(cudaEventRecord(r.a, st));
    g_prof.push_back(r);
    return (int)g_prof.size() - 1;
}
void prof_end(int rec, cudaStream_t st) { CLES_CUDA(cudaEventRecord(g_prof[rec].b, st)); }

void set_last_error(const std::string& s) { g_last_error = s; }
void count_launch(int n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
int64_t launch_count() { return g_launches.load(std::memory_order_relaxed); }
void check_launch(const char* what) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) throw Error(CLES_ECUDA, std::string(what) + " launch: " + cudaGetErrorString(e));
}

// ---------------------------------------------------------------- presets ----
// lele_d1_6 / pade_d1_4 / compact_filter (src/kernels.jl:61-111) and
// lele_d1_10 (src/kernels_banded.jl:54-64).
namespace {
void clear(cles_scheme* s, const char* name) {
    std::memset(s, 0, sizeof(*s));
    std::snprintf(s->name, sizeof(s->name), "%s", name);
}
void tri_row(cles_scheme* s, int j, double sub, double dia, double sup, std::initializer_list<double> rhs) {
    s->clo_lhs[j][0] = sub;
    s->clo_lhs[j][1] = dia;
    s->clo_lhs[j][2] = sup;
    int k = 0;
    for (double v : rhs) s->clo_rhs[j][k++] = v;
    s->clo_len[j] = k;
}
}  // namespace

}  // namespace cles

using namespace cles;

struct cles_plan {
    cles_ctx* ctx = nullptr;
    CompactPlan plan;
    int layout = CLES_LAYOUT_PADDED;
    int n[3]{}, pad[3]{};
    int64_t elem_off = 0, sy = 0, sz = 0, field_elems = 0;
    DevBuf fbuf, obuf;
};

struct cles_split_plan {
    cles_ctx* ctx = nullptr;
    SplitPlan sp;
    int64_t elem_off = 0, sy = 0, sz = 0, field_elems = 0;
    DevBuf zbuf;
};

struct cles_solver {
    cles_ctx* ctx = nullptr;
    std::unique_ptr<SolverBase> s;
};

#define API_BEGIN try {
#define API_END                                         \
    }                                                   \
    catch (const cles::Error& e) {                      \
        set_last_error(e.what());                       \
        return e.code;                                  \
    }                                                   \
    catch (const std::exception& e) {                   \
        set_last_error(e.what());                       \
        return CLES_EINVAL;                             \
    }                                                   \
    catch (...) {                                       \
        set_last_error("unknown error");                \
        return CLES_EINVAL;                             \
    }                                                   \
    set_last_error("");                                 \
    return CLES_OK;

extern "C" {

const char* cles_last_error(void) { return g_last_error.c_str(); }

int cles_profile_enable(int on) {
    API_BEGIN
    g_prof.clear();
    g_event_next = 0;
    g_prof_on = on != 0;
    API_END
}

int cles_profile_read(cles_profile_entry* out, int max_entries, int* n_entries) {
    API_BEGIN
    if (!out || !n_entries) throw Error(CLES_EINVAL, "null argument");
    static const char* names[3] = {"compact_x", "compact_y", "compact_z"};
    cles_profile_entry acc[3];
    std::memset(acc, 0, sizeof(acc));
    for (int k = 0; k < 3; ++k) std::snprintf(acc[k].name, sizeof(acc[k].name), "%s", names[k]);
    for (const ProfRec& r : g_prof) {
        CLES_CUDA(cudaEventSynchronize(r.b));
        float ms = 0.f;
        CLES_CUDA(cudaEventElapsedTime(&ms, r.a, r.b));
        acc[r.family].launches += 1;
        acc[r.family].total_ms += ms;
        acc[r.family].bytes += r.bytes;
    }
    int n = 0;
    for (int k = 0; k < 3 && n < max_entries; ++k)
        if (acc[k].launches) out[n++] = acc[k];
    *n_entries = n;
    API_END
}
int64_t cles_kernel_launches(void) { return g_launches.load(); }

int cles_scheme_lele_d1_6(cles_scheme* s) {
    if (!s) return CLES_EINVAL;
    clear(s, "Lele C6 first derivative");
    s->q = 1;
    s->lhs[0] = 1.0 / 3.0;
    s->M = 2;
    s->coeffs[0] = 7.0 / 9.0;
    s->coeffs[1] = 1.0 / 36.0;
    s->symmetric = 0;
    s->nc = 2;
    tri_row(s, 0, 0.0, 1.0, 2.0, {-5.0 / 2.0, 2.0, 1.0 / 2.0});
    tri_row(s, 1, 1.0 / 4.0, 1.0, 1.0 / 4.0, {-3.0 / 4.0, 0.0, 3.0 / 4.0});
    return CLES_OK;
}

int cles_scheme_pade_d1_4(cles_scheme* s) {
    if (!s) return CLES_EINVAL;
    clear(s, "Pade C4 first derivative");
    s->q = 1;
    s->lhs[0] = 1.0 / 4.0;
    s->M = 1;
    s->coeffs[0] = 3.0 / 4.0;
    s->nc = 1;
    tri_row(s, 0, 0.0, 1.0, 2.0, {-5.0 / 2.0, 2.0, 1.0 / 2.0});
    return CLES_OK;
}

int cles_scheme_compact_filter(double af, cles_scheme* s) {
    if (!s) return CLES_EINVAL;
    clear(s, "Gaitonde-Visbal C8 filter");
    s->q = 1;
    s->lhs[0] = af;
    s->a0 = (93 + 70 * af) / 128;
    s->M = 4;
    s->coeffs[0] = (7 + 18 * af) / 16 / 2;
    s->coeffs[1] = (-7 + 14 * af) / 32 / 2;
    s->coeffs[2] = (1 - 2 * af) / 16 / 2;
    s->coeffs[3] = (-1 + 2 * af) / 128 / 2;
    s->symmetric = 1;
    s->nc = 4;
    // row 1 unfiltered; rows 2-4 centred filters of order 2, 4, 6 with the same alpha_f
    const double f2[2] = {(1 + 2 * af) / 2, (1 + 2 * af) / 2};
    const double f4[3] = {(5 + 6 * af) / 8, (1 + 2 * af) / 2, (-1 + 2 * af) / 8};
    const double f6[4] = {(11 + 10 * af) / 16, (15 + 34 * af) / 32, (-3 + 6 * af) / 16, (1 - 2 * af) / 32};
    auto centred = [&](int j, const double* c, int len) {
        int k = 0;
        for (int m = len - 1; m >= 1; --m) s->clo_rhs[j][k++] = c[m] / 2;
        s->clo_rhs[j][k++] = c[0];
        for (int m = 1; m < len; ++m) s->clo_rhs[j][k++] = c[m] / 2;
        s->clo_len[j] = k;
    };
    s->clo_lhs[0][1] = 1.0;
    s->clo_rhs[0][0] = 1.0;
    s->clo_len[0] = 1;
    for (int j = 1; j < 4; ++j) {
        s->clo_lhs[j][0] = af;
        s->clo_lhs[j][1] = 1.0;
        s->clo_lhs[j][2] = af;
    }
    centred(1, f2, 2);
    centred(2, f4, 3);
    centred(3, f6, 4);
    return CLES_OK;
}

int cles_scheme_lele_d1_10(cles_scheme* s) {
    if (!s) return CLES_EINVAL;
    clear(s, "Lele C10 first derivative");
    s->q = 2;
    s->lhs[0] = 1.0 / 2.0;
    s->lhs[1] = 1.0 / 20.0;
    s->M = 3;
    s->coeffs[0] = 17.0 / 24.0;
    s->coeffs[1] = 101.0 / 600.0;
    s->coeffs[2] = 1.0 / 600.0;
    s->nc = 3;
    // rows 1-2: the C6 one-sided closures; row 3: the C6 interior row
    const double lhs[3][5] = {{0, 0, 1, 2, 0}, {0, 1.0 / 4.0, 1, 1.0 / 4.0, 0}, {0, 1.0 / 3.0, 1, 1.0 / 3.0, 0}};
    for (int j = 0; j < 3; ++j)
        for (int t = 0; t < 5; ++t) s->clo_lhs[j][t] = lhs[j][t];
    const double r0[3] = {-5.0 / 2.0, 2.0, 1.0 / 2.0}, r1[3] = {-3.0 / 4.0, 0.0, 3.0 / 4.0};
    const double r2[5] = {-1.0 / 36.0, -7.0 / 9.0, 0.0, 7.0 / 9.0, 1.0 / 36.0};
    for (int t = 0; t < 3; ++t) { s->clo_rhs[0][t] = r0[t]; s->clo_rhs[1][t] = r1[t]; }
    for (int t = 0; t < 5; ++t) s->clo_rhs[2][t] = r2[t];
    s->clo_len[0] = 3;
    s->clo_len[1] = 3;
    s->clo_len[2] = 5;
    return CLES_OK;
}

// ---------------------------------------------------------------- context ----
int cles_ctx_create(int device, void* stream, size_t budget, cles_ctx** out) {
    API_BEGIN
    if (!out) throw Error(CLES_EINVAL, "null output pointer");
    int count = 0;
    CLES_CUDA(cudaGetDeviceCount(&count));
    if (device < 0 || device >= count) throw Error(CLES_EINVAL, "no such CUDA device");
    CLES_CUDA(cudaSetDevice(device));
    cudaDeviceProp prop;
    CLES_CUDA(cudaGetDeviceProperties(&prop, device));
    if (prop.major < 10) throw Error(CLES_ECUDA, "this library is built for sm_100a (B200); device is sm_" +
                                                      std::to_string(prop.major) + std::to_string(prop.minor));
    auto* c = new cles_ctx();
    c->device = device;
    c->stream = reinterpret_cast<cudaStream_t>(stream);
    c->budget = budget;
    *out = c;
    API_END
}

void cles_ctx_destroy(cles_ctx* ctx) { ctx_release(ctx); }

int cles_ctx_set_stream(cles_ctx* ctx, void* stream) {
    API_BEGIN
    if (!ctx) throw Error(CLES_EINVAL, "null context");
    ctx->stream = reinterpret_cast<cudaStream_t>(stream);
    API_END
}

int cles_selftest_bounded_wait(cles_ctx* ctx, int64_t limit_ns) {
    API_BEGIN
    if (!ctx) throw Error(CLES_EINVAL, "null context");
    if (limit_ns < 1000 || limit_ns > 2000000000LL)
        throw Error(CLES_EINVAL, "limit_ns must lie in [1e3, 2e9]");
    CLES_CUDA(cudaSetDevice(ctx->device));
    launch_wait_selftest((uint64_t)limit_ns, ctx->stream);
    if (take_device_timeouts(ctx->stream))
        throw Error(CLES_ETIMEOUT, "a bounded device wait expired (self-test)");
    API_END
}

// ------------------------------------------------------------------ plans ----
int cles_plan_create(cles_ctx* ctx, const cles_grid* grid, const cles_scheme* scheme, int dim, double h, int dtype,
                     int layout, cles_plan** out) {
    API_BEGIN
    if (!ctx || !grid || !scheme || !out) throw Error(CLES_EINVAL, "null argument");
    if (dim < 1 || dim > 3) throw Error(CLES_EINVAL, "dim must be 1, 2 or 3");
    if (dtype != CLES_F64 && dtype != CLES_F32) throw Error(CLES_EINVAL, "dtype must be CLES_F64 or CLES_F32");
    if (layout != CLES_LAYOUT_PADDED && layout != CLES_LAYOUT_INTERIOR) throw Error(CLES_EINVAL, "unknown layout");
    if (!(h > 0)) throw Error(CLES_EINVAL, "grid spacing must be positive");
    for (int k = 0; k < 3; ++k)
        if (grid->n_global[k] < 1) throw Error(CLES_EINVAL, "n_global must be >= 1");
    if (grid->n_global[dim - 1] <= 1) throw Error(CLES_EINVAL, "dimension is collapsed");
    if (scheme->M > grid->n_halo && layout == CLES_LAYOUT_PADDED)
        throw Error(CLES_EINVAL, "stencil half-width " + std::to_string(scheme->M) + " exceeds halo width " +
                                     std::to_string(grid->n_halo));
    CLES_CUDA(cudaSetDevice(ctx->device));
    auto* p = new cles_plan();
    try {
        p->ctx = ctx;
        p->layout = layout;
        for (int k = 0; k < 3; ++k) {
            p->n[k] = grid->n_global[k];
            p->pad[k] = (layout == CLES_LAYOUT_PADDED && grid->n_global[k] > 1) ? grid->n_halo : 0;
        }
        const int d = dim - 1;
        const bool periodic = grid->periodic[d] != 0;
        build_compact_plan(p->plan, *scheme, p->n, d, periodic, h, dtype);
        const int64_t F0 = p->n[0] + 2 * p->pad[0], F1 = p->n[1] + 2 * p->pad[1], F2 = p->n[2] + 2 * p->pad[2];
        p->sy = F0;
        p->sz = F0 * F1;
        p->elem_off = p->pad[0] + p->pad[1] * F0 + p->pad[2] * F0 * F1;
        p->field_elems = F0 * F1 * F2;
    } catch (...) {
        delete p;
        throw;
    }
    ctx_retain(ctx);
    *out = p;
    API_END
}

void cles_plan_destroy(cles_plan* plan) {
    if (!plan) return;
    cles_ctx* c = plan->ctx;
    cudaSetDevice(c->device);
    delete plan;
    ctx_release(c);
}

static int apply_impl(cles_plan* plan, const void* f, void* out, int count, int64_t stride) {
    API_BEGIN
    if (!plan || !f || !out) throw Error(CLES_EINVAL, "null argument");
    if (count < 1) throw Error(CLES_EINVAL, "count must be >= 1");
    const size_t el = plan->plan.dtype == CLES_F64 ? sizeof(double) : sizeof(float);
    FieldView vin{const_cast<char*>(reinterpret_cast<const char*>(f)) + el * plan->elem_off, stride, plan->sy, plan->sz};
    FieldView vout{reinterpret_cast<char*>(out) + el * plan->elem_off, stride, plan->sy, plan->sz};
    launch_compact(plan->plan, vin, vout, count, OUT_STORE, plan->ctx->stream);
    API_END
}

int cles_apply_along(cles_plan* plan, const void* f_dev, void* out_dev) {
    if (!plan) return CLES_EINVAL;
    return apply_impl(plan, f_dev, out_dev, 1, plan->field_elems);
}

int cles_apply_along_batch(cles_plan* plan, const void* f_dev, void* out_dev, int count, int64_t field_stride) {
    return apply_impl(plan, f_dev, out_dev, count, field_stride);
}

int cles_apply_along_host(cles_plan* plan, const void* f_host, void* out_host) {
    API_BEGIN
    if (!plan || !f_host || !out_host) throw Error(CLES_EINVAL, "null argument");
    CLES_CUDA(cudaSetDevice(plan->ctx->device));
    const size_t el = plan->plan.dtype == CLES_F64 ? sizeof(double) : sizeof(float);
    const size_t bytes = el * (size_t)plan->field_elems;
    if (!plan->fbuf.p) {
        plan->fbuf.alloc(plan->ctx, bytes);
        plan->obuf.alloc(plan->ctx, bytes);
    }
    cudaStream_t st = plan->ctx->stream;
    CLES_CUDA(cudaMemcpyAsync(plan->fbuf.p, f_host, bytes, cudaMemcpyHostToDevice, st));
    CLES_CUDA(cudaMemcpyAsync(plan->obuf.p, out_host, bytes, cudaMemcpyHostToDevice, st));
    int rc = apply_impl(plan, plan->fbuf.p, plan->obuf.p, 1, plan->field_elems);
    if (rc != CLES_OK) return rc;
    CLES_CUDA(cudaMemcpyAsync(out_host, plan->obuf.p, bytes, cudaMemcpyDeviceToHost, st));
    CLES_CUDA(cudaStreamSynchronize(st));
    API_END
}

// ------------------------------------------------------------ split lines ----
int cles_split_plan_create(cles_ctx* ctx, const cles_split_desc* d, const cles_scheme* scheme, double h, int dtype,
                           cles_split_plan** out) {
    API_BEGIN
    if (!ctx || !d || !scheme || !out) throw Error(CLES_EINVAL, "null argument");
    if (d->dim < 1 || d->dim > 3) throw Error(CLES_EINVAL, "dim must be 1, 2 or 3");
    if (dtype != CLES_F64 && dtype != CLES_F32) throw Error(CLES_EINVAL, "dtype must be CLES_F64 or CLES_F32");
    if (!(h > 0)) throw Error(CLES_EINVAL, "grid spacing must be positive");
    for (int k = 0; k < 3; ++k)
        if (d->n_local[k] < 1) throw Error(CLES_EINVAL, "n_local must be >= 1");
    if (d->n_local[d->dim - 1] <= 1 || d->n_global <= 1) throw Error(CLES_EINVAL, "dimension is collapsed");
    if (scheme->M > d->n_halo)
        throw Error(CLES_EINVAL, "stencil half-width " + std::to_string(scheme->M) + " exceeds halo width " +
                                     std::to_string(d->n_halo));
    CLES_CUDA(cudaSetDevice(ctx->device));
    auto* p = new cles_split_plan();
    try {
        p->ctx = ctx;
        build_split_plan(p->sp, *scheme, d->n_local, d->dim - 1, d->periodic != 0, d->n_global, d->ranks, d->rank, h,
                         dtype);
        int pad[3];
        for (int k = 0; k < 3; ++k) pad[k] = d->n_local[k] > 1 ? d->n_halo : 0;
        const int64_t F0 = d->n_local[0] + 2 * pad[0], F1 = d->n_local[1] + 2 * pad[1],
                      F2 = d->n_local[2] + 2 * pad[2];
        p->sy = F0;
        p->sz = F0 * F1;
        p->elem_off = pad[0] + pad[1] * F0 + pad[2] * F0 * F1;
        p->field_elems = F0 * F1 * F2;
    } catch (...) {
        delete p;
        throw;
    }
    ctx_retain(ctx);
    *out = p;
    API_END
}

void cles_split_plan_destroy(cles_split_plan* plan) {
    if (!plan) return;
    cles_ctx* c = plan->ctx;
    cudaSetDevice(c->device);
    delete plan;
    ctx_release(c);
}

int cles_split_plan_info(const cles_split_plan* plan, cles_split_info* out) {
    API_BEGIN
    if (!plan || !out) throw Error(CLES_EINVAL, "null argument");
    const SplitPlan& sp = plan->sp;
    out->halo_elems = (int64_t)sp.M * sp.lines;
    out->iface_elems = (int64_t)2 * sp.q * sp.lines;
    out->field_elems = plan->field_elems;
    out->prev = sp.prev;
    out->next = sp.next;
    out->ranks = sp.ranks;
    out->q = sp.q;
    out->M = sp.M;
    API_END
}

static FieldView split_view(const cles_split_plan* p, const void* f, int64_t stride) {
    const size_t el = p->sp.dtype == CLES_F64 ? sizeof(double) : sizeof(float);
    return FieldView{const_cast<char*>(reinterpret_cast<const char*>(f)) + el * p->elem_off, stride, p->sy, p->sz};
}

static void split_check(const cles_split_plan* p, const void* f, int count, int64_t stride) {
    if (!p || !f) throw Error(CLES_EINVAL, "null argument");
    if (count < 1) throw Error(CLES_EINVAL, "count must be >= 1");
    if (count > 1 && stride < p->field_elems) throw Error(CLES_EINVAL, "field_stride below the padded field size");
}

int cles_split_halo_pack(cles_split_plan* plan, const void* f_dev, void* send_lo, void* send_hi, int count,
                         int64_t field_stride) {
    API_BEGIN
    split_check(plan, f_dev, count, field_stride);
    if ((plan->sp.lo_open && !send_lo) || (plan->sp.hi_open && !send_hi))
        throw Error(CLES_EINVAL, "missing send buffer for an end with a neighbour");
    CLES_CUDA(cudaSetDevice(plan->ctx->device));
    split_halo(plan->sp, split_view(plan, f_dev, field_stride), send_lo, send_hi, count, true, plan->ctx->stream);
    API_END
}

int cles_split_halo_unpack(cles_split_plan* plan, const void* recv_lo, const void* recv_hi, void* f_dev, int count,
                           int64_t field_stride) {
    API_BEGIN
    split_check(plan, f_dev, count, field_stride);
    if ((plan->sp.lo_open && !recv_lo) || (plan->sp.hi_open && !recv_hi))
        throw Error(CLES_EINVAL, "missing receive buffer for an end with a neighbour");
    CLES_CUDA(cudaSetDevice(plan->ctx->device));
    split_halo(plan->sp, split_view(plan, f_dev, field_stride), const_cast<void*>(recv_lo),
               const_cast<void*>(recv_hi), count, false, plan->ctx->stream);
    API_END
}

int cles_split_apply_begin(cles_split_plan* plan, const void* f_dev, void* out_dev, void* iface, int count,
                           int64_t field_stride) {
    API_BEGIN
    split_check(plan, f_dev, count, field_stride);
    if (!out_dev || !iface) throw Error(CLES_EINVAL, "null argument");
    CLES_CUDA(cudaSetDevice(plan->ctx->device));
    launch_compact_split(plan->sp.local, split_view(plan, f_dev, field_stride), split_view(plan, out_dev, field_stride),
                         count, iface, plan->ctx->stream);
    API_END
}

int cles_split_apply_end(cles_split_plan* plan, const void* iface_all, void* out_dev, int count,
                         int64_t field_stride) {
    API_BEGIN
    split_check(plan, out_dev, count, field_stride);
    if (!iface_all) throw Error(CLES_EINVAL, "null argument");
    CLES_CUDA(cudaSetDevice(plan->ctx->device));
    const size_t el = plan->sp.dtype == CLES_F64 ? sizeof(double) : sizeof(float);
    const size_t zb = el * (size_t)count * 2 * plan->sp.q * plan->sp.lines;
    if (plan->zbuf.bytes < zb) {
        CLES_CUDA(cudaStreamSynchronize(plan->ctx->stream));   // a smaller buffer may still be in use
        plan->zbuf.release();
        plan->zbuf.alloc(plan->ctx, zb);
    }
    split_correct(plan->sp, iface_all, plan->zbuf.p, split_view(plan, out_dev, field_stride), count,
                  plan->ctx->stream);
    API_END
}

// ----------------------------------------------------------------- solver ----
void cles_step_control_default(cles_step_control* c) {
    if (!c) return;
    c->predict = 0.0;
    c->max_growth = 0.0;
    c->landing_steps = 2;
    c->dt_min = 0.0;
    c->dt_min_ratio = 1e-8;
    c->retries = 0;
    c->cfl_backoff = 0.5;
    c->savepoint_interval = 25;
}

void cles_solver_desc_default(cles_solver_desc* d) {
    if (!d) return;
    std::memset(d, 0, sizeof(*d));
    for (int k = 0; k < 3; ++k) {
        d->n_global[k] = 1;
        d->L[k] = 1.0;
        d->bc[k][0] = d->bc[k][1] = CLES_BC_PERIODIC;
    }
    d->n_species = 1;
    d->R[0] = 1.0;
    d->gamma[0] = 1.4;
    d->mu0 = 0.0;
    d->Pr = 0.7;
    d->Sc = 0.7;
    d->art_enabled = 1;
    d->C_mu = 0.002;
    d->C_beta = 1.0;
    d->C_kappa = 0.01;
    d->C_D = 0.01;
    d->beta_sensor = CLES_BETA_STRAIN;
    cles_scheme_lele_d1_6(&d->deriv);
    cles_scheme_compact_filter(0.45, &d->filt);
    d->cfl = 0.5;
    d->filter_interval = 1;
    cles_step_control_default(&d->control);
    d->n_halo = 4;
    d->precision = CLES_PREC_FP64;
    d->eos = CLES_EOS_IDEAL;
    d->T_guess = 300.0;
}

int cles_solver_create(cles_ctx* ctx, const cles_solver_desc* desc, cles_solver** out) {
    API_BEGIN
    if (!ctx || !desc || !out) throw Error(CLES_EINVAL, "null argument");
    CLES_CUDA(cudaSetDevice(ctx->device));
    auto* s = new cles_solver();
    s->ctx = ctx;
    try {
        s->s = make_solver(ctx, *desc);
    } catch (...) {
        delete s;
        throw;
    }
    ctx_retain(ctx);
    *out = s;
    API_END
}

int cles_solver_create_decomposed(cles_ctx* ctx, const cles_solver_desc* desc, const cles_decomp* decomp,
                                  const cles_exchange* ex, cles_solver** out) {
    API_BEGIN
    if (!ctx || !desc || !decomp || !ex || !out) throw Error(CLES_EINVAL, "null argument");
    CLES_CUDA(cudaSetDevice(ctx->device));
    auto* s = new cles_solver();
    s->ctx = ctx;
    try {
        s->s = make_solver(ctx, *desc, decomp, ex);
    } catch (...) {
        delete s;
        throw;
    }
    ctx_retain(ctx);
    *out = s;
    API_END
}

void cles_solver_destroy(cles_solver* s) {
    if (!s) return;
    cles_ctx* c = s->ctx;
    cudaSetDevice(c->device);
    delete s;
    ctx_release(c);
}

#define SOLVER_CALL(body)                                        \
    API_BEGIN                                                    \
    if (!s) throw Error(CLES_EINVAL, "null solver");             \
    CLES_CUDA(cudaSetDevice(s->ctx->device));                    \
    body;                                                        \
    API_END

int cles_solver_info_get(const cles_solver* s, cles_solver_info* out) {
    API_BEGIN
    if (!s || !out) throw Error(CLES_EINVAL, "null argument");
    *out = s->s->info();
    API_END
}

int cles_set_state(cles_solver* s, const double* Q, int layout) { SOLVER_CALL(s->s->set_state(Q, layout)) }
int cles_get_state(cles_solver* s, double* Q, int layout) { SOLVER_CALL(s->s->get_state(Q, layout)) }
int cles_state_device(cles_solver* s, double** Q) { SOLVER_CALL(*Q = s->s->state_device()) }
int cles_apply_bcs(cles_solver* s) { SOLVER_CALL(s->s->apply_bcs()) }
int cles_max_rate(cles_solver* s, double* rate, double* rho_min) { SOLVER_CALL(s->s->max_rate(rate, rho_min)) }
int cles_compute_rhs(cles_solver* s, int primitives_current) { SOLVER_CALL(s->s->compute_rhs(primitives_current != 0)) }
int cles_get_rhs(cles_solver* s, double* dQ, int layout) { SOLVER_CALL(s->s->get_rhs(dQ, layout)) }
int cles_step(cles_solver* s, double dt, int prepared) { SOLVER_CALL(s->s->step(dt, prepared != 0)) }
int cles_filter_state(cles_solver* s) { SOLVER_CALL(s->s->filter_state()) }
int cles_get_field(cles_solver* s, int which, double* host, int layout) { SOLVER_CALL(s->s->get_field(which, host, layout)) }
int cles_kinetic_energy(cles_solver* s, double* ke) { SOLVER_CALL(*ke = s->s->kinetic_energy()) }
int cles_dissipation_rate(cles_solver* s, double* eps) { SOLVER_CALL(*eps = s->s->dissipation_rate()) }

int cles_get_clock(const cles_solver* s, double* t, int64_t* step, double* cfl) {
    API_BEGIN
    if (!s) throw Error(CLES_EINVAL, "null solver");
    if (t) *t = s->s->t;
    if (step) *step = s->s->step_count;
    if (cfl) *cfl = s->s->cfl;
    API_END
}

int cles_set_clock(cles_solver* s, double t, int64_t step, double cfl) {
    API_BEGIN
    if (!s) throw Error(CLES_EINVAL, "null solver");
    s->s->t = t;
    s->s->step_count = step;
    s->s->cfl = cfl;
    API_END
}

int cles_solver_switch_bc(cles_solver* s, int dim, int side) { SOLVER_CALL(s->s->switch_bc(dim, side)) }

int cles_solver_set_face_fn(cles_solver* s, int dim, int side, int which, cles_face_fn fn, void* user) {
    SOLVER_CALL(s->s->set_face_fn(dim, side, which, fn, user))
}

int cles_solver_bc_switched(const cles_solver* s, int dim, int side, int* switched) {
    API_BEGIN
    if (!s || !switched) throw Error(CLES_EINVAL, "null argument");
    *switched = s->s->bc_switched(dim, side) ? 1 : 0;
    API_END
}

// ------------------------------------------------------------ checkpoints --
namespace {
constexpr uint64_t kCkptMagic = 0x434c4553434b5054ull;   // "CLES CKPT" (src/io.jl:6)

// _ckpt_name (src/io.jl:8-9): prefix.rNNNN.ckpt with the communicator rank
std::string ckpt_name(const char* prefix, int rank) {
    char num[16];
    std::snprintf(num, sizeof(num), "%04d", rank);
    return std::string(prefix) + ".r" + num + ".ckpt";
}
int ckpt_rank(const cles_solver* s) {
    const cles_decomp* dc = s->s->decomposition();
    return dc ? dc->rank : 0;
}

struct FileCloser {
    FILE* f;
    ~FileCloser() { if (f) std::fclose(f); }
};
}  // namespace

int cles_checkpoint_save(cles_solver* s, const char* prefix) {
    API_BEGIN
    if (!s || !prefix) throw Error(CLES_EINVAL, "null argument");
    CLES_CUDA(cudaSetDevice(s->ctx->device));
    const cles_solver_info I = s->s->info();
    const size_t n = (size_t)I.cells * I.n_cons;
    std::vector<double> buf(n);
    s->s->get_state(buf.data(), CLES_LAYOUT_INTERIOR);
    const std::string path = ckpt_name(prefix, ckpt_rank(s));
    FileCloser fc{std::fopen(path.c_str(), "wb")};
    if (!fc.f) throw Error(CLES_EINVAL, "cannot open " + path + " for writing");
    int64_t hdr[10];
    hdr[0] = I.n_cons;
    const cles_decomp* dc = s->s->decomposition();
    for (int d = 0; d < 3; ++d) {
        hdr[1 + d] = s->s->desc.n_global[d];
        hdr[4 + d] = I.n_local[d];              // this rank's block
        hdr[7 + d] = dc ? dc->coords[d] : 0;    // its coordinates in the process grid
    }
    const double t = s->s->t;
    const int64_t step = s->s->step_count;
    bool ok = std::fwrite(&kCkptMagic, sizeof(kCkptMagic), 1, fc.f) == 1 &&
              std::fwrite(hdr, sizeof(int64_t), 10, fc.f) == 10 && std::fwrite(&t, sizeof(t), 1, fc.f) == 1 &&
              std::fwrite(&step, sizeof(step), 1, fc.f) == 1 && std::fwrite(buf.data(), sizeof(double), n, fc.f) == n;
    if (!ok) throw Error(CLES_EINVAL, "short write to " + path);
    API_END
}

int cles_checkpoint_load(cles_solver* s, const char* prefix) {
    API_BEGIN
    if (!s || !prefix) throw Error(CLES_EINVAL, "null argument");
    CLES_CUDA(cudaSetDevice(s->ctx->device));
    const cles_solver_info I = s->s->info();
    const std::string path = ckpt_name(prefix, ckpt_rank(s));
    FileCloser fc{std::fopen(path.c_str(), "rb")};
    if (!fc.f) throw Error(CLES_EINVAL, "cannot open " + path);
    uint64_t magic = 0;
    int64_t hdr[10];
    if (std::fread(&magic, sizeof(magic), 1, fc.f) != 1 || magic != kCkptMagic)
        throw Error(CLES_EINVAL, "not a CompactLES checkpoint");
    if (std::fread(hdr, sizeof(int64_t), 10, fc.f) != 10) throw Error(CLES_EINVAL, "truncated checkpoint header");
    if (hdr[0] != I.n_cons) throw Error(CLES_EINVAL, "conserved layout mismatch");
    for (int d = 0; d < 3; ++d)
        if (hdr[1 + d] != s->s->desc.n_global[d]) throw Error(CLES_EINVAL, "global grid mismatch");
    const cles_decomp* dc = s->s->decomposition();
    for (int d = 0; d < 3; ++d)
        if (hdr[4 + d] != I.n_local[d]) throw Error(CLES_EINVAL, "decomposition mismatch");
    for (int d = 0; d < 3; ++d)
        if (hdr[7 + d] != (dc ? dc->coords[d] : 0)) throw Error(CLES_EINVAL, "rank layout mismatch");
    double t = 0.0;
    int64_t step = 0;
    const size_t n = (size_t)I.cells * I.n_cons;
    std::vector<double> buf(n);
    if (std::fread(&t, sizeof(t), 1, fc.f) != 1 || std::fread(&step, sizeof(step), 1, fc.f) != 1 ||
        std::fread(buf.data(), sizeof(double), n, fc.f) != n)
        throw Error(CLES_EINVAL, "truncated checkpoint");
    s->s->set_state(buf.data(), CLES_LAYOUT_INTERIOR);
    s->s->t = t;
    s->s->step_count = step;
    API_END
}

int cles_check_step(const cles_step_control* c, double dt, double rho_min, double dt_seen, int64_t step, double t,
                    double cfl, int* reason) {
    API_BEGIN
    (void)step; (void)t; (void)cfl;
    if (!c || !reason) throw Error(CLES_EINVAL, "null argument");
    *reason = check_step(*c, dt, rho_min, dt_seen);
    API_END
}

int cles_run(cles_solver* s, double tfinal, int64_t nmax, cles_run_result* out) {
    int rc = CLES_OK;
    API_BEGIN
    if (!s) throw Error(CLES_EINVAL, "null solver");
    CLES_CUDA(cudaSetDevice(s->ctx->device));
    rc = s->s->run(tfinal, nmax, out);
    if (rc == CLES_EFAILURE) {
        set_last_error("SolverFailure: step control rejected the step (see cles_run_result.failure)");
        return rc;
    }
    API_END
}

int cles_run_graph(cles_solver* s, double tfinal, int64_t nmax, cles_run_result* out) {
    int rc = CLES_OK;
    API_BEGIN
    if (!s) throw Error(CLES_EINVAL, "null solver");
    CLES_CUDA(cudaSetDevice(s->ctx->device));
    rc = run_graph(*s->s, tfinal, nmax, out);
    if (rc == CLES_EFAILURE) {
        set_last_error("SolverFailure: step control rejected the step (see cles_run_result.failure)");
        return rc;
    }
    API_END
}

int cles_step_host(cles_solver* s, double* Q_host, int layout, double tfinal, cles_run_result* out) {
    int rc = CLES_OK;
    API_BEGIN
    if (!s || !Q_host) throw Error(CLES_EINVAL, "null argument");
    CLES_CUDA(cudaSetDevice(s->ctx->device));
    s->s->set_state(Q_host, layout);
    rc = s->s->run(tfinal, s->s->step_count + 1, out);
    s->s->get_state(Q_host, layout);
    if (rc == CLES_EFAILURE) {
        set_last_error("SolverFailure: step control rejected the step (see cles_run_result.failure)");
        return rc;
    }
    API_END
}

}  // extern "C"

// ---------------------------------------------------------------- batches ----
struct cles_batch {
    cles_ctx* ctx = nullptr;
    std::unique_ptr<BatchBase> b;
    std::vector<std::pair<int64_t, int>> layouts;   // member id -> layout it was added with
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
    double now() const {
        return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
    int layout_of(int64_t id) const {
        for (auto& e : layouts)
            if (e.first == id) return e.second;
        throw Error(CLES_EINVAL, "no batch member with this id");
    }
};

int cles_batch_create(cles_ctx* ctx, const cles_solver_desc* cls, cles_batch** out) {
    API_BEGIN
    if (!ctx || !cls || !out) throw Error(CLES_EINVAL, "null argument");
    CLES_CUDA(cudaSetDevice(ctx->device));
    auto* b = new cles_batch();
    try {
        b->ctx = ctx;
        b->b = make_batch(ctx, *cls);
    } catch (...) {
        delete b;
        throw;
    }
    ctx_retain(ctx);
    *out = b;
    API_END
}

void cles_batch_destroy(cles_batch* b) {
    if (!b) return;
    cles_ctx* c = b->ctx;
    cudaSetDevice(c->device);
    delete b;
    ctx_release(c);
}

int cles_batch_add(cles_batch* b, const cles_solver_desc* desc, const double* Q0, int layout, double tfinal,
                   int64_t nmax, int64_t* id) {
    API_BEGIN
    if (!b || !desc || !Q0 || !id) throw Error(CLES_EINVAL, "null argument");
    CLES_CUDA(cudaSetDevice(b->ctx->device));
    *id = b->b->add(*desc, Q0, layout, tfinal, nmax, b->now());
    b->layouts.emplace_back(*id, layout);
    API_END
}

int cles_batch_step(cles_batch* b, int* n_active) {
    API_BEGIN
    if (!b) throw Error(CLES_EINVAL, "null batch");
    CLES_CUDA(cudaSetDevice(b->ctx->device));
    const int n = b->b->step(b->now());
    if (n_active) *n_active = n;
    API_END
}

int cles_batch_run(cles_batch* b, int64_t max_steps, int* n_active) {
    API_BEGIN
    if (!b) throw Error(CLES_EINVAL, "null batch");
    CLES_CUDA(cudaSetDevice(b->ctx->device));
    int n = b->b->n_active();
    for (int64_t s = 0; s < max_steps && n > 0; ++s) n = b->b->step(b->now());
    if (n == 0) b->b->step(b->now());   // retires the last members (nothing left to step)
    if (n_active) *n_active = n;
    API_END
}

int cles_batch_status(cles_batch* b, int64_t id, cles_request_status* out) {
    API_BEGIN
    if (!b || !out) throw Error(CLES_EINVAL, "null argument");
    b->b->status(id, out);
    API_END
}

int cles_batch_fetch(cles_batch* b, int64_t id, double* Q) {
    API_BEGIN
    if (!b || !Q) throw Error(CLES_EINVAL, "null argument");
    CLES_CUDA(cudaSetDevice(b->ctx->device));
    b->b->fetch(id, Q, b->layout_of(id));
    API_END
}

int cles_batch_cancel(cles_batch* b, int64_t id) {
    API_BEGIN
    if (!b) throw Error(CLES_EINVAL, "null batch");
    b->b->remove(id, b->now());
    API_END
}

int cles_batch_stats_get(const cles_batch* b, cles_batch_stats* out) {
    API_BEGIN
    if (!b || !out) throw Error(CLES_EINVAL, "null argument");
    b->b->stats(out);
    API_END
}

int cles_batch_set_strategy(cles_batch* b, int strategy) {
    API_BEGIN
    if (!b) throw Error(CLES_EINVAL, "null batch");
    b->b->set_strategy(strategy);
    API_END
}
