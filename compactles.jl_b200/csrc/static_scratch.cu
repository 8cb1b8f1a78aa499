// cles_max_rate_static: the CFL rate / minimum-density reduction of max_rate
// for callers that cannot allocate device memory.
//
// Some callers of this library cannot call cudaMalloc: code running inside a
// host framework that owns every device allocation (a Julia/MPI application
// with its own memory pool, a plugin whose host forbids allocation after
// start-up, a process running under a fixed HBM budget), or code that must
// not allocate between CUDA-graph captures.  For them this entry point keeps
// its only scratch -- one (rate, min density) pair per thread block -- in a
// file-scope __device__ array that exists from the moment the library is
// loaded on a device until the process exits, so a call never allocates.
//
// Limits and sharing:
//   * the array holds kStaticPartials partials of kCellsPerBlock cells each,
//     so a call accepts at most CLES_STATIC_MAX_CELLS = 16384 * 2048 =
//     33,554,432 cells (e.g. a 256^3 or 320^3 box) and rejects larger grids
//     with CLES_EINVAL before launching anything;
//   * every call on a device shares the one array.  Each call writes every
//     partial it later reads, so nothing has to start at zero, but two calls
//     whose kernels overlap on the GPU (different streams, no ordering between
//     them) race on the array and may return each other's partials.  Order such
//     calls on one stream or synchronise between them;
//   * the first call on a device looks up the array's device address with
//     cudaGetSymbolAddress (once per device context, with that device
//     current).  Make that first call before any stream capture.  The address
//     is cached together with the context's unique id (cuCtxGetId): after a
//     cudaDeviceReset the module is loaded into a new context, the ids differ
//     and the next call looks the address up again instead of using a stale
//     one (that call is again a set-up call, outside any capture);
//   * `stream` must belong to the current device (checked with
//     cudaStreamGetDevice; a stream of another device is CLES_EINVAL).
// Scope: an ideal mixture (R and gamma per species) on a uniform Cartesian
// grid, one 1/h per dimension.  The per-cell arithmetic is the one of
// cles_max_rate for such a solver in FP64 (the primitives of
// src/physics.jl:604-653 and the rate of src/timestep.jl:125-175), so the
// two return identical values there.  It has no per-node 1/h (stretched or
// curvilinear grids), no curvature_rate term (src/timestep.jl:150-161) and
// no NASA-9 thermodynamics, and it reads FP64 primitives where a mixed-
// precision solver rounds them to FP32: on those solvers use cles_max_rate.

#include <cuda.h>

#include <mutex>

#include "cles_internal.h"

namespace cles {
namespace {

constexpr int kStaticThreads = 256;
constexpr int kCellsPerThread = 8;
constexpr int64_t kCellsPerBlock = (int64_t)kStaticThreads * kCellsPerThread;
constexpr int kStaticPartials = 16384;
static_assert(kCellsPerBlock * kStaticPartials == CLES_STATIC_MAX_CELLS, "limit in cles.h");

// The scratch: (rate, rho_min) per block, 16384 * 2 doubles = 256 KiB per device.
static __device__ __align__(256) double g_rate_scratch[2 * kStaticPartials];

struct StaticRateArgs {
    double Rk[CLES_MAX_SPECIES];
    double cvk[CLES_MAX_SPECIES];
    double inv_h[3];
    double mu0, Pr, Sc;
};

__device__ __forceinline__ double smax(double x, double y) {
    if (x != x) return x;
    if (y != y) return y;
    return y > x ? y : x;
}
__device__ __forceinline__ double smin(double x, double y) {
    if (x != x) return x;
    if (y != y) return y;
    return y < x ? y : x;
}

__global__ void __launch_bounds__(kStaticThreads)
k_rate_static_partial(const double* __restrict__ Q, const double* __restrict__ art, int64_t cells, int Ns,
                      StaticRateArgs a, double* __restrict__ scratch) {
    double rate = 0.0, rmin = __longlong_as_double(0x7ff0000000000000LL);
    const int64_t b0 = (int64_t)blockIdx.x * kCellsPerBlock;
    for (int t = 0; t < kCellsPerThread; ++t) {
        const int64_t I = b0 + (int64_t)t * kStaticThreads + threadIdx.x;
        if (I >= cells) break;
        double rq = 0.0;
        for (int sp = 0; sp < Ns; ++sp) rq += Q[I + cells * sp];
        rmin = smin(rmin, rq);
        // primitives (placeholders where rho <= 0, as the reference)
        double r, u, v, w, c, cp;
        if (rq > 0) {
            const double ri = 1 / rq;
            double Rm = 0.0, cvm = 0.0;
            for (int sp = 0; sp < Ns; ++sp) {
                const double q = Q[I + cells * sp];
                Rm += q * a.Rk[sp];
                cvm += q * a.cvk[sp];
            }
            Rm *= ri;
            cvm *= ri;
            u = Q[I + cells * (Ns + 0)] * ri;
            v = Q[I + cells * (Ns + 1)] * ri;
            w = Q[I + cells * (Ns + 2)] * ri;
            const double e = Q[I + cells * (Ns + 3)] * ri - 0.5 * (u * u + v * v + w * w);
            const double T = smax(e / cvm, 1e-300);
            const double gm = 1 + Rm / cvm;
            r = rq;
            c = sqrt(gm * Rm * T);
            cp = cvm + Rm;
        } else {
            r = 1; u = 0; v = 0; w = 0; c = 1; cp = 1;
        }
        const double ri = 1 / r;
        const double uv[3] = {u, v, w};
        double acc = 0.0, dsum = 0.0;
        for (int d = 0; d < 3; ++d) {
            if (a.inv_h[d] == 0.0) continue;  // collapsed dimension
            acc += (fabs(uv[d]) + c) * a.inv_h[d];
            dsum += a.inv_h[d] * a.inv_h[d];
        }
        double Dmax = a.mu0 / (a.Sc * r);
        for (int sp = 0; sp < Ns; ++sp) Dmax = smax(Dmax, a.mu0 / (a.Sc * r) + art[I + cells * (3 + sp)]);
        const double nu = (a.mu0 + art[I] + art[I + cells]) * ri + (a.mu0 * cp / a.Pr + art[I + 2 * cells]) * ri / cp + Dmax;
        acc += 2 * nu * dsum;
        rate = smax(rate, acc);
    }
    __shared__ double sr[kStaticThreads], sm[kStaticThreads];
    sr[threadIdx.x] = rate;
    sm[threadIdx.x] = rmin;
    __syncthreads();
    for (int s = kStaticThreads / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) {
            sr[threadIdx.x] = smax(sr[threadIdx.x], sr[threadIdx.x + s]);
            sm[threadIdx.x] = smin(sm[threadIdx.x], sm[threadIdx.x + s]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        scratch[2 * blockIdx.x] = sr[0];
        scratch[2 * blockIdx.x + 1] = sm[0];
    }
}

__global__ void __launch_bounds__(kStaticThreads)
k_rate_static_final(const double* __restrict__ scratch, int nb, double* __restrict__ out) {
    __shared__ double sr[kStaticThreads], sm[kStaticThreads];
    double rate = 0.0, rmin = __longlong_as_double(0x7ff0000000000000LL);
    for (int b = threadIdx.x; b < nb; b += kStaticThreads) {
        rate = smax(rate, scratch[2 * b]);
        rmin = smin(rmin, scratch[2 * b + 1]);
    }
    sr[threadIdx.x] = rate;
    sm[threadIdx.x] = rmin;
    __syncthreads();
    for (int s = kStaticThreads / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) {
            sr[threadIdx.x] = smax(sr[threadIdx.x], sr[threadIdx.x + s]);
            sm[threadIdx.x] = smin(sm[threadIdx.x], sm[threadIdx.x + s]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out[0] = sr[0];
        out[1] = sm[0];
    }
}

// Device address of g_rate_scratch, looked up once per device context.
constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
double* g_scratch_ptr[kMaxDevices] = {};
unsigned long long g_scratch_ctx[kMaxDevices] = {};

using CtxGetCurrentFn = CUresult (*)(CUcontext*);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);

// Unique id of the current device context (cuCtxGetId, through the runtime's
// driver entry points so the library needs no libcuda link).
unsigned long long current_context_id() {
    static CtxGetCurrentFn get_cur = nullptr;
    static CtxGetIdFn get_id = nullptr;
    if (!get_cur || !get_id) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            throw Error(CLES_ECUDA, "cuCtxGetCurrent is unavailable");
        get_cur = reinterpret_cast<CtxGetCurrentFn>(p);
        if (cudaGetDriverEntryPoint("cuCtxGetId", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            throw Error(CLES_ECUDA, "cuCtxGetId is unavailable");
        get_id = reinterpret_cast<CtxGetIdFn>(p);
    }
    CUcontext c = nullptr;
    unsigned long long id = 0;
    if (get_cur(&c) != CUDA_SUCCESS || !c || get_id(c, &id) != CUDA_SUCCESS)
        throw Error(CLES_ECUDA, "no current CUDA context");
    return id;
}

double* scratch_for_current_device() {
    int dev = 0;
    CLES_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) throw Error(CLES_EINVAL, "device index out of range");
    CLES_CUDA(cudaSetDevice(dev));   // makes the device's primary context current on this thread
    const unsigned long long ctx = current_context_id();
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_ptr[dev] || g_scratch_ctx[dev] != ctx) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_rate_scratch);
        if (e != cudaSuccess || !p)
            throw Error(CLES_ECUDA, std::string("cudaGetSymbolAddress(g_rate_scratch): ") + cudaGetErrorString(e));
        g_scratch_ptr[dev] = static_cast<double*>(p);
        g_scratch_ctx[dev] = ctx;
    }
    return g_scratch_ptr[dev];
}

}  // namespace
}  // namespace cles

using namespace cles;

extern "C" int cles_max_rate_static(const double* Q_dev, const double* art_dev, int64_t cells, int n_species,
                                    const double* R, const double* gamma, const double* inv_h, double mu0, double Pr,
                                    double Sc, double* result_dev, void* stream) {
    try {
        if (!Q_dev || !art_dev || !R || !gamma || !inv_h || !result_dev)
            throw Error(CLES_EINVAL, "cles_max_rate_static: null argument");
        if (n_species < 1 || n_species > CLES_MAX_SPECIES)
            throw Error(CLES_EINVAL, "cles_max_rate_static: species count must be 1.." + std::to_string(CLES_MAX_SPECIES));
        if (cells < 1 || cells > CLES_STATIC_MAX_CELLS)
            throw Error(CLES_EINVAL, "cles_max_rate_static: " + std::to_string(cells) +
                                         " cells exceed the static scratch limit of " +
                                         std::to_string((long long)CLES_STATIC_MAX_CELLS) +
                                         " cells; use cles_max_rate on a solver instead");
        StaticRateArgs a{};
        for (int k = 0; k < n_species; ++k) {
            if (!(gamma[k] > 1.0)) throw Error(CLES_EINVAL, "cles_max_rate_static: gamma must exceed 1");
            a.Rk[k] = R[k];
            a.cvk[k] = R[k] / (gamma[k] - 1);
        }
        for (int d = 0; d < 3; ++d) a.inv_h[d] = inv_h[d];
        a.mu0 = mu0;
        a.Pr = Pr;
        a.Sc = Sc;
        cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
        if (st) {
            int dev = 0, sdev = 0;
            CLES_CUDA(cudaGetDevice(&dev));
            CLES_CUDA(cudaStreamGetDevice(st, &sdev));
            if (sdev != dev)
                throw Error(CLES_EINVAL, "cles_max_rate_static: the stream belongs to device " +
                                             std::to_string(sdev) + ", not the current device " +
                                             std::to_string(dev));
        }
        double* scratch = scratch_for_current_device();
        const int nb = (int)((cells + kCellsPerBlock - 1) / kCellsPerBlock);
        k_rate_static_partial<<<nb, kStaticThreads, 0, st>>>(Q_dev, art_dev, cells, n_species, a, scratch);
        count_launch();
        check_launch("k_rate_static_partial");
        k_rate_static_final<<<1, kStaticThreads, 0, st>>>(scratch, nb, result_dev);
        count_launch();
        check_launch("k_rate_static_final");
    } catch (const Error& e) {
        set_last_error(e.what());
        return e.code;
    } catch (const std::exception& e) {
        set_last_error(e.what());
        return CLES_EINVAL;
    }
    set_last_error("");
    return CLES_OK;
}
