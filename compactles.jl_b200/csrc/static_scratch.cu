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
//     cudaGetSymbolAddress (once per device, with that device current).  Make
//     that first call before any stream capture.
// The per-cell arithmetic is the one of cles_max_rate (the primitives of
// src/physics.jl:604-653 and the rate of src/timestep.jl:125-175), so both
// entry points return identical values for the same inputs.

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

// Device address of g_rate_scratch, looked up once per device.
constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
double* g_scratch_ptr[kMaxDevices] = {};

double* scratch_for_current_device() {
    int dev = 0;
    CLES_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) throw Error(CLES_EINVAL, "device index out of range");
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_ptr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_rate_scratch);
        if (e != cudaSuccess || !p)
            throw Error(CLES_ECUDA, std::string("cudaGetSymbolAddress(g_rate_scratch): ") + cudaGetErrorString(e));
        g_scratch_ptr[dev] = static_cast<double*>(p);
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
        double* scratch = scratch_for_current_device();
        const int nb = (int)((cells + kCellsPerBlock - 1) / kCellsPerBlock);
        cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
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
