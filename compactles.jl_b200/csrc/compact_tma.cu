// TMA-pipelined compact operator for periodic tridiagonal y/z lines.
//
// y and z lines are strided in memory (x is contiguous), so a group of 32
// consecutive-x lines is a 2-D box {32 x, n along the line} of the field: one
// `cp.async.bulk.tensor` copy brings it into shared memory as tile[g][lane],
// which every thread then reads by column without bank conflicts.  The kernel
// is persistent (one CTA per SM) and keeps NS tiles in flight: the copy of a
// later group is issued as soon as the current tile has been read into
// registers, so HBM is busy while the segments solve.  Compute per group is
// the segmented spike solve of compact.cu (fill, per-segment Thomas sweep,
// interface values from the reduced inverse, correction) with the segment
// coefficients as kernel parameters; results go straight from registers to
// global memory with coalesced stores (lanes are consecutive x).
//
// Every mbarrier wait is bounded by the global timer (2 s): on expiry the
// kernel records the timeout in g_wait_timeouts and returns; the host turns it
// into CLES_ETIMEOUT.  A TMA box start is always a multiple of 32 elements in
// x (256 B in FP64, 128 B in FP32), so the 16-byte rule on the innermost
// coordinate holds.

#include <cuda.h>
#include <cudaTypedefs.h>

#include <mutex>

#include "cles_internal.h"

namespace cles {

__device__ int g_wait_timeouts;

namespace {

constexpr int kLanes = 32;

__device__ __forceinline__ unsigned smem_addr(const void* p) {
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Wait for phase `parity` of `bar`, at most ~2 s.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, unsigned parity) {
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = global_ns();
    while (true) {
        if (mbar_try_wait(bar, parity)) return true;
        if (global_ns() - t0 > 2000000000ull) return false;
    }
}

__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, uint64_t* bar, int c0, int c1, int c2,
                                            int c3) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
        "%5}], [%6];" ::"r"(smem_addr(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_addr(bar))
        : "memory");
}

template <typename T>
__device__ __forceinline__ T tl(const double* d, const float* f, int i) {
    if (sizeof(T) == 8) return T(d[i]);
    return T(f[i]);
}

template <typename T, int M, int MS>
__global__ void __launch_bounds__(256, 1)
    k_compact_tma(const __grid_constant__ CUtensorMap map, const __grid_constant__ CompactParams P,
                  const __grid_constant__ TileLineParams TL,
                  const T* __restrict__ Gg, const FieldView out, const int mode, const int count, const int NS,
                  const RkEpilogue rk) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const int n = P.n, S = P.S;
    constexpr int m = MS;  // points per segment (TL.m == MS at launch)
    const int N = 2 * S;
    const size_t tile_elems = (size_t)n * kLanes;
    T* tiles = reinterpret_cast<T*>(smem_raw);
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem_raw + sizeof(T) * tile_elems * NS);
    T* red = reinterpret_cast<T*>(bars + 8);
    const int RP = N + 1;
    T* Gs = red + (size_t)kLanes * RP;

    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int seg = tid >> 5;
    const int off = seg * m;
    // work items: (component, group of 32 x-consecutive lines)
    const int gx = (P.nx + kLanes - 1) / kLanes;
    const int other = P.dim == 1 ? P.nz : P.ny;
    const int groups = gx * other;
    const int work = groups * count;

    if (tid == 0) {
        for (int s = 0; s < NS; ++s) mbar_init(&bars[s], 1);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    for (int i = tid; i < N * N; i += blockDim.x) Gs[i] = Gg[i];
    __syncthreads();

    const unsigned tile_bytes = (unsigned)(sizeof(T) * tile_elems);
    auto issue = [&](int w, int s) {
        const int c = w / groups, g = w - (w / groups) * groups;
        const int x0 = (g % gx) * kLanes, o = g / gx;
        mbar_expect_tx(&bars[s], tile_bytes);
        if (P.dim == 1) tma_load_4d(tiles + tile_elems * s, &map, &bars[s], x0, 0, o, c);
        else tma_load_4d(tiles + tile_elems * s, &map, &bars[s], x0, o, 0, c);
    };
    if (tid == 0)
        for (int s = 0; s < NS; ++s) {
            const int w = blockIdx.x + s * gridDim.x;
            if (w < work) issue(w, s);
        }

    const T a0 = T(P.a0);
    T ci[M];
#pragma unroll
    for (int k = 0; k < M; ++k) ci[k] = T(P.ci[k]);

    int it = 0;
    for (int w = blockIdx.x; w < work; w += gridDim.x, ++it) {
        const int stage = it % NS;
        const unsigned parity = (unsigned)((it / NS) & 1);
        // bounded wait, decided block-wide so no thread is left at a barrier
        const bool ok = mbar_wait_bounded(&bars[stage], parity);
        if (__syncthreads_or(!ok)) {
            if (tid == 0) atomicAdd(&g_wait_timeouts, 1);
            return;
        }
        const T* tile = tiles + tile_elems * stage;
        // ---- fill from the tile (periodic wrap by index) ----
        T y[MS];
        {
            T wv[MS + 2 * M];
#pragma unroll
            for (int j = 0; j < MS + 2 * M; ++j) {
                if (j < m + 2 * M) {
                    int g = off - M + j;
                    g = g < 0 ? g + n : (g >= n ? g - n : g);
                    wv[j] = tile[g * kLanes + lane];
                } else {
                    wv[j] = T(0);
                }
            }
#pragma unroll
            for (int i = 0; i < MS; ++i) {
                T acc;
                if (P.symmetric) {
                    acc = a0 * wv[i + M];
#pragma unroll
                    for (int k = 1; k <= M; ++k) acc += ci[k - 1] * (wv[i + M + k] + wv[i + M - k]);
                } else {
                    acc = T(0);
#pragma unroll
                    for (int k = 1; k <= M; ++k) acc += ci[k - 1] * (wv[i + M + k] - wv[i + M - k]);
                }
                y[i] = acc;
            }
        }
        __syncthreads();  // the tile is consumed: refill it with a later group
        if (tid == 0) {
            const int w2 = w + NS * gridDim.x;
            if (w2 < work) issue(w2, stage);
        }
        // ---- segment Thomas sweep (uniform coefficients) ----
#pragma unroll
        for (int i = 1; i < MS; ++i)
            if (i < m) y[i] -= tl<T>(TL.l, TL.lf, i) * y[i - 1];
#pragma unroll
        for (int i = 0; i < MS; ++i)
            if (i == m - 1) y[i] *= tl<T>(TL.dinv, TL.dinvf, i);
#pragma unroll
        for (int i = MS - 2; i >= 0; --i)
            if (i < m - 1) y[i] = (y[i] - tl<T>(TL.c, TL.cf, i) * y[i + 1]) * tl<T>(TL.dinv, TL.dinvf, i);
        // ---- interface values ----
        T* rl = red + (size_t)lane * RP;
        rl[2 * seg] = y[0];
#pragma unroll
        for (int i = 0; i < MS; ++i)
            if (i == m - 1) rl[2 * seg + 1] = y[i];
        __syncthreads();
        const int prev = seg == 0 ? S - 1 : seg - 1;
        const int next = seg == S - 1 ? 0 : seg + 1;
        const T* gp = Gs + (size_t)(2 * prev + 1) * N;
        const T* gn = Gs + (size_t)(2 * next) * N;
        T zp = T(0), zn = T(0);
        for (int j = 0; j < N; ++j) {
            const T r = rl[j];
            zp += gp[j] * r;
            zn += gn[j] * r;
        }
#pragma unroll
        for (int i = 0; i < MS; ++i)
            if (i < m) y[i] -= tl<T>(TL.v, TL.vf, i) * zp + tl<T>(TL.w, TL.wf, i) * zn;
        // ---- store ----
        const int c = w / groups, g = w - (w / groups) * groups;
        const int x = (g % gx) * kLanes + lane, o = g / gx;
        if (x < P.nx) {
            T* base = reinterpret_cast<T*>(out.base) + (int64_t)c * out.comp_stride + x;
            int64_t st, ob;
            if (P.dim == 1) { st = out.sy; ob = (int64_t)o * out.sz; }
            else { st = out.sz; ob = (int64_t)o * out.sy; }
            base += ob + (int64_t)off * st;
            if (mode == OUT_RK) {
                const int64_t eo = (int64_t)c * out.comp_stride + x + ob + (int64_t)off * st;
                const double rdt = rk.dtp ? *rk.dtp : rk.dt;
                double* Qp = rk.Q + eo;
                double* dp = rk.du + eo;
#pragma unroll
                for (int i0 = 0; i0 < MS; i0 += 8) {
                    T o[8];
                    double dv[8], qv[8];
#pragma unroll
                    for (int q = 0; q < 8; ++q) {
                        o[q] = base[(int64_t)(i0 + q) * st];
                        dv[q] = dp[(int64_t)(i0 + q) * st];
                        qv[q] = Qp[(int64_t)(i0 + q) * st];
                    }
#pragma unroll
                    for (int q = 0; q < 8; ++q) {
                        const T dq = o[q] - y[i0 + q];
                        const double v = rk.A * dv[q] + rdt * double(dq);
                        dp[(int64_t)(i0 + q) * st] = v;
                        Qp[(int64_t)(i0 + q) * st] = qv[q] + rk.B * v;
                    }
                }
            } else if (mode == OUT_SUBTRACT) {
                // read the old values 8 at a time before writing, so the loads
                // of a chunk are in flight together instead of one per store
#pragma unroll
                for (int i0 = 0; i0 < MS; i0 += 8) {
                    T o[8];
#pragma unroll
                    for (int q = 0; q < 8; ++q) o[q] = base[(int64_t)(i0 + q) * st];
#pragma unroll
                    for (int q = 0; q < 8; ++q) base[(int64_t)(i0 + q) * st] = o[q] - y[i0 + q];
                }
            } else {
#pragma unroll
                for (int i = 0; i < MS; ++i) base[(int64_t)i * st] = mode == OUT_NEGATE ? -y[i] : y[i];
            }
        }
        // the interface buffer is rewritten only after the next group's first
        // barrier, which every thread reaches after finishing these stores
    }
}

// --------------------------------------------------------------- host side --
PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
        else
            cudaGetLastError();
    });
    return fn;
}

int g_num_sms = 0;

template <typename T, int M, int MS>
void launch_tma_ms(const CompactPlan& plan, const CUtensorMap& map, const FieldView& out, int count, int mode,
                  cudaStream_t st, const T* G, const RkEpilogue& rk) {
    const CompactParams& P = plan.P;
    const int NS = sizeof(T) == 8 ? 3 : 4;
    const int N = 2 * P.S;
    const size_t smem = sizeof(T) * (size_t)P.n * kLanes * NS + 8 * sizeof(uint64_t) +
                        sizeof(T) * ((size_t)kLanes * (N + 1) + (size_t)N * N);
    auto kern = k_compact_tma<T, M, MS>;
    static int configured = 0;
    if (configured < (int)smem) {
        CLES_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        configured = (int)smem;
    }
    if (!g_num_sms) {
        int dev = 0;
        CLES_CUDA(cudaGetDevice(&dev));
        CLES_CUDA(cudaDeviceGetAttribute(&g_num_sms, cudaDevAttrMultiProcessorCount, dev));
    }
    const int gx = (P.nx + kLanes - 1) / kLanes;
    const int work = gx * (P.dim == 1 ? P.nz : P.ny) * count;
    const int grid = work < g_num_sms ? work : g_num_sms;
    kern<<<grid, kLanes * P.S, smem, st>>>(map, P, plan.TL, G, out, mode, count, NS, rk);
    count_launch();
    check_launch("k_compact_tma");
}

template <typename T, int M>
bool launch_tma_m(const CompactPlan& plan, const CUtensorMap& map, const FieldView& out, int count, int mode,
                  cudaStream_t st, const T* G, const RkEpilogue& rk) {
    switch (plan.TL.m) {
        case 32: launch_tma_ms<T, M, 32>(plan, map, out, count, mode, st, G, rk); return true;
        case 16: launch_tma_ms<T, M, 16>(plan, map, out, count, mode, st, G, rk); return true;
        default: return false;
    }
}

}  // namespace

bool try_launch_tma(const CompactPlan& plan, const FieldView& in, const FieldView& out, int count, int mode,
                    cudaStream_t st, const RkEpilogue* rkp) {
    RkEpilogue rk{nullptr, nullptr, 0.0, 0.0, 0.0, nullptr};
    if (rkp) rk = *rkp;
    if (mode == OUT_RK && !rkp) return false;
    if (!plan.has_tl) return false;
    const CompactParams& P = plan.P;
    if (P.dim == 0 || P.q != 1 || !P.periodic || P.n > 256 || P.S * kLanes > 256) return false;
    if (P.M < 1 || P.M > 4 || P.M == 3) return false;
    PFN_cuTensorMapEncodeTiled_v12000 enc = encode_fn();
    if (!enc) return false;
    const size_t el = plan.dtype == CLES_F64 ? 8 : 4;
    // TMA needs a 16-byte aligned base and strides that are multiples of 16 bytes
    if ((uintptr_t)in.base % 16 || (in.sy * el) % 16 || (in.sz * el) % 16 || (in.comp_stride * el) % 16) return false;
    if (in.comp_stride < (int64_t)P.nz * in.sz) return false;
    CUtensorMap map;
    cuuint64_t dims[4] = {(cuuint64_t)P.nx, (cuuint64_t)P.ny, (cuuint64_t)P.nz, (cuuint64_t)count};
    cuuint64_t strides[3] = {(cuuint64_t)(in.sy * el), (cuuint64_t)(in.sz * el), (cuuint64_t)(in.comp_stride * el)};
    cuuint32_t box[4] = {(cuuint32_t)kLanes, (cuuint32_t)(P.dim == 1 ? P.n : 1), (cuuint32_t)(P.dim == 2 ? P.n : 1), 1};
    cuuint32_t estr[4] = {1, 1, 1, 1};
    CUresult r = enc(&map, plan.dtype == CLES_F64 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4,
                     in.base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return false;
    const int M = P.M;
    if (plan.TL.m != 32 && plan.TL.m != 16) return false;
    if (plan.dtype == CLES_F64) {
        const double* G = plan.tab64 + P.off_G;
        if (M == 1) return launch_tma_m<double, 1>(plan, map, out, count, mode, st, G, rk);
        if (M == 2) return launch_tma_m<double, 2>(plan, map, out, count, mode, st, G, rk);
        return launch_tma_m<double, 4>(plan, map, out, count, mode, st, G, rk);
    }
    const float* G = plan.tab32 + P.off_G;
    if (M == 1) return launch_tma_m<float, 1>(plan, map, out, count, mode, st, G, rk);
    if (M == 2) return launch_tma_m<float, 2>(plan, map, out, count, mode, st, G, rk);
    return launch_tma_m<float, 4>(plan, map, out, count, mode, st, G, rk);
}

bool launch_compact_rk(const CompactPlan& plan, const FieldView& in, const FieldView& out, int count,
                       const RkEpilogue& rk, cudaStream_t st) {
    if (count <= 0 || plan.P.lines == 0) return false;
    int rec = -1;
    if (profiling()) {
        const double el = plan.dtype == CLES_F64 ? 8.0 : 4.0;
        const double pts = (double)plan.P.lines * plan.P.n * count;
        // input read, dQ read, du and Q read and written (8 bytes each)
        rec = prof_begin(st, plan.P.dim, pts * (2.0 * el + 32.0));
    }
    const bool ok = try_launch_tma(plan, in, out, count, OUT_RK, st, &rk);
    if (rec >= 0) prof_end(rec, st);
    return ok;
}

int take_device_timeouts(cudaStream_t st) {
    int h = 0;
    CLES_CUDA(cudaMemcpyFromSymbolAsync(&h, g_wait_timeouts, sizeof(int), 0, cudaMemcpyDeviceToHost, st));
    CLES_CUDA(cudaStreamSynchronize(st));
    if (h) {
        const int zero = 0;
        CLES_CUDA(cudaMemcpyToSymbolAsync(g_wait_timeouts, &zero, sizeof(int), 0, cudaMemcpyHostToDevice, st));
        CLES_CUDA(cudaStreamSynchronize(st));
    }
    return h;
}

}  // namespace cles
