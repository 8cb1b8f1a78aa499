// TMA-pipelined compact operators for y/z lines: periodic tridiagonal lines
// with identical segments (k_compact_tma), and closed or pentadiagonal lines
// with per-segment tables (k_compact_tg).
//
// y and z lines are strided in memory (x is contiguous), so a group of 32
// consecutive-x lines is a 2-D box {32 x, n along the line} of the field: one
// `cp.async.bulk.tensor` copy brings it into shared memory as tile[g][lane],
// which every thread then reads by column without bank conflicts.  The
// kernels are persistent (two CTAs per SM for 32-point segments, one for
// 16-point ones and for the FP64 RK-fused store of k_compact_tma) and keep NS
// tiles in flight: the copy of a later group is issued as soon as the current
// tile has been read into registers, so HBM is busy while the segments solve.  Compute per group is
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

constexpr uint64_t kWaitLimitNs = 2000000000ull;

// Wait for phase `parity` of `bar`, at most limit_ns (2 s in every operator).
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, unsigned parity,
                                                  uint64_t limit_ns = kWaitLimitNs) {
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = global_ns();
    while (true) {
        if (mbar_try_wait(bar, parity)) return true;
        if (global_ns() - t0 > limit_ns) return false;
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

__device__ __forceinline__ void prefetch_l2(const void* p) {
    asm volatile("prefetch.global.L2 [%0];" ::"l"(reinterpret_cast<uint64_t>(p)));
}

// The MS + 2M stencil inputs of the segment starting at line index `off`,
// read down one column of a tile whose row g + H holds line index g (PITCH
// elements a row; `col` already points at this lane's column).  The segment's
// own MS values sit at fixed offsets from one address; only the M values
// before and the M after it can fall beyond the line: they wrap on periodic
// lines, read the halo row at an open end and clamp to the end value
// otherwise (closure rows replace what a clamped value feeds).
template <typename T, int M, int MS, int PITCH>
__device__ __forceinline__ void gather_window(const T* col, int off, int n, int H, bool periodic, bool lo_open,
                                              bool hi_open, T (&wv)[MS + 2 * M]) {
    const T* mid = col + (off + H) * PITCH;
#pragma unroll
    for (int j = 0; j < MS; ++j) wv[M + j] = mid[j * PITCH];
#pragma unroll
    for (int k = 0; k < M; ++k) {
        int g = off - M + k;
        if (g < 0) g = periodic ? g + n : (lo_open ? g : 0);
        wv[k] = col[(g + H) * PITCH];
        int h = off + MS + k;
        if (h >= n) h = periodic ? h - n : (hi_open ? h : n - 1);
        wv[MS + M + k] = col[(h + H) * PITCH];
    }
}

template <typename T>
__device__ __forceinline__ T tl(const double* d, const float* f, int i) {
    if (sizeof(T) == 8) return T(d[i]);
    return T(f[i]);
}

// CPS persistent CTAs share an SM.  Lines of 32-point segments run two (at
// most 128 registers a thread; as many tiles in flight as half the SM's
// shared memory holds: 3 in FP32, 1 for a 256-point FP64 line): one CTA of 8
// warps, whose segments all wait on the same tile, cannot keep an SM's issue
// slots busy.  The FP64 RK-fused store is the exception: its three extra
// global streams (dQ, du, Q) want the deeper pipeline of one CTA with three
// tiles in flight (256^3 Taylor-Green step, z lines: 5.5 TB/s against 5.1).
template <typename T, int M, int MS, int CPS>
__global__ void __launch_bounds__(MS == 16 ? 512 : 256, CPS)
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
        if (mode == OUT_RK || mode == OUT_SUBTRACT) {
            // the store phase reads the output (and du, Q for the RK update):
            // pull those rows into L2 now, while the tile is still arriving.
            // Lane l takes row off + l of its segment, both 128-byte halves.
            const int c = w / groups, g = w - (w / groups) * groups;
            const int x0 = (g % gx) * kLanes, o = g / gx;
            if (lane < MS) {
                const int64_t st = P.dim == 1 ? out.sy : out.sz;
                const int64_t ob = P.dim == 1 ? (int64_t)o * out.sz : (int64_t)o * out.sy;
                const int64_t e = (int64_t)c * out.comp_stride + x0 + ob + (int64_t)(off + lane) * st;
                const bool second = x0 + 16 < P.nx;
                const T* ob_ = reinterpret_cast<const T*>(out.base) + e;
                prefetch_l2(ob_);
                if (sizeof(T) == 8 && second) prefetch_l2(ob_ + 16);
                if (mode == OUT_RK) {
                    prefetch_l2(rk.du + e);
                    prefetch_l2(rk.Q + e);
                    if (second) {
                        prefetch_l2(rk.du + e + 16);
                        prefetch_l2(rk.Q + e + 16);
                    }
                }
            }
        }
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
            gather_window<T, M, MS, kLanes>(tile + lane, off, n, 0, true, false, false, wv);
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

template <typename T>
__device__ __forceinline__ T tgv(const double* d, const float* f, int i) {
    if (sizeof(T) == 8) return T(d[i]);
    return T(f[i]);
}

// Local solve of one segment of class CLS (0 first, 1 interior, 2 last).
template <typename T, int Q, int MS, int CLS>
__device__ __forceinline__ void tg_solve(const TileGenParams& G, T (&y)[MS]) {
    if (Q == 1) {
#pragma unroll
        for (int i = 1; i < MS; ++i) y[i] -= tgv<T>(G.f[CLS][0], G.ff[CLS][0], i) * y[i - 1];
        y[MS - 1] *= tgv<T>(G.f[CLS][1], G.ff[CLS][1], MS - 1);
#pragma unroll
        for (int i = MS - 2; i >= 0; --i)
            y[i] = (y[i] - tgv<T>(G.f[CLS][2], G.ff[CLS][2], i) * y[i + 1]) * tgv<T>(G.f[CLS][1], G.ff[CLS][1], i);
    } else {
#pragma unroll
        for (int k = 0; k < MS - 1; ++k) {
            y[k + 1] -= tgv<T>(G.f[CLS][0], G.ff[CLS][0], k) * y[k];
            if (k + 2 < MS) y[k + 2] -= tgv<T>(G.f[CLS][1], G.ff[CLS][1], k) * y[k];
        }
#pragma unroll
        for (int i = MS - 1; i >= 0; --i) {
            T acc = y[i];
            if (i + 1 < MS) acc -= tgv<T>(G.f[CLS][2], G.ff[CLS][2], i) * y[i + 1];
            if (i + 2 < MS) acc -= tgv<T>(G.f[CLS][3], G.ff[CLS][3], i) * y[i + 2];
            y[i] = acc * tgv<T>(G.f[CLS][4], G.ff[CLS][4], i);
        }
    }
}

// The interface values one segment needs: the previous segment's tails and
// the next segment's heads, rows of the reduced inverse times the gathered
// heads and tails.  The 4Q dot products run in one pass over the gathered
// values with two partial sums each, so their FMA chains overlap instead of
// running one after the other.  N = 2qS is even.
template <typename T, int Q>
__device__ __forceinline__ void tg_interface(const T* Gs, const T* rl, int N, int prev, int next, bool has_prev,
                                             bool has_next, T (&zp)[Q], T (&zn)[Q]) {
    const T* gp[Q];
    const T* gn[Q];
    T ap[Q][2], an[Q][2];
#pragma unroll
    for (int t = 0; t < Q; ++t) {
        gp[t] = Gs + (size_t)(2 * Q * prev + Q + t) * N;
        gn[t] = Gs + (size_t)(2 * Q * next + t) * N;
        ap[t][0] = ap[t][1] = an[t][0] = an[t][1] = T(0);
    }
    for (int j = 0; j < N; j += 2) {
        const T r0 = rl[j], r1 = rl[j + 1];
#pragma unroll
        for (int t = 0; t < Q; ++t) {
            ap[t][0] += gp[t][j] * r0;
            ap[t][1] += gp[t][j + 1] * r1;
            an[t][0] += gn[t][j] * r0;
            an[t][1] += gn[t][j + 1] * r1;
        }
    }
#pragma unroll
    for (int t = 0; t < Q; ++t) {
        zp[t] = has_prev ? ap[t][0] + ap[t][1] : T(0);
        zn[t] = has_next ? an[t][0] + an[t][1] : T(0);
    }
}

template <typename T, int Q, int MS, int CLS>
__device__ __forceinline__ void tg_correct(const TileGenParams& G, T (&y)[MS], const T (&zp)[Q], const T (&zn)[Q]) {
#pragma unroll
    for (int i = 0; i < MS; ++i) {
        T acc = T(0);
#pragma unroll
        for (int t = 0; t < Q; ++t)
            acc += tgv<T>(G.v[CLS][t], G.vf[CLS][t], i) * zp[t] + tgv<T>(G.w[CLS][t], G.wf[CLS][t], i) * zn[t];
        y[i] -= acc;
    }
}

// General tile kernel: the same pipeline for y/z lines whose segments are not
// all alike -- closed lines (closure rows in the first and last segment, spikes
// that stop at the ends) and the pentadiagonal C10 scheme (q = 2, two head and
// two tail values per segment).  Segment coefficients come from the plan's
// three segment classes (first, interior, last) as kernel parameters, the
// closure stencils read the whole line from the tile, and the reduced inverse
// (2qS)^2 sits in shared memory.  Two CTAs share an SM (at most 128 registers
// a thread), each with the tiles in flight that half the shared memory holds.
template <typename T, int Q, int M, int MS>
__global__ void __launch_bounds__(256, 2)
    k_compact_tg(const __grid_constant__ CUtensorMap map, const __grid_constant__ CompactParams P,
                 const __grid_constant__ TileGenParams GP, const T* __restrict__ tab, const FieldView out,
                 const int mode, const int count, const int NS, const RkEpilogue rk, const int H,
                 T* __restrict__ iface) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const int n = P.n, S = P.S;
    constexpr int m = MS;  // points per segment (all segments equal at launch)
    const int N = 2 * Q * S;
    // a split line's tile also holds the H = M halo rows beyond each end
    // (tile row g + H is line index g, g in [-H, n + H))
    const size_t tile_elems = (size_t)(n + 2 * H) * kLanes;
    T* tiles = reinterpret_cast<T*>(smem_raw);
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem_raw + sizeof(T) * tile_elems * NS);
    T* red = reinterpret_cast<T*>(bars + 8);
    const int RP = N + 1;
    T* Gs = red + (size_t)kLanes * RP;

    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int seg = tid >> 5;
    const int off = seg * m;
    const bool periodic = P.periodic != 0;
    const int gx = (P.nx + kLanes - 1) / kLanes;
    const int other = P.dim == 1 ? P.nz : P.ny;
    const int groups = gx * other;
    const int work = groups * count;

    if (tid == 0) {
        for (int s = 0; s < NS; ++s) mbar_init(&bars[s], 1);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    for (int i = tid; i < N * N; i += blockDim.x) Gs[i] = tab[P.off_G + i];
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
    const int cls = seg == 0 ? 0 : (seg == S - 1 ? 2 : 1);   // warp-uniform
    const bool has_prev = periodic || seg > 0;
    const bool has_next = periodic || seg < S - 1;
    const int prev = seg == 0 ? S - 1 : seg - 1;
    const int next = seg == S - 1 ? 0 : seg + 1;

    int it = 0;
    for (int w = blockIdx.x; w < work; w += gridDim.x, ++it) {
        const int stage = it % NS;
        const unsigned parity = (unsigned)((it / NS) & 1);
        const bool ok = mbar_wait_bounded(&bars[stage], parity);
        if (__syncthreads_or(!ok)) {
            if (tid == 0) atomicAdd(&g_wait_timeouts, 1);
            return;
        }
        const T* tile = tiles + tile_elems * stage;
        // ---- fill: interior stencil, closure rows at closed edges ----
        T y[MS];
        {
            T wv[MS + 2 * M];
            gather_window<T, M, MS, kLanes>(tile + lane, off, n, H, periodic, P.lo_open, P.hi_open, wv);
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
        if (P.lo_closed && seg == 0) {
#pragma unroll
            for (int i = 0; i < kMaxClo; ++i) {
                if (i < P.nc) {
                    T acc = T(0);
#pragma unroll
                    for (int k = 0; k < kMaxCloLen; ++k)
                        if (k < P.clo_len[i]) acc += T(P.clo[i][k]) * tile[(k + H) * kLanes + lane];
                    y[i] = acc;
                }
            }
        }
        if (P.hi_closed && seg == S - 1) {
#pragma unroll
            for (int i = MS - kMaxClo; i < MS; ++i) {
                if (i >= m - P.nc) {
                    T acc = T(0);
#pragma unroll
                    for (int k = 0; k < kMaxCloLen; ++k)
                        if (k < P.clo_len[m - 1 - i])
                            acc += T(P.chi[m - 1 - i][k]) * tile[(n - 1 - k + H) * kLanes + lane];
                    y[i] = acc;
                }
            }
        }
        __syncthreads();  // the tile is consumed: refill it with a later group
        if (tid == 0) {
            const int w2 = w + NS * gridDim.x;
            if (w2 < work) issue(w2, stage);
        }
        // ---- local solve with this segment's factorisation ----
        if (cls == 0) tg_solve<T, Q, MS, 0>(GP, y);
        else if (cls == 1) tg_solve<T, Q, MS, 1>(GP, y);
        else tg_solve<T, Q, MS, 2>(GP, y);
        // ---- interface values: heads and tails, then the reduced inverse ----
        T* rl = red + (size_t)lane * RP;
#pragma unroll
        for (int t = 0; t < Q; ++t) {
            rl[2 * Q * seg + t] = y[t];
            rl[2 * Q * seg + Q + t] = y[MS - Q + t];
        }
        __syncthreads();
        T zp[Q], zn[Q];
        tg_interface<T, Q>(Gs, rl, N, prev, next, has_prev, has_next, zp, zn);
        if (cls == 0) tg_correct<T, Q, MS, 0>(GP, y, zp, zn);
        else if (cls == 1) tg_correct<T, Q, MS, 1>(GP, y, zp, zn);
        else tg_correct<T, Q, MS, 2>(GP, y, zp, zn);
        // ---- store ----
        const int c = w / groups, g = w - (w / groups) * groups;
        const int x = (g % gx) * kLanes + lane, o = g / gx;
        if (iface && x < P.nx) {
            // a split line's local heads and tails: [comp][2q][lines], line = x + o nx
            T* ifc = iface + (int64_t)c * 2 * Q * P.lines + x + (int64_t)o * P.nx;
            if (seg == 0) {
#pragma unroll
                for (int t = 0; t < Q; ++t) ifc[(int64_t)t * P.lines] = y[t];
            }
            if (seg == S - 1) {
#pragma unroll
                for (int t = 0; t < Q; ++t) ifc[(int64_t)(Q + t) * P.lines] = y[MS - Q + t];
            }
        }
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
                    T o8[8];
                    double dv[8], qv[8];
#pragma unroll
                    for (int q = 0; q < 8; ++q) {
                        o8[q] = base[(int64_t)(i0 + q) * st];
                        dv[q] = dp[(int64_t)(i0 + q) * st];
                        qv[q] = Qp[(int64_t)(i0 + q) * st];
                    }
#pragma unroll
                    for (int q = 0; q < 8; ++q) {
                        const T dq = o8[q] - y[i0 + q];
                        const double v = rk.A * dv[q] + rdt * double(dq);
                        dp[(int64_t)(i0 + q) * st] = v;
                        Qp[(int64_t)(i0 + q) * st] = qv[q] + rk.B * v;
                    }
                }
            } else if (mode == OUT_SUBTRACT) {
#pragma unroll
                for (int i0 = 0; i0 < MS; i0 += 8) {
                    T o8[8];
#pragma unroll
                    for (int q = 0; q < 8; ++q) o8[q] = base[(int64_t)(i0 + q) * st];
#pragma unroll
                    for (int q = 0; q < 8; ++q) base[(int64_t)(i0 + q) * st] = o8[q] - y[i0 + q];
                }
            } else {
#pragma unroll
                for (int i = 0; i < MS; ++i) base[(int64_t)i * st] = mode == OUT_NEGATE ? -y[i] : y[i];
            }
        }
    }
}

// x lines in the general tile form.  x is the contiguous direction, so a
// group of 32 lines is 32 rows of the field: every warp copies whole rows with
// coalesced 4/8-byte cp.async into a transposed shared-memory tile
// tile[g * 33 + lane] (pitch 33: the column reads of the segment threads and
// the row writes of the copies are both free of bank conflicts).  The compute
// is that of k_compact_tg (three segment classes, closures, reduced inverse in
// shared memory); results go back into the same tile, so that the stores are
// coalesced rows again, and the tile is refilled once they are out.  Two CTAs
// share an SM (at most 128 registers a thread), each with one FP64 tile or two
// FP32 tiles: while one CTA waits on its copies the other computes.
__device__ __forceinline__ void cp_async_el(void* dst, const void* src, int bytes) {
    if (bytes == 8)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

template <typename T, int Q, int M, int MS, int NS>
__global__ void __launch_bounds__(256, 2)
    k_compact_xt(const __grid_constant__ CompactParams P, const __grid_constant__ TileGenParams GP,
                 const T* __restrict__ tab, const FieldView in, const FieldView out, const int mode, const int count,
                 const int H, T* __restrict__ iface) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    constexpr int TP = kLanes + 1;
    const int n = P.n, S = P.S;
    constexpr int m = MS;
    const int N = 2 * Q * S;
    // input tiles also hold a split line's H = M halo elements beyond each
    // end (tile row g + H is line index g); the output tile holds the line
    const size_t tile_elems = (size_t)(n + 2 * H) * TP;
    T* tin = reinterpret_cast<T*>(smem_raw);
    T* red = tin + tile_elems * NS;
    const int RP = N + 1;
    T* Gs = red + (size_t)kLanes * RP;

    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int seg = tid >> 5;           // also the warp index
    const int nwarps = blockDim.x >> 5;
    const int off = seg * m;
    const bool periodic = P.periodic != 0;
    const int64_t lines = P.lines;
    const int groups = (int)((lines + kLanes - 1) / kLanes);
    const int work = groups * count;
    const int cls = seg == 0 ? 0 : (seg == S - 1 ? 2 : 1);
    const bool has_prev = periodic || seg > 0;
    const bool has_next = periodic || seg < S - 1;
    const int prev = seg == 0 ? S - 1 : seg - 1;
    const int next = seg == S - 1 ? 0 : seg + 1;

    for (int i = tid; i < N * N; i += blockDim.x) Gs[i] = tab[P.off_G + i];

    auto row_of = [&](const FieldView& v, int line) -> int64_t {
        const int j = line % P.ny, k = line / P.ny;
        return (int64_t)j * v.sy + (int64_t)k * v.sz;
    };
    // warp w copies rows w, w + nwarps, ...; lane strides the row
    auto issue = [&](int w, int s) {
        if (w < work) {
            const int c = w / groups, g0 = (w - c * groups) * kLanes;
            const T* base = reinterpret_cast<const T*>(in.base) + (int64_t)c * in.comp_stride;
            T* dst = tin + tile_elems * s;
            for (int l = seg; l < kLanes; l += nwarps) {
                const int line = g0 + l;
                if (line >= lines) break;
                const T* row = base + row_of(in, line) - H;
                for (int g = lane; g < n + 2 * H; g += kLanes)
                    cp_async_el(dst + (size_t)g * TP + l, row + g, (int)sizeof(T));
            }
        }
        cp_async_commit();   // an empty group keeps the count in step
    };
#pragma unroll
    for (int s = 0; s < NS; ++s) issue(blockIdx.x + s * gridDim.x, s);

    const T a0 = T(P.a0);
    T ci[M];
#pragma unroll
    for (int k = 0; k < M; ++k) ci[k] = T(P.ci[k]);

    int it = 0;
    for (int w = blockIdx.x; w < work; w += gridDim.x, ++it) {
        const int stage = it % NS;
        if (mode == OUT_SUBTRACT) {
            // the subtract store reads this group's output rows: pull them
            // into L2 while the group's rows are still arriving (lane l < the
            // row's 128-byte lines takes line l; its offset stays below n)
            const int c = w / groups, g0 = (w - c * groups) * kLanes;
            const T* obase = reinterpret_cast<const T*>(out.base) + (int64_t)c * out.comp_stride;
            const int per_row = (n * (int)sizeof(T) + 127) / 128;
            for (int l = seg; l < kLanes; l += nwarps) {
                const int line = g0 + l;
                if (line >= lines) break;
                if (lane < per_row) prefetch_l2(obase + row_of(out, line) + lane * (128 / (int)sizeof(T)));
            }
        }
        cp_async_wait<NS - 1>();
        __syncthreads();   // this group's rows are in the tile for every thread
        const T* tile = tin + tile_elems * stage;
        T y[MS];
        {
            T wv[MS + 2 * M];
            gather_window<T, M, MS, TP>(tile + lane, off, n, H, periodic, P.lo_open, P.hi_open, wv);
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
        if (P.lo_closed && seg == 0) {
#pragma unroll
            for (int i = 0; i < kMaxClo; ++i) {
                if (i < P.nc) {
                    T acc = T(0);
#pragma unroll
                    for (int k = 0; k < kMaxCloLen; ++k)
                        if (k < P.clo_len[i]) acc += T(P.clo[i][k]) * tile[(k + H) * TP + lane];
                    y[i] = acc;
                }
            }
        }
        if (P.hi_closed && seg == S - 1) {
#pragma unroll
            for (int i = MS - kMaxClo; i < MS; ++i) {
                if (i >= m - P.nc) {
                    T acc = T(0);
#pragma unroll
                    for (int k = 0; k < kMaxCloLen; ++k)
                        if (k < P.clo_len[m - 1 - i])
                            acc += T(P.chi[m - 1 - i][k]) * tile[(n - 1 - k + H) * TP + lane];
                    y[i] = acc;
                }
            }
        }
        if (cls == 0) tg_solve<T, Q, MS, 0>(GP, y);
        else if (cls == 1) tg_solve<T, Q, MS, 1>(GP, y);
        else tg_solve<T, Q, MS, 2>(GP, y);
        T* rl = red + (size_t)lane * RP;
#pragma unroll
        for (int t = 0; t < Q; ++t) {
            rl[2 * Q * seg + t] = y[t];
            rl[2 * Q * seg + Q + t] = y[MS - Q + t];
        }
        __syncthreads();   // interface values visible; every thread has read the tile
        T zp[Q], zn[Q];
        tg_interface<T, Q>(Gs, rl, N, prev, next, has_prev, has_next, zp, zn);
        if (cls == 0) tg_correct<T, Q, MS, 0>(GP, y, zp, zn);
        else if (cls == 1) tg_correct<T, Q, MS, 1>(GP, y, zp, zn);
        else tg_correct<T, Q, MS, 2>(GP, y, zp, zn);
        if (iface) {
            // a split line's local heads and tails: [comp][2q][lines]
            const int c = w / groups;
            const int64_t line = (int64_t)(w - c * groups) * kLanes + lane;
            if (line < lines) {
                T* ifc = iface + (int64_t)c * 2 * Q * lines + line;
                if (seg == 0) {
#pragma unroll
                    for (int t = 0; t < Q; ++t) ifc[(int64_t)t * lines] = y[t];
                }
                if (seg == S - 1) {
#pragma unroll
                    for (int t = 0; t < Q; ++t) ifc[(int64_t)(Q + t) * lines] = y[MS - Q + t];
                }
            }
        }
        T* tout = tin + tile_elems * stage + (size_t)H * TP;   // results go back into the input tile
#pragma unroll
        for (int i = 0; i < MS; ++i) tout[(size_t)(off + i) * TP + lane] = y[i];
        __syncthreads();   // the output tile is complete
        {
            const int c = w / groups, g0 = (w - c * groups) * kLanes;
            T* base = reinterpret_cast<T*>(out.base) + (int64_t)c * out.comp_stride;
            for (int l = seg; l < kLanes; l += nwarps) {
                const int line = g0 + l;
                if (line >= lines) break;
                T* row = base + row_of(out, line);
                if (mode == OUT_SUBTRACT) {
                    // read the row's old values four a lane before writing,
                    // so that their loads are in flight together
                    constexpr int kPerLane = 4;
                    for (int g0 = lane; g0 < n; g0 += kPerLane * kLanes) {
                        T old[kPerLane];
#pragma unroll
                        for (int k = 0; k < kPerLane; ++k)
                            if (g0 + k * kLanes < n) old[k] = row[g0 + k * kLanes];
#pragma unroll
                        for (int k = 0; k < kPerLane; ++k) {
                            const int g = g0 + k * kLanes;
                            if (g < n) row[g] = old[k] - tout[(size_t)g * TP + l];
                        }
                    }
                } else {
                    for (int g = lane; g < n; g += kLanes) {
                        const T v = tout[(size_t)g * TP + l];
                        row[g] = mode == OUT_NEGATE ? -v : v;
                    }
                }
            }
        }
        __syncthreads();   // the tile is written out: refill it
        issue(w + NS * gridDim.x, stage);
    }
    cp_async_wait<0>();
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

int num_sms() {
    if (!g_num_sms) {
        int dev = 0;
        CLES_CUDA(cudaGetDevice(&dev));
        CLES_CUDA(cudaDeviceGetAttribute(&g_num_sms, cudaDevAttrMultiProcessorCount, dev));
    }
    return g_num_sms;
}

// Tiles in flight (1 to 3) for a CTA that shares its SM with another: half of
// the 227 KB, less 1 KB the runtime reserves per CTA and the CTA's own
// interface buffers.  A tile is at most 256 rows of 32 lanes (64 KB in FP64).
inline int tiles_for_two_ctas(size_t tile_bytes, size_t extra) {
    const size_t fit = ((227 * 1024) / 2 - 1024 - extra) / tile_bytes;
    return fit < 1 ? 1 : (fit > 3 ? 3 : (int)fit);
}

template <typename T, int M, int MS, int CPS>
void launch_tma_ms(const CompactPlan& plan, const CUtensorMap& map, const FieldView& out, int count, int mode,
                  cudaStream_t st, const T* G, const RkEpilogue& rk) {
    const CompactParams& P = plan.P;
    constexpr int per_sm = CPS;
    const int N = 2 * P.S;
    const size_t extra = 8 * sizeof(uint64_t) + sizeof(T) * ((size_t)kLanes * (N + 1) + (size_t)N * N);
    const size_t tile_bytes = sizeof(T) * (size_t)P.n * kLanes;
    int NS = sizeof(T) == 8 ? 3 : 4;
    if (per_sm == 2) NS = tiles_for_two_ctas(tile_bytes, extra);
    const size_t smem = tile_bytes * NS + extra;
    auto kern = k_compact_tma<T, M, MS, CPS>;
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
    const int slots = g_num_sms * (2 * (smem + 1024) <= 227 * 1024 ? per_sm : 1);
    const int grid = work < slots ? work : slots;
    kern<<<grid, kLanes * P.S, smem, st>>>(map, P, plan.TL, G, out, mode, count, NS, rk);
    count_launch();
    check_launch("k_compact_tma");
}

template <typename T, int M>
bool launch_tma_m(const CompactPlan& plan, const CUtensorMap& map, const FieldView& out, int count, int mode,
                  cudaStream_t st, const T* G, const RkEpilogue& rk) {
    switch (plan.TL.m) {
        case 32:
            if constexpr (sizeof(T) == 8) {
                if (mode == OUT_RK) {
                    launch_tma_ms<T, M, 32, 1>(plan, map, out, count, mode, st, G, rk);
                    return true;
                }
            }
            launch_tma_ms<T, M, 32, 2>(plan, map, out, count, mode, st, G, rk);
            return true;
        case 16: launch_tma_ms<T, M, 16, 1>(plan, map, out, count, mode, st, G, rk); return true;
        default: return false;
    }
}

template <typename T, int Q, int M, int MS>
void launch_tg_ms(const CompactPlan& plan, const CUtensorMap& map, const FieldView& out, int count, int mode,
                  cudaStream_t st, const T* tab, const RkEpilogue& rk, int H, T* iface) {
    const CompactParams& P = plan.P;
    const int N = 2 * Q * P.S;
    const size_t extra = 8 * sizeof(uint64_t) + sizeof(T) * ((size_t)kLanes * (N + 1) + (size_t)N * N);
    const size_t tile_bytes = sizeof(T) * (size_t)(P.n + 2 * H) * kLanes;
    const int NS = tiles_for_two_ctas(tile_bytes, extra);
    const size_t smem = tile_bytes * NS + extra;
    auto kern = k_compact_tg<T, Q, M, MS>;
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
    // at least two persistent CTAs per SM (the kernel is built for two), more
    // for lines of fewer than 8 segments, as shared memory allows
    int per_sm = 256 / (kLanes * P.S);
    if (per_sm < 2) per_sm = 2;
    const int by_smem = (int)((227 * 1024) / (smem + 1024));
    if (per_sm > by_smem) per_sm = by_smem;
    if (per_sm < 1) per_sm = 1;
    const int slots = g_num_sms * per_sm;
    const int grid = work < slots ? work : slots;
    kern<<<grid, kLanes * P.S, smem, st>>>(map, P, plan.TG, tab, out, mode, count, NS, rk, H, iface);
    count_launch();
    check_launch("k_compact_tg");
}

template <typename T>
bool launch_tg(const CompactPlan& plan, const CUtensorMap& map, const FieldView& out, int count, int mode,
               cudaStream_t st, const T* tab, const RkEpilogue& rk, int H = 0, T* iface = nullptr) {
    const CompactParams& P = plan.P;
    const bool m32 = P.seg_base == 32;
    if (P.q == 1) {
        switch (P.M) {
            case 1: m32 ? launch_tg_ms<T, 1, 1, 32>(plan, map, out, count, mode, st, tab, rk, H, iface)
                        : launch_tg_ms<T, 1, 1, 16>(plan, map, out, count, mode, st, tab, rk, H, iface); return true;
            case 2: m32 ? launch_tg_ms<T, 1, 2, 32>(plan, map, out, count, mode, st, tab, rk, H, iface)
                        : launch_tg_ms<T, 1, 2, 16>(plan, map, out, count, mode, st, tab, rk, H, iface); return true;
            case 4: m32 ? launch_tg_ms<T, 1, 4, 32>(plan, map, out, count, mode, st, tab, rk, H, iface)
                        : launch_tg_ms<T, 1, 4, 16>(plan, map, out, count, mode, st, tab, rk, H, iface); return true;
            default: return false;
        }
    }
    if (P.q == 2 && P.M == 3) {
        m32 ? launch_tg_ms<T, 2, 3, 32>(plan, map, out, count, mode, st, tab, rk, H, iface)
            : launch_tg_ms<T, 2, 3, 16>(plan, map, out, count, mode, st, tab, rk, H, iface);
        return true;
    }
    return false;
}

template <typename T, int Q, int M, int MS>
void launch_xt_ms(const CompactPlan& plan, const FieldView& in, const FieldView& out, int count, int mode,
                  cudaStream_t st, const T* tab, int H, T* iface) {
    const CompactParams& P = plan.P;
    constexpr int NS = sizeof(T) == 8 ? 1 : 2;
    const int N = 2 * Q * P.S;
    const size_t smem = sizeof(T) * ((size_t)(P.n + 2 * H) * (kLanes + 1) * NS +
                                     (size_t)kLanes * (N + 1) + (size_t)N * N);
    auto kern = k_compact_xt<T, Q, M, MS, NS>;
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
    const int64_t groups = (P.lines + kLanes - 1) / kLanes;
    const int64_t work = groups * count;
    // at least two persistent CTAs per SM (the kernel is built for two), more
    // for lines of fewer than 8 segments, as shared memory allows
    int per_sm = 256 / (kLanes * P.S);
    if (per_sm < 2) per_sm = 2;
    const int by_smem = (int)((227 * 1024) / (smem + 1024));
    if (per_sm > by_smem) per_sm = by_smem;
    if (per_sm < 1) per_sm = 1;
    const int64_t slots = (int64_t)g_num_sms * per_sm;
    const int grid = (int)(work < slots ? work : slots);
    kern<<<grid, kLanes * P.S, smem, st>>>(P, plan.TG, tab, in, out, mode, count, H, iface);
    count_launch();
    check_launch("k_compact_xt");
}

template <typename T>
bool launch_xt(const CompactPlan& plan, const FieldView& in, const FieldView& out, int count, int mode,
               cudaStream_t st, const T* tab, int H = 0, T* iface = nullptr) {
    const CompactParams& P = plan.P;
    const bool m32 = P.seg_base == 32;
    if (P.q == 1) {
        switch (P.M) {
            case 1: m32 ? launch_xt_ms<T, 1, 1, 32>(plan, in, out, count, mode, st, tab, H, iface)
                        : launch_xt_ms<T, 1, 1, 16>(plan, in, out, count, mode, st, tab, H, iface); return true;
            case 2: m32 ? launch_xt_ms<T, 1, 2, 32>(plan, in, out, count, mode, st, tab, H, iface)
                        : launch_xt_ms<T, 1, 2, 16>(plan, in, out, count, mode, st, tab, H, iface); return true;
            case 4: m32 ? launch_xt_ms<T, 1, 4, 32>(plan, in, out, count, mode, st, tab, H, iface)
                        : launch_xt_ms<T, 1, 4, 16>(plan, in, out, count, mode, st, tab, H, iface); return true;
            default: return false;
        }
    }
    if (P.q == 2 && P.M == 3) {
        m32 ? launch_xt_ms<T, 2, 3, 32>(plan, in, out, count, mode, st, tab, H, iface)
            : launch_xt_ms<T, 2, 3, 16>(plan, in, out, count, mode, st, tab, H, iface);
        return true;
    }
    return false;
}

}  // namespace

bool try_launch_xt(const CompactPlan& plan, const FieldView& in, const FieldView& out, int count, int mode,
                   cudaStream_t st) {
    if (!plan.has_tg || plan.P.dim != 0 || mode == OUT_RK) return false;
    if (plan.P.lo_open || plan.P.hi_open) return false;   // halo rows are not staged here
    const CompactParams& P = plan.P;
    if (P.n > 256 || P.S * kLanes > 256) return false;
    // a persistent CTA holds ~200 KB of shared memory: worth it only when the
    // launch has work for every SM (small grids, often run concurrently on
    // other streams, keep the light generic kernel)
    if (((P.lines + kLanes - 1) / kLanes) * count < num_sms()) return false;
    const size_t el = plan.dtype == CLES_F64 ? 8 : 4;
    // cp.async of one element needs element-aligned addresses only
    if ((uintptr_t)in.base % el || (uintptr_t)out.base % el) return false;
    if (plan.dtype == CLES_F64) return launch_xt<double>(plan, in, out, count, mode, st, plan.tab64);
    return launch_xt<float>(plan, in, out, count, mode, st, plan.tab32);
}

bool try_launch_tma(const CompactPlan& plan, const FieldView& in, const FieldView& out, int count, int mode,
                    cudaStream_t st, const RkEpilogue* rkp) {
    RkEpilogue rk{nullptr, nullptr, 0.0, 0.0, 0.0, nullptr};
    if (rkp) rk = *rkp;
    if (mode == OUT_RK && !rkp) return false;
    if (!plan.has_tl && !plan.has_tg) return false;
    if (plan.P.lo_open || plan.P.hi_open) return false;   // split lines: try_launch_tg_split
    const CompactParams& P = plan.P;
    // 16-point segments run 16 warps per line group (512 threads), 32-point ones 8
    const int max_threads = plan.has_tl && plan.TL.m == 16 ? 512 : 256;
    if (P.dim == 0 || P.n > 256 || P.S * kLanes > max_threads) return false;
    if (!plan.has_tl) {
        const int64_t gx = (P.nx + kLanes - 1) / kLanes;
        if (gx * (P.dim == 1 ? P.nz : P.ny) * count < num_sms()) return false;   // see try_launch_xt
    }
    if (plan.has_tl && (P.q != 1 || !P.periodic || P.M < 1 || P.M > 4 || P.M == 3)) return false;
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
    if (!plan.has_tl) {
        if (plan.dtype == CLES_F64) return launch_tg<double>(plan, map, out, count, mode, st, plan.tab64, rk);
        return launch_tg<float>(plan, map, out, count, mode, st, plan.tab32, rk);
    }
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

bool try_launch_tg_split(const CompactPlan& plan, const FieldView& in, const FieldView& out, int count, void* iface,
                         cudaStream_t st) {
    if (!plan.has_tg) return false;
    const CompactParams& P = plan.P;
    if (P.dim == 0) {
        // x pieces: cp.async rows widened by the M halo elements at each end
        if (P.n > 256 || P.S * kLanes > 256) return false;
        if (((P.lines + kLanes - 1) / kLanes) * count < num_sms()) return false;
        const size_t el = plan.dtype == CLES_F64 ? 8 : 4;
        if ((uintptr_t)in.base % el || (uintptr_t)out.base % el) return false;
        const int H = (P.lo_open || P.hi_open) ? P.M : 0;
        if (plan.dtype == CLES_F64)
            return launch_xt<double>(plan, in, out, count, OUT_STORE, st, plan.tab64, H, static_cast<double*>(iface));
        return launch_xt<float>(plan, in, out, count, OUT_STORE, st, plan.tab32, H, static_cast<float*>(iface));
    }
    if (P.S * kLanes > 256) return false;
    // the box covers the line and the M halo rows beyond each end (both ends,
    // so the tile layout does not depend on which end is open)
    const int H = (P.lo_open || P.hi_open) ? P.M : 0;
    const int rows = P.n + 2 * H;
    if (rows > 256) return false;   // TMA box extent limit
    const int64_t gx = (P.nx + kLanes - 1) / kLanes;
    if (gx * (P.dim == 1 ? P.nz : P.ny) * count < num_sms()) return false;
    PFN_cuTensorMapEncodeTiled_v12000 enc = encode_fn();
    if (!enc) return false;
    const size_t el = plan.dtype == CLES_F64 ? 8 : 4;
    if ((uintptr_t)in.base % 16 || (in.sy * el) % 16 || (in.sz * el) % 16 || (in.comp_stride * el) % 16) return false;
    const int64_t lstride = P.dim == 1 ? in.sy : in.sz;
    if (in.comp_stride < (int64_t)(P.nz + (P.dim == 2 ? 2 * H : 0)) * in.sz) return false;
    // the map starts H planes before the interior along the line: every box
    // starts at line coordinate 0, x at a multiple of 32
    void* base = const_cast<char*>(reinterpret_cast<const char*>(in.base)) - (int64_t)H * lstride * (int64_t)el;
    CUtensorMap map;
    cuuint64_t dims[4] = {(cuuint64_t)P.nx, (cuuint64_t)(P.ny + (P.dim == 1 ? 2 * H : 0)),
                          (cuuint64_t)(P.nz + (P.dim == 2 ? 2 * H : 0)), (cuuint64_t)count};
    cuuint64_t strides[3] = {(cuuint64_t)(in.sy * el), (cuuint64_t)(in.sz * el), (cuuint64_t)(in.comp_stride * el)};
    cuuint32_t box[4] = {(cuuint32_t)kLanes, (cuuint32_t)(P.dim == 1 ? rows : 1), (cuuint32_t)(P.dim == 2 ? rows : 1), 1};
    cuuint32_t estr[4] = {1, 1, 1, 1};
    CUresult r = enc(&map, plan.dtype == CLES_F64 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4,
                     base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return false;
    const RkEpilogue rk{nullptr, nullptr, 0.0, 0.0, 0.0, nullptr};
    if (plan.dtype == CLES_F64)
        return launch_tg<double>(plan, map, out, count, OUT_STORE, st, plan.tab64, rk, H, static_cast<double*>(iface));
    return launch_tg<float>(plan, map, out, count, OUT_STORE, st, plan.tab32, rk, H, static_cast<float*>(iface));
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

// The expiry path of the bounded wait, run on purpose: one CTA initialises an
// mbarrier and waits on its first phase, which nothing completes (no copy is
// issued and no thread arrives, so nothing is in flight when it gives up).
// It records the expiry in g_wait_timeouts exactly as the operators do.
__global__ void k_wait_selftest(uint64_t limit_ns) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    __syncthreads();
    const bool ok = mbar_wait_bounded(&bar, 0u, limit_ns);
    if (__syncthreads_or(!ok) && threadIdx.x == 0) atomicAdd(&g_wait_timeouts, 1);
}

void launch_wait_selftest(uint64_t limit_ns, cudaStream_t st) {
    k_wait_selftest<<<1, 64, 0, st>>>(limit_ns);
    check_launch("k_wait_selftest");
    count_launch(1);
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
