// Directional compact operators as batched line solves on sm_100a.
//
// One CTA owns LB lines (`lane` = line within the CTA) cut into S segments
// (`seg` = thread row), so thread (lane, seg) owns at most kMaxSeg points of
// one line in registers.  Per application:
//   1. gather   — the segment's RHS window f[off-M, off+m+M): straight from
//                 global memory for y/z lines (lanes are consecutive x, so every
//                 warp load is one coalesced 32-element row), from a transposed
//                 shared-memory tile for x lines (the tile is filled with
//                 coalesced row loads; column reads are bank-conflict free);
//   2. fill     — interior stencil a0 f + sum c_m (f+m ± f-m) and the closure
//                 rows at closed edges (src/operators.jl:113-174);
//   3. solve    — local Thomas (q = 1) or banded LU (q = 2) sweep with the
//                 segment's own factorisation (src/tridiag.jl:46-57,
//                 src/banded.jl:63-80);
//   4. interface — heads/tails to shared memory, each thread forms the two
//                 interface values it needs from the precomputed inverse of the
//                 reduced system (src/tridiag.jl:136-170, src/banded.jl:177-214);
//   5. correct  — x = y - V z_prev - W z_next, then store (overwrite, negate, or
//                 subtract-accumulate into the output).
// Periodic lines wrap by index and closed lines use closure rows, so halos of
// the caller's arrays are never read -- except at the open ends of a split
// line (one rank's piece), where the stencil reads the halo the caller filled
// from the neighbouring rank, as the reference's fill does after
// exchange_halos! (src/operators.jl:113-174).

#include <cstdio>
#include <type_traits>

#include "cles_internal.h"
#include "compact_body.cuh"

namespace cles {

namespace {

template <typename T, int Q, int M, bool XMODE, int MS>
__global__ void __launch_bounds__(512) k_compact(const __grid_constant__ CompactParams P, const T* __restrict__ tab,
                                                  const FieldView in, const FieldView out, const int mode,
                                                  T* __restrict__ iface) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    compact_lines<T, Q, M, XMODE, MS>(P, tab, in, out, mode, iface, blockIdx.x * P.LB, blockIdx.y, nullptr, smem_raw);
}

// ---------------------------------------------------------------------------
// Warp-per-line kernel for periodic tridiagonal x lines of n = 32 * XP points
// (XP = 2, 4, 6, 8, 12, 16).
// Lane s of a warp owns the XP contiguous points [s*XP, (s+1)*XP) of one line:
// vector loads and stores straight from/to global memory (the warp covers the
// whole contiguous line), stencil halos from the neighbouring lanes by shuffle,
// the lane's Thomas sweep in registers, and the 32-segment interface system by
// parallel cyclic reduction across the lanes with precomputed 2x2 matrices.
// Vector type of the lane's loads and stores: double2, or float4 where the
// lane's XP points are a multiple of 4 (float2 otherwise).
template <typename T, int XP> struct Vec;
template <int XP> struct Vec<double, XP> { using type = double2; static constexpr int W = 2; };
template <int XP> struct Vec<float, XP> {
    using type = typename std::conditional<XP % 4 == 0, float4, float2>::type;
    static constexpr int W = XP % 4 == 0 ? 4 : 2;
};

template <typename T>
__device__ __forceinline__ T wl(const double* d, const float* f, int i) {
    if (sizeof(T) == 8) return T(d[i]);
    return T(f[i]);
}

template <typename T, int M, int XP>
__global__ void __launch_bounds__(256) k_compact_xw(const __grid_constant__ CompactParams P, const __grid_constant__ WarpLineParams W, const FieldView in,
                                                    const FieldView out, const int mode) {
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int line = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (line >= P.lines) return;  // whole warps leave together; no block barrier below
    const int comp = blockIdx.y;
    const int j = line % P.ny, k = line / P.ny;
    const T* src = reinterpret_cast<const T*>(in.base) + (int64_t)comp * in.comp_stride + j * in.sy + k * in.sz + lane * XP;
    T* dst = reinterpret_cast<T*>(out.base) + (int64_t)comp * out.comp_stride + j * out.sy + k * out.sz + lane * XP;
    using V = typename Vec<T, XP>::type;
    constexpr int VW = Vec<T, XP>::W;
    T f[XP];
#pragma unroll
    for (int q = 0; q < XP / VW; ++q) {
        const V v = __ldg(reinterpret_cast<const V*>(src) + q);
        const T* pv = reinterpret_cast<const T*>(&v);
#pragma unroll
        for (int e = 0; e < VW; ++e) f[q * VW + e] = pv[e];
    }
    const int lm = (lane + 31) & 31, lp = (lane + 1) & 31;
    T wv[XP + 2 * M];
#pragma unroll
    for (int q = 0; q < M; ++q) {
        wv[q] = __shfl_sync(FULL, f[XP - M + q], lm);
        wv[M + XP + q] = __shfl_sync(FULL, f[q], lp);
    }
#pragma unroll
    for (int i = 0; i < XP; ++i) wv[M + i] = f[i];
    // fill (src/operators.jl:155-172 interior rows)
    T y[XP];
    const T a0 = T(P.a0);
#pragma unroll
    for (int i = 0; i < XP; ++i) {
        T acc;
        if (P.symmetric) {
            acc = a0 * wv[i + M];
#pragma unroll
            for (int m = 1; m <= M; ++m) acc += T(P.ci[m - 1]) * (wv[i + M + m] + wv[i + M - m]);
        } else {
            acc = T(0);
#pragma unroll
            for (int m = 1; m <= M; ++m) acc += T(P.ci[m - 1]) * (wv[i + M + m] - wv[i + M - m]);
        }
        y[i] = acc;
    }
    // lane-local Thomas sweep (src/tridiag.jl:46-57)
#pragma unroll
    for (int i = 1; i < XP; ++i) y[i] -= wl<T>(W.l, W.lf, i) * y[i - 1];
    y[XP - 1] *= wl<T>(W.dinv, W.dinvf, XP - 1);
#pragma unroll
    for (int i = XP - 2; i >= 0; --i) y[i] = (y[i] - wl<T>(W.c, W.cf, i) * y[i + 1]) * wl<T>(W.dinv, W.dinvf, i);
    // interface values: parallel cyclic reduction over the 32 lanes
    T h = y[0], t = y[XP - 1];
#pragma unroll
    for (int s = 0; s < 4; ++s) {
        const int d = 1 << s;
        const T mh = __shfl_sync(FULL, h, (lane - d) & 31), mt = __shfl_sync(FULL, t, (lane - d) & 31);
        const T ph = __shfl_sync(FULL, h, (lane + d) & 31), pt = __shfl_sync(FULL, t, (lane + d) & 31);
        const T* al = nullptr;
        (void)al;
        const T nh = h + wl<T>(W.alpha[s], W.alphaf[s], 0) * mh + wl<T>(W.alpha[s], W.alphaf[s], 1) * mt +
                     wl<T>(W.gamma[s], W.gammaf[s], 0) * ph + wl<T>(W.gamma[s], W.gammaf[s], 1) * pt;
        const T nt = t + wl<T>(W.alpha[s], W.alphaf[s], 2) * mh + wl<T>(W.alpha[s], W.alphaf[s], 3) * mt +
                     wl<T>(W.gamma[s], W.gammaf[s], 2) * ph + wl<T>(W.gamma[s], W.gammaf[s], 3) * pt;
        h = nh;
        t = nt;
    }
    {
        const T oh = __shfl_sync(FULL, h, (lane + 16) & 31), ot = __shfl_sync(FULL, t, (lane + 16) & 31);
        const T rh = h + wl<T>(W.alpha_f, W.alpha_ff, 0) * oh + wl<T>(W.alpha_f, W.alpha_ff, 1) * ot;
        const T rt = t + wl<T>(W.alpha_f, W.alpha_ff, 2) * oh + wl<T>(W.alpha_f, W.alpha_ff, 3) * ot;
        h = wl<T>(W.binv_f, W.binv_ff, 0) * rh + wl<T>(W.binv_f, W.binv_ff, 1) * rt;
        t = wl<T>(W.binv_f, W.binv_ff, 2) * rh + wl<T>(W.binv_f, W.binv_ff, 3) * rt;
    }
    const T tprev = __shfl_sync(FULL, t, lm);
    const T hnext = __shfl_sync(FULL, h, lp);
#pragma unroll
    for (int i = 0; i < XP; ++i) y[i] -= wl<T>(W.v, W.vf, i) * tprev + wl<T>(W.w, W.wf, i) * hnext;
    // store
#pragma unroll
    for (int q = 0; q < XP / VW; ++q) {
        V v;
        T* pv = reinterpret_cast<T*>(&v);
        if (mode == OUT_SUBTRACT) {
            const V o = *(reinterpret_cast<const V*>(dst) + q);
            const T* po = reinterpret_cast<const T*>(&o);
#pragma unroll
            for (int e = 0; e < VW; ++e) pv[e] = po[e] - y[q * VW + e];
        } else if (mode == OUT_NEGATE) {
#pragma unroll
            for (int e = 0; e < VW; ++e) pv[e] = -y[q * VW + e];
        } else {
#pragma unroll
            for (int e = 0; e < VW; ++e) pv[e] = y[q * VW + e];
        }
        reinterpret_cast<V*>(dst)[q] = v;
    }
}

template <typename T, int M>
void launch_xw_m(const CompactPlan& plan, const FieldView& in, const FieldView& out, int count, int mode,
                 cudaStream_t st) {
    const int lines_per_cta = 8;
    dim3 grid((unsigned)((plan.P.lines + lines_per_cta - 1) / lines_per_cta), (unsigned)count);
    switch (plan.XW.XP) {
        case 2:
            // the stencil halo comes from the neighbouring lanes' XP points: XP >= M
            if constexpr (M <= 2) k_compact_xw<T, M, 2><<<grid, 32 * lines_per_cta, 0, st>>>(plan.P, plan.XW, in, out, mode);
            else throw Error(CLES_EINVAL, "warp-line kernel: fewer points per lane than the stencil half-width");
            break;
        case 4: k_compact_xw<T, M, 4><<<grid, 32 * lines_per_cta, 0, st>>>(plan.P, plan.XW, in, out, mode); break;
        case 6: k_compact_xw<T, M, 6><<<grid, 32 * lines_per_cta, 0, st>>>(plan.P, plan.XW, in, out, mode); break;
        case 8: k_compact_xw<T, M, 8><<<grid, 32 * lines_per_cta, 0, st>>>(plan.P, plan.XW, in, out, mode); break;
        case 12: k_compact_xw<T, M, 12><<<grid, 32 * lines_per_cta, 0, st>>>(plan.P, plan.XW, in, out, mode); break;
        case 16: k_compact_xw<T, M, 16><<<grid, 32 * lines_per_cta, 0, st>>>(plan.P, plan.XW, in, out, mode); break;
        default: throw Error(CLES_EINVAL, "warp-line kernel: unsupported points per lane");
    }
    count_launch();
    check_launch("k_compact_xw");
}

template <typename T>
bool try_launch_xw(const CompactPlan& plan, const FieldView& in, const FieldView& out, int count, int mode,
                   cudaStream_t st) {
    if (!plan.has_xw) return false;
    // vector accesses need 16-byte aligned rows
    const size_t el = sizeof(T);
    auto aligned = [&](const FieldView& v) {
        return ((uintptr_t)v.base % 16 == 0) && ((v.sy * el) % 16 == 0) && ((v.sz * el) % 16 == 0) &&
               ((v.comp_stride * el) % 16 == 0 || count == 1);
    };
    if (!aligned(in) || !aligned(out)) return false;
    switch (plan.P.M) {
        case 1: launch_xw_m<T, 1>(plan, in, out, count, mode, st); return true;
        case 2: launch_xw_m<T, 2>(plan, in, out, count, mode, st); return true;
        case 4: launch_xw_m<T, 4>(plan, in, out, count, mode, st); return true;
        default: return false;
    }
}

template <typename T, int Q, int M, bool X, int MS>
void launch_t(const CompactParams& P, const T* tab, const FieldView& in, const FieldView& out, int count, int mode,
              cudaStream_t st, T* iface) {
    const int N = 2 * Q * P.S;
    size_t smem = 0;
    if (X) smem += sizeof(T) * (size_t)P.n * (P.LB + 1);
    if (P.pcr) smem += sizeof(T) * (size_t)P.LB * 4 * P.S;
    else if (P.hasred) smem += sizeof(T) * (size_t)P.LB * (N + 1);
    auto kern = k_compact<T, Q, M, X, MS>;
    static thread_local int configured = 0;
    if (smem > 48 * 1024 && configured < (int)smem) {
        CLES_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        configured = (int)smem;
    }
    dim3 grid((unsigned)((P.lines + P.LB - 1) / P.LB), (unsigned)count);
    dim3 block((unsigned)(P.LB * P.S));
    kern<<<grid, block, smem, st>>>(P, tab, in, out, mode, iface);
    count_launch();
    check_launch("k_compact");
}

template <typename T, int Q, bool X>
void dispatch_m(const CompactParams& P, const T* tab, const FieldView& in, const FieldView& out, int count, int mode,
                cudaStream_t st, T* iface) {
    // shorter register tiles for the short segments of few-line closed plans
    const int mmax = P.seg_base + (P.seg_rem ? 1 : 0);
    if constexpr (Q == 1) {
      if (mmax <= 16 && P.M != 3) {
        const bool eight = mmax <= 8;
        switch (P.M) {
            case 1: eight ? launch_t<T, Q, 1, X, 8>(P, tab, in, out, count, mode, st, iface)
                          : launch_t<T, Q, 1, X, 16>(P, tab, in, out, count, mode, st, iface); return;
            case 2: eight ? launch_t<T, Q, 2, X, 8>(P, tab, in, out, count, mode, st, iface)
                          : launch_t<T, Q, 2, X, 16>(P, tab, in, out, count, mode, st, iface); return;
            default: eight ? launch_t<T, Q, 4, X, 8>(P, tab, in, out, count, mode, st, iface)
                           : launch_t<T, Q, 4, X, 16>(P, tab, in, out, count, mode, st, iface); return;
        }
      }
    }
    switch (P.M) {
        case 1: launch_t<T, Q, 1, X, kMaxSeg>(P, tab, in, out, count, mode, st, iface); break;
        case 2: launch_t<T, Q, 2, X, kMaxSeg>(P, tab, in, out, count, mode, st, iface); break;
        case 3: launch_t<T, Q, 3, X, kMaxSeg>(P, tab, in, out, count, mode, st, iface); break;
        case 4: launch_t<T, Q, 4, X, kMaxSeg>(P, tab, in, out, count, mode, st, iface); break;
        default: throw Error(CLES_EINVAL, "unsupported stencil half-width");
    }
}

template <typename T>
void dispatch(const CompactParams& P, const T* tab, const FieldView& in, const FieldView& out, int count, int mode,
              cudaStream_t st, T* iface = nullptr) {
    const bool X = P.dim == 0;
    if (P.q == 1) {
        if (X) dispatch_m<T, 1, true>(P, tab, in, out, count, mode, st, iface);
        else dispatch_m<T, 1, false>(P, tab, in, out, count, mode, st, iface);
    } else {
        if (X) dispatch_m<T, 2, true>(P, tab, in, out, count, mode, st, iface);
        else dispatch_m<T, 2, false>(P, tab, in, out, count, mode, st, iface);
    }
}

}  // namespace

void launch_compact(const CompactPlan& plan, const FieldView& in, const FieldView& out, int count, int mode,
                    cudaStream_t st) {
    if (count <= 0 || plan.P.lines == 0) return;
    int rec = -1;
    if (profiling()) {
        const double el = plan.dtype == CLES_F64 ? 8.0 : 4.0;
        const double pts = (double)plan.P.lines * plan.P.n * count;
        rec = prof_begin(st, plan.P.dim, pts * el * (mode == OUT_SUBTRACT ? 3.0 : 2.0));
    }
    if (plan.dtype == CLES_F64) {
        if (!try_launch_xw<double>(plan, in, out, count, mode, st) && !try_launch_xt(plan, in, out, count, mode, st) &&
            !try_launch_tma(plan, in, out, count, mode, st))
            dispatch<double>(plan.P, plan.tab64, in, out, count, mode, st);
    } else {
        if (!try_launch_xw<float>(plan, in, out, count, mode, st) && !try_launch_xt(plan, in, out, count, mode, st) &&
            !try_launch_tma(plan, in, out, count, mode, st))
            dispatch<float>(plan.P, plan.tab32, in, out, count, mode, st);
    }
    if (rec >= 0) prof_end(rec, st);
}

void launch_compact_split(const CompactPlan& plan, const FieldView& in, const FieldView& out, int count, void* iface,
                          cudaStream_t st) {
    if (count <= 0 || plan.P.lines == 0) return;
    if (try_launch_tg_split(plan, in, out, count, iface, st)) return;
    if (plan.dtype == CLES_F64)
        dispatch<double>(plan.P, plan.tab64, in, out, count, OUT_STORE, st, static_cast<double*>(iface));
    else
        dispatch<float>(plan.P, plan.tab32, in, out, count, OUT_STORE, st, static_cast<float*>(iface));
}

}  // namespace cles
