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

#include <algorithm>
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
// Few long closed x lines cut into pieces (SigPlan).  k_compact_pieces: the
// CTAs of the three piece classes in one launch (blockIdx.x picks the class),
// each the segmented solve of its pieces with open ends reading the
// neighbouring pieces' points, local solutions to `loc`, heads and tails to
// the class's iface block.  k_sig_correct: per (piece, line, field) the 2q
// unknowns beside the piece from the dense inverse of the piece-interface
// system, then x = y - V z_prev - W z_next into `out` by mode.
struct SigLocal {
    FieldView in[3], loc[3];
    void* iface[3];
    int nblk[3];
};

template <typename T, int Q, int M, int MS>
__global__ void __launch_bounds__(512) k_compact_pieces(const __grid_constant__ CompactParams P0,
                                                         const __grid_constant__ CompactParams P1,
                                                         const __grid_constant__ CompactParams P2,
                                                         const T* __restrict__ tab0, const T* __restrict__ tab1,
                                                         const T* __restrict__ tab2, const __grid_constant__ SigLocal L) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    int b = blockIdx.x, c = 0;
    if (b >= L.nblk[0]) {
        b -= L.nblk[0];
        c = 1;
        if (b >= L.nblk[1]) {
            b -= L.nblk[1];
            c = 2;
        }
    }
    const CompactParams& P = c == 0 ? P0 : (c == 1 ? P1 : P2);
    const T* tab = c == 0 ? tab0 : (c == 1 ? tab1 : tab2);
    compact_lines<T, Q, M, true, MS>(P, tab, L.in[c], L.loc[c], OUT_STORE, static_cast<T*>(L.iface[c]), b * P.LB,
                                     blockIdx.y, nullptr, smem_raw);
}

struct SigCorrect {
    const void* iface[3];
    int64_t lines_c[3];
    const void* tab;
    int64_t off_V[3], off_W[3], off_G;
    FieldView loc, out;            // element (g, line) of field c: base + c comp_stride + line offset + g
    int len[3];
    int P, ny;                     // pieces; the plan's ny (line l: j = l % ny, k = l / ny)
};

constexpr int kSigPts = 4;   // points per thread of the correction (pieces of at most 1024 points)
template <typename T, int Q, int MODE>
__global__ void __launch_bounds__(256) k_sig_correct(const __grid_constant__ SigCorrect C) {
    __shared__ T h[2 * Q * 64];
    __shared__ T grow[2 * Q][2 * Q * 64];
    __shared__ T z[2 * Q];
    const int k = blockIdx.x, P = C.P, N = 2 * Q * P;
    const int64_t l = blockIdx.y;
    const int comp = blockIdx.z;
    auto cls = [&](int kk) { return kk == 0 ? 0 : (kk == P - 1 ? 2 : 1); };
    const int c = cls(k), len = C.len[c];
    const int off = k == 0 ? 0 : C.len[0] + (k - 1) * C.len[1];
    const T* tab = static_cast<const T*>(C.tab);
    const T* V = tab + C.off_V[c];
    const T* W = tab + C.off_W[c];
    const int64_t jj = l % C.ny, kz = l / C.ny;
    const T* lp = static_cast<const T*>(C.loc.base) + (int64_t)comp * C.loc.comp_stride + jj * C.loc.sy +
                  kz * C.loc.sz + off;
    T* op = static_cast<T*>(C.out.base) + (int64_t)comp * C.out.comp_stride + jj * C.out.sy + kz * C.out.sz + off;
    // loads that do not wait for the interface unknowns, issued first
    T yv[kSigPts], vv[kSigPts][Q], wv[kSigPts][Q], ov[kSigPts];
#pragma unroll
    for (int e = 0; e < kSigPts; ++e) {
        const int i = threadIdx.x + e * blockDim.x;
        if (i < len) {
            yv[e] = lp[i];
#pragma unroll
            for (int t = 0; t < Q; ++t) {
                vv[e][t] = V[t * len + i];
                wv[e][t] = W[t * len + i];
            }
            if (MODE == OUT_SUBTRACT) ov[e] = op[i];
        }
    }
    // the 2q rows of the inverse this piece needs: prev tail rows, next head rows
    for (int j = threadIdx.x; j < 2 * Q * N; j += blockDim.x) {
        const int rr = j / N, col = j % N, t = rr % Q;
        const bool nxt = rr >= Q;
        const bool exists = nxt ? k + 1 < P : k > 0;
        const int row = nxt ? 2 * Q * (k + 1) + t : 2 * Q * (k - 1) + Q + t;
        grow[rr][col] = exists ? tab[C.off_G + (int64_t)row * N + col] : T(0);
    }
    for (int j = threadIdx.x; j < N; j += blockDim.x) {
        const int kk = j / (2 * Q), r = j % (2 * Q), cc = cls(kk);
        const int64_t lc = cc == 1 ? (int64_t)(kk - 1) + (int64_t)(P - 2) * l : l;
        h[j] = static_cast<const T*>(C.iface[cc])[((int64_t)comp * 2 * Q + r) * C.lines_c[cc] + lc];
    }
    __syncthreads();
    // z[0..q): previous piece's tail, z[q..2q): next piece's head; one warp each
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    if (warp < 2 * Q) {
        T acc = T(0);
        for (int j = lane; j < N; j += 32) acc += grow[warp][j] * h[j];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (lane == 0) z[warp] = acc;
    }
    __syncthreads();
#pragma unroll
    for (int e = 0; e < kSigPts; ++e) {
        const int i = threadIdx.x + e * blockDim.x;
        if (i < len) {
            T acc = T(0);
#pragma unroll
            for (int t = 0; t < Q; ++t) acc += vv[e][t] * z[t] + wv[e][t] * z[Q + t];
            const T r = yv[e] - acc;
            if (MODE == OUT_NEGATE) op[i] = -r;
            else if (MODE == OUT_SUBTRACT) op[i] = ov[e] - r;
            else op[i] = r;
        }
    }
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

template <typename T, int Q, int M, int MS>
void launch_pieces(const SigPlan& sp, const SigLocal& L, int count, cudaStream_t st) {
    size_t smem = 0;
    for (int c = 0; c < 3; ++c) {
        const CompactParams& P = sp.cls[c].P;
        const int N = 2 * Q * P.S;
        size_t s = sizeof(T) * (size_t)P.n * (P.LB + 1);
        if (P.hasred) s += sizeof(T) * (size_t)P.LB * (N + 1);
        smem = std::max(smem, s);
    }
    auto kern = k_compact_pieces<T, Q, M, MS>;
    if (smem > 48 * 1024) CLES_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const CompactParams& P0 = sp.cls[0].P;
    dim3 grid((unsigned)(L.nblk[0] + L.nblk[1] + L.nblk[2]), (unsigned)count);
    auto tb = [&](int c) -> const T* {
        return sizeof(T) == 8 ? reinterpret_cast<const T*>(sp.cls[c].tab64) : reinterpret_cast<const T*>(sp.cls[c].tab32);
    };
    kern<<<grid, (unsigned)(P0.LB * P0.S), smem, st>>>(sp.cls[0].P, sp.cls[1].P, sp.cls[2].P, tb(0), tb(1), tb(2), L);
    count_launch();
    check_launch("k_compact_pieces");
}

template <typename T, int Q>
void launch_sig_correct(const SigCorrect& C, int64_t lines, int count, int mode, cudaStream_t st) {
    dim3 grid((unsigned)C.P, (unsigned)lines, (unsigned)count);
    if (mode == OUT_NEGATE) k_sig_correct<T, Q, OUT_NEGATE><<<grid, 256, 0, st>>>(C);
    else if (mode == OUT_SUBTRACT) k_sig_correct<T, Q, OUT_SUBTRACT><<<grid, 256, 0, st>>>(C);
    else k_sig_correct<T, Q, OUT_STORE><<<grid, 256, 0, st>>>(C);
    count_launch();
    check_launch("k_sig_correct");
}

template <typename T>
void launch_sig(const CompactPlan& plan, const FieldView& in, const FieldView& out, int count, int mode,
                cudaStream_t st) {
    const SigPlan& sp = *plan.sig;
    if (mode != OUT_STORE && mode != OUT_NEGATE && mode != OUT_SUBTRACT)
        throw Error(CLES_EINVAL, "internal: pieced lines store, negate or subtract");
    const CompactParams& P = plan.P;
    const int n = P.n, Pp = sp.P, q = sp.q;
    const int64_t L = sp.lines;
    // the stride between lines of the plan (one of ny, nz is 1)
    const int64_t in_ls = P.ny > 1 ? in.sy : in.sz;
    for (int c0 = 0; c0 < count; c0 += kSigFields) {
        const int cc = std::min(kSigFields, count - c0);
        const T* ib = static_cast<const T*>(in.base) + (int64_t)c0 * in.comp_stride;
        T* ob = static_cast<T*>(out.base) + (int64_t)c0 * out.comp_stride;
        T* lb = static_cast<T*>(sp.loc);
        const int64_t lcs = L * n;   // loc: [field][line][n]
        SigLocal Lc;
        const int64_t off_c[3] = {0, sp.len[0], sp.len[0] + (int64_t)(Pp - 2) * sp.len[1]};
        for (int c = 0; c < 3; ++c) {
            const bool midc = c == 1;
            Lc.in[c] = FieldView{const_cast<T*>(ib) + off_c[c], in.comp_stride, midc ? (int64_t)sp.len[1] : in_ls,
                                 midc ? in_ls : 0};
            Lc.loc[c] = FieldView{lb + off_c[c], lcs, midc ? (int64_t)sp.len[1] : (int64_t)n, midc ? (int64_t)n : 0};
            Lc.iface[c] = sp.iface[c];
            const CompactParams& Pc = sp.cls[c].P;
            Lc.nblk[c] = (int)((Pc.lines + Pc.LB - 1) / Pc.LB);
        }
        if (q == 1) {
            switch (P.M) {
                case 1: launch_pieces<T, 1, 1, 16>(sp, Lc, cc, st); break;
                case 2: launch_pieces<T, 1, 2, 16>(sp, Lc, cc, st); break;
                case 4: launch_pieces<T, 1, 4, 16>(sp, Lc, cc, st); break;
                default: throw Error(CLES_EINVAL, "pieced lines: unsupported stencil half-width");
            }
        } else {
            if (P.M != 3) throw Error(CLES_EINVAL, "pieced lines: unsupported stencil half-width");
            launch_pieces<T, 2, 3, kMaxSeg>(sp, Lc, cc, st);
        }
        SigCorrect C;
        for (int c = 0; c < 3; ++c) {
            C.iface[c] = sp.iface[c];
            C.lines_c[c] = sp.cls[c].P.lines;
            C.off_V[c] = sp.off_V[c];
            C.off_W[c] = sp.off_W[c];
            C.len[c] = sp.len[c];
        }
        C.tab = sp.tab;
        C.off_G = sp.off_G;
        C.loc = FieldView{lb, lcs, P.ny > 1 ? (int64_t)n : 0, P.ny > 1 ? 0 : (int64_t)n};
        C.out = FieldView{ob, out.comp_stride, out.sy, out.sz};
        C.P = Pp;
        C.ny = P.ny;
        if (q == 1) launch_sig_correct<T, 1>(C, L, cc, mode, st);
        else launch_sig_correct<T, 2>(C, L, cc, mode, st);
    }
}

}  // namespace

void launch_compact(const CompactPlan& plan, const FieldView& in, const FieldView& out, int count, int mode,
                    cudaStream_t st) {
    if (count <= 0 || plan.P.lines == 0) return;
    if (plan.sig) {
        int rec = -1;
        if (profiling()) {
            const double el = plan.dtype == CLES_F64 ? 8.0 : 4.0;
            rec = prof_begin(st, plan.P.dim, (double)plan.P.lines * plan.P.n * count * el *
                                                 (mode == OUT_SUBTRACT ? 3.0 : 2.0));
        }
        if (plan.dtype == CLES_F64) launch_sig<double>(plan, in, out, count, mode, st);
        else launch_sig<float>(plan, in, out, count, mode, st);
        if (rec >= 0) prof_end(rec, st);
        return;
    }
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
