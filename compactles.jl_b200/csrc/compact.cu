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

#include "cles_internal.h"

namespace cles {

namespace {

template <typename T>
__device__ __forceinline__ T ldg(const T* p) { return __ldg(p); }

struct LineMap {
    int64_t base;      // element offset of line element 0 (without component offset)
    int64_t stride;    // element stride along the line
};

__device__ __forceinline__ LineMap line_map(const CompactParams& P, const FieldView& v, int line) {
    // lines < 2^31 (checked at plan time), so 32-bit division suffices
    LineMap L;
    if (P.dim == 0) {
        const int j = line % P.ny, k = line / P.ny;
        L.base = j * v.sy + k * v.sz;
        L.stride = 1;
    } else if (P.dim == 1) {
        const int i = line % P.nx, k = line / P.nx;
        L.base = i + k * v.sz;
        L.stride = v.sy;
    } else {
        const int i = line % P.nx, j = line / P.nx;
        L.base = i + j * v.sy;
        L.stride = v.sz;
    }
    return L;
}

// g in [-n, 2n): periodic wrap without a division; closed lines clamp (the
// clamped values are never used by a closure row); an open end keeps g, whose
// element lies in the caller's halo (g >= -M, g < n + M).
__device__ __forceinline__ int wrap_index(int g, int n, bool periodic, bool lo_open = false, bool hi_open = false) {
    if (periodic) return g < 0 ? g + n : (g >= n ? g - n : g);
    return g < 0 ? (lo_open ? g : 0) : (g >= n ? (hi_open ? g : n - 1) : g);
}

// Cooperative copy between the CTA's x lines (contiguous rows in global
// memory) and the transposed tile: up to 32 threads per row, coalesced.
template <typename T, bool LOAD>
__device__ __forceinline__ void tile_rows(const CompactParams& P, const FieldView& v, T* g_field, T* tile, int line0,
                                          int nl, int n, int TP, int mode) {
    const int nt = blockDim.x;
    if (nl * 32 <= nt) {
        // few rows (long lines, few per CTA): the whole block strides each row
        for (int l = 0; l < nl; ++l) {
            const LineMap Ll = line_map(P, v, line0 + l);
            T* row = g_field + Ll.base;
            for (int g = threadIdx.x; g < n; g += nt) {
                if (LOAD) {
                    tile[g * TP + l] = row[g];
                } else {
                    const T val = tile[g * TP + l];
                    if (mode == OUT_STORE) row[g] = val;
                    else if (mode == OUT_NEGATE) row[g] = -val;
                    else row[g] = row[g] - val;
                }
            }
        }
        return;
    }
    const int tpr = nt < 32 ? nt : 32;
    const int rows_per_pass = nt / tpr;
    const int r = threadIdx.x / tpr, c = threadIdx.x - (threadIdx.x / tpr) * tpr;
    if (r >= rows_per_pass) return;
    for (int l = r; l < nl; l += rows_per_pass) {
        const LineMap Ll = line_map(P, v, line0 + l);
        T* row = g_field + Ll.base;
        if (LOAD) {
            for (int g = c; g < n; g += tpr) tile[g * TP + l] = row[g];
        } else {
            for (int g = c; g < n; g += tpr) {
                const T val = tile[g * TP + l];
                if (mode == OUT_STORE) row[g] = val;
                else if (mode == OUT_NEGATE) row[g] = -val;
                else row[g] = row[g] - val;
            }
        }
    }
}

template <typename T, int Q, int M, bool XMODE, int MS>
__global__ void __launch_bounds__(512) k_compact(const __grid_constant__ CompactParams P, const T* __restrict__ tab,
                                                  const FieldView in, const FieldView out, const int mode,
                                                  T* __restrict__ iface) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* smem = reinterpret_cast<T*>(smem_raw);
    const int LB = P.LB, S = P.S, n = P.n;
    const int lane = threadIdx.x % LB;
    const int seg = threadIdx.x / LB;
    const int line0 = blockIdx.x * LB;
    const int line = line0 + lane;
    const bool valid = line < P.lines;
    const int comp = blockIdx.y;
    const T* __restrict__ fin = reinterpret_cast<const T*>(in.base) + (int64_t)comp * in.comp_stride;
    T* __restrict__ fout = reinterpret_cast<T*>(out.base) + (int64_t)comp * out.comp_stride;
    const int off = seg * P.seg_base + min(seg, P.seg_rem);
    const int m = P.seg_base + (seg < P.seg_rem ? 1 : 0);
    const bool periodic = P.periodic != 0;
    const int TP = LB + 1;  // tile pitch (x lines)
    T* tile = smem;
    T* red = XMODE ? smem + (size_t)n * TP : smem;
    const int N = 2 * Q * S;

    LineMap Lin = line_map(P, in, valid ? line : line0);
    LineMap Lout = line_map(P, out, valid ? line : line0);

    // ---- 1. gather --------------------------------------------------------
    const int nl = (int)((int64_t)LB < P.lines - line0 ? (int64_t)LB : P.lines - line0);
    if (XMODE) {
        tile_rows<T, true>(P, in, const_cast<T*>(fin), tile, line0, nl, n, TP, 0);
        __syncthreads();
    }
    constexpr int WN = MS + 2 * M;
    T w[WN];
#pragma unroll
    for (int j = 0; j < WN; ++j) {
        if (j < m + 2 * M) {
            const int g = wrap_index(off - M + j, n, periodic, P.lo_open, P.hi_open);
            if (XMODE && g >= 0 && g < n) w[j] = tile[g * TP + lane];
            else w[j] = valid ? fin[Lin.base + (int64_t)g * Lin.stride] : T(0);
        } else {
            w[j] = T(0);
        }
    }
    auto ld = [&](int g) -> T {
        if (XMODE) return tile[g * TP + lane];
        return valid ? fin[Lin.base + (int64_t)g * Lin.stride] : T(0);
    };

    // ---- 2. fill -----------------------------------------------------------
    T y[MS];
    const T a0 = T(P.a0);
    T ci[M];
#pragma unroll
    for (int k = 0; k < M; ++k) ci[k] = T(P.ci[k]);
#pragma unroll
    for (int i = 0; i < MS; ++i) {
        if (i < m) {
            T acc;
            if (P.symmetric) {
                acc = a0 * w[i + M];
#pragma unroll
                for (int k = 1; k <= M; ++k) acc += ci[k - 1] * (w[i + M + k] + w[i + M - k]);
            } else {
                acc = T(0);
#pragma unroll
                for (int k = 1; k <= M; ++k) acc += ci[k - 1] * (w[i + M + k] - w[i + M - k]);
            }
            y[i] = acc;
        } else {
            y[i] = T(0);
        }
    }
    if (P.lo_closed && seg == 0) {
#pragma unroll
        for (int i = 0; i < kMaxClo; ++i) {
            if (i < P.nc) {
                T acc = T(0);
                for (int k = 0; k < P.clo_len[i]; ++k) acc += T(P.clo[i][k]) * ld(k);
                y[i] = acc;
            }
        }
    }
    if (P.hi_closed && seg == S - 1) {
#pragma unroll
        for (int i = 0; i < MS; ++i) {
            if (i < m && i >= m - P.nc) {
                const int jr = m - 1 - i;
                T acc = T(0);
                for (int k = 0; k < P.clo_len[jr]; ++k) acc += T(P.chi[jr][k]) * ld(n - 1 - k);
                y[i] = acc;
            }
        }
    }

    // ---- 3. local solve -----------------------------------------------------
    const T* f0 = tab + P.off_f0 + (int64_t)seg * kMaxSeg;
    const T* f1 = tab + P.off_f1 + (int64_t)seg * kMaxSeg;
    const T* f2 = tab + P.off_f2 + (int64_t)seg * kMaxSeg;
    if (Q == 1) {
#pragma unroll
        for (int i = 1; i < MS; ++i)
            if (i < m) y[i] -= ldg(f0 + i) * y[i - 1];
#pragma unroll
        for (int i = 0; i < MS; ++i)
            if (i == m - 1) y[i] *= ldg(f1 + i);
#pragma unroll
        for (int i = MS - 2; i >= 0; --i)
            if (i < m - 1) y[i] = (y[i] - ldg(f2 + i) * y[i + 1]) * ldg(f1 + i);
    } else {
        const T* f3 = tab + P.off_f3 + (int64_t)seg * kMaxSeg;
        const T* f4 = tab + P.off_f4 + (int64_t)seg * kMaxSeg;
#pragma unroll
        for (int k = 0; k < MS - 1; ++k) {
            if (k < m - 1) y[k + 1] -= ldg(f0 + k) * y[k];
            if (k + 2 < MS && k < m - 2) y[k + 2] -= ldg(f1 + k) * y[k];
        }
#pragma unroll
        for (int i = MS - 1; i >= 0; --i) {
            if (i < m) {
                T acc = y[i];
                if (i + 1 < MS && i + 1 < m) acc -= ldg(f2 + i) * y[i + 1];
                if (i + 2 < MS && i + 2 < m) acc -= ldg(f3 + i) * y[i + 2];
                y[i] = acc * ldg(f4 + i);
            }
        }
    }

    // ---- 4. interface solve -----------------------------------------------
    if (Q == 1 && P.pcr) {
        // closed tridiagonal line: block cyclic reduction of the interface
        // system in X_s = (head_s, tail_s) with precomputed 2x2 blocks,
        // double-buffered in shared memory (4 S values per line)
        T tail = T(0);
#pragma unroll
        for (int i = 0; i < MS; ++i)
            if (i == m - 1) tail = y[i];
        T* cur = red + (size_t)lane * 4 * S;
        T* nxt = cur + 2 * S;
        cur[2 * seg] = y[0];
        cur[2 * seg + 1] = tail;
        __syncthreads();
        const T* pc = tab + P.off_pcr + (int64_t)seg * 8;
        for (int l = 0; l < P.pcr_levels; ++l) {
            const int k = 1 << l;
            const T* c = pc + (int64_t)l * S * 8;
            T r0 = cur[2 * seg], r1 = cur[2 * seg + 1];
            if (seg - k >= 0) {
                const T p0 = cur[2 * (seg - k)], p1 = cur[2 * (seg - k) + 1];
                r0 += ldg(c + 0) * p0 + ldg(c + 1) * p1;
                r1 += ldg(c + 2) * p0 + ldg(c + 3) * p1;
            }
            if (seg + k < S) {
                const T p0 = cur[2 * (seg + k)], p1 = cur[2 * (seg + k) + 1];
                r0 += ldg(c + 4) * p0 + ldg(c + 5) * p1;
                r1 += ldg(c + 6) * p0 + ldg(c + 7) * p1;
            }
            nxt[2 * seg] = r0;
            nxt[2 * seg + 1] = r1;
            __syncthreads();
            T* t = cur; cur = nxt; nxt = t;
        }
        {
            // nxt was last read before the final barrier: it takes the solution
            const T* bi = pc + (int64_t)P.pcr_levels * S * 8;
            const T r0 = cur[2 * seg], r1 = cur[2 * seg + 1];
            nxt[2 * seg] = ldg(bi + 0) * r0 + ldg(bi + 1) * r1;
            nxt[2 * seg + 1] = ldg(bi + 2) * r0 + ldg(bi + 3) * r1;
        }
        __syncthreads();
        const T zp = seg > 0 ? nxt[2 * (seg - 1) + 1] : T(0);      // tail of the previous segment
        const T zn = seg < S - 1 ? nxt[2 * (seg + 1)] : T(0);      // head of the next segment
        const T* V = tab + P.off_V + (int64_t)seg * kMaxSeg;
        const T* W = tab + P.off_W + (int64_t)seg * kMaxSeg;
#pragma unroll
        for (int i = 0; i < MS; ++i)
            if (i < m) y[i] -= ldg(V + i) * zp + ldg(W + i) * zn;
    } else if (P.hasred) {
        const int RP = N + 1;  // pitch of the per-line interface vector
        T* rl = red + (size_t)lane * RP;
#pragma unroll
        for (int i = 0; i < MS; ++i) {
            if (i < Q) rl[2 * Q * seg + i] = y[i];
            if (i < m && i >= m - Q) rl[2 * Q * seg + Q + (i - (m - Q))] = y[i];
        }
        __syncthreads();
        T zp[Q], zn[Q];
#pragma unroll
        for (int t = 0; t < Q; ++t) { zp[t] = T(0); zn[t] = T(0); }
        const bool has_prev = periodic || seg > 0;
        const bool has_next = periodic || seg < S - 1;
        const int prev = seg == 0 ? S - 1 : seg - 1;
        const int next = seg == S - 1 ? 0 : seg + 1;
        const T* G = tab + P.off_G;
        if (has_prev) {
#pragma unroll
            for (int t = 0; t < Q; ++t) {
                const T* g = G + (int64_t)(2 * Q * prev + Q + t) * N;
                T acc = T(0);
                for (int j = 0; j < N; ++j) acc += ldg(g + j) * rl[j];
                zp[t] = acc;
            }
        }
        if (has_next) {
#pragma unroll
            for (int t = 0; t < Q; ++t) {
                const T* g = G + (int64_t)(2 * Q * next + t) * N;
                T acc = T(0);
                for (int j = 0; j < N; ++j) acc += ldg(g + j) * rl[j];
                zn[t] = acc;
            }
        }
        const T* V = tab + P.off_V + (int64_t)seg * Q * kMaxSeg;
        const T* W = tab + P.off_W + (int64_t)seg * Q * kMaxSeg;
#pragma unroll
        for (int i = 0; i < MS; ++i) {
            if (i < m) {
                T acc = T(0);
#pragma unroll
                for (int t = 0; t < Q; ++t) acc += ldg(V + t * kMaxSeg + i) * zp[t] + ldg(W + t * kMaxSeg + i) * zn[t];
                y[i] -= acc;
            }
        }
    }

    // ---- 5. store ------------------------------------------------------------
    if (iface && valid) {
        // local solution's head and tail of a split line: [comp][2q][lines]
        T* ifc = iface + (int64_t)comp * 2 * Q * P.lines + line;
        if (seg == 0) {
#pragma unroll
            for (int t = 0; t < Q; ++t) ifc[(int64_t)t * P.lines] = y[t];
        }
        if (seg == S - 1) {
#pragma unroll
            for (int i = 0; i < MS; ++i)
                if (i < m && i >= m - Q) ifc[(int64_t)(Q + i - (m - Q)) * P.lines] = y[i];
        }
    }
    if (XMODE) {
        __syncthreads();  // every window/closure read of the tile is done
#pragma unroll
        for (int i = 0; i < MS; ++i)
            if (i < m) tile[(off + i) * TP + lane] = y[i];
        __syncthreads();
        tile_rows<T, false>(P, out, fout, tile, line0, nl, n, TP, mode);
    } else {
        // In place (out == in) is safe: with S > 1 the interface barrier
        // separates every window read of a line from its stores, with S = 1 a
        // line belongs to one thread, and different CTAs own disjoint lines.
        if (!valid) return;
#pragma unroll
        for (int i = 0; i < MS; ++i) {
            if (i < m) {
                T* o = fout + Lout.base + (int64_t)(off + i) * Lout.stride;
                if (mode == OUT_STORE) *o = y[i];
                else if (mode == OUT_NEGATE) *o = -y[i];
                else *o = *o - y[i];
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Warp-per-line kernel for periodic tridiagonal x lines of n = 32 * XP points.
// Lane s of a warp owns the XP contiguous points [s*XP, (s+1)*XP) of one line:
// vector loads and stores straight from/to global memory (the warp covers the
// whole contiguous line), stencil halos from the neighbouring lanes by shuffle,
// the lane's Thomas sweep in registers, and the 32-segment interface system by
// parallel cyclic reduction across the lanes with precomputed 2x2 matrices.
template <typename T> struct Vec;
template <> struct Vec<double> { using type = double2; static constexpr int W = 2; };
template <> struct Vec<float> { using type = float4; static constexpr int W = 4; };

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
    using V = typename Vec<T>::type;
    constexpr int VW = Vec<T>::W;
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
        case 4: k_compact_xw<T, M, 4><<<grid, 32 * lines_per_cta, 0, st>>>(plan.P, plan.XW, in, out, mode); break;
        case 8: k_compact_xw<T, M, 8><<<grid, 32 * lines_per_cta, 0, st>>>(plan.P, plan.XW, in, out, mode); break;
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
