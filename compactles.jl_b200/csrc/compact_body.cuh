// Device body of the generic compact line solve, shared by the one-grid
// launches (compact.cu) and the batched launches over many grids (batch.cu).
// See compact.cu for the algorithm.
#pragma once

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

// Low-storage RK update of one stored value, element e of the state: with
// dq = out - D(f), v = A du + dt dq; du = v; Q += B v (src/timestep.jl:86-95).
struct RkStore {
    double* Q;
    double* du;
    double A, B, dt;
    int64_t e0;   // element offset of the output's row base within the state
};
__device__ __forceinline__ void rk_store(const RkStore& r, int64_t e, double dq) {
    const double v = r.A * r.du[e] + r.dt * dq;
    r.du[e] = v;
    r.Q[e] += r.B * v;
}

// Cooperative copy between the CTA's x lines (contiguous rows in global
// memory) and the transposed tile: up to 32 threads per row, coalesced.
// OUT_RK (batched solves only) applies the RK update instead of storing.
template <typename T, bool LOAD, bool RK = false>
__device__ __forceinline__ void tile_rows(const CompactParams& P, const FieldView& v, T* g_field, T* tile, int line0,
                                          int nl, int n, int TP, int mode, const RkStore* rk = nullptr) {
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
                    else if (RK && mode == OUT_RK) rk_store(*rk, rk->e0 + Ll.base + g, double(row[g] - val));
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
                else if (RK && mode == OUT_RK) rk_store(*rk, rk->e0 + Ll.base + g, double(row[g] - val));
                else row[g] = row[g] - val;
            }
        }
    }
}

// The line solve of one CTA: lines [line0, line0 + LB) of component `comp`.
// RK (batched solves): mode OUT_RK applies the RK update of the state in rk
// instead of a store, and the interface inverse is staged in shared memory.
template <typename T, int Q, int M, bool XMODE, int MS, bool RK = false>
__device__ __forceinline__ void compact_lines(const CompactParams& P, const T* __restrict__ tab, const FieldView& in,
                                              const FieldView& out, const int mode, T* __restrict__ iface,
                                              const int line0, const int comp, const RkStore* rk,
                                              unsigned char* smem_raw) {
    T* smem = reinterpret_cast<T*>(smem_raw);
    const int LB = P.LB, S = P.S, n = P.n;
    const int lane = threadIdx.x % LB;
    const int seg = threadIdx.x / LB;
    const int line = line0 + lane;
    const bool valid = line < P.lines;
    const T* __restrict__ fin = reinterpret_cast<const T*>(in.base) + (int64_t)comp * in.comp_stride;
    T* __restrict__ fout = reinterpret_cast<T*>(out.base) + (int64_t)comp * out.comp_stride;
    const int off = seg * P.seg_base + min(seg, P.seg_rem);
    const int m = P.seg_base + (seg < P.seg_rem ? 1 : 0);
    const bool periodic = P.periodic != 0;
    const int TP = LB + 1;  // tile pitch (x lines)
    T* tile = smem;
    T* red = XMODE ? smem + (size_t)n * TP : smem;
    // batched launches stage the dense inverse of the interface system in
    // shared memory (row pitch N + 1, so segments of one warp hit different
    // banks) instead of reading it from global memory per thread
    T* Gsm = nullptr;
    if constexpr (RK) {
        if (P.hasred && !(Q == 1 && P.pcr)) {
            const int Nq = 2 * Q * S;
            Gsm = red + (size_t)LB * (Nq + 1);
            for (int i = threadIdx.x; i < Nq * Nq; i += blockDim.x)
                Gsm[(i / Nq) * (Nq + 1) + i % Nq] = tab[P.off_G + i];
        }
    }
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
        // closure row jr sits at i = m - 1 - jr; written as selects over every
        // element (static indices keep y in registers)
        T hv[kMaxClo];
#pragma unroll
        for (int jr = 0; jr < kMaxClo; ++jr) {
            T acc = T(0);
            if (jr < P.nc)
                for (int k = 0; k < P.clo_len[jr]; ++k) acc += T(P.chi[jr][k]) * ld(n - 1 - k);
            hv[jr] = acc;
        }
#pragma unroll
        for (int i = 0; i < MS; ++i)
#pragma unroll
            for (int jr = 0; jr < kMaxClo; ++jr) y[i] = (jr < P.nc && i == m - 1 - jr) ? hv[jr] : y[i];
    }

    // ---- 3. local solve -----------------------------------------------------
    const T* f0 = tab + P.off_f0 + (int64_t)seg * kMaxSeg;
    const T* f1 = tab + P.off_f1 + (int64_t)seg * kMaxSeg;
    const T* f2 = tab + P.off_f2 + (int64_t)seg * kMaxSeg;
    if (Q == 1) {
#pragma unroll
        for (int i = 1; i < MS; ++i)
            if (i < m) y[i] -= ldg(f0 + i) * y[i - 1];
        {
            // the last row's pivot, as a select over every element: a branch
            // taken for one i would be folded into a dynamic index of y and
            // move y to local memory
            const T dl = ldg(f1 + (m - 1));
#pragma unroll
            for (int i = 0; i < MS; ++i) y[i] = (i == m - 1) ? y[i] * dl : y[i];
        }
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
        for (int i = 0; i < MS; ++i) tail = (i == m - 1) ? y[i] : tail;
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
        {
            // heads y[0..Q), tails y[m-Q..m) by a window sliding over y while
            // i < m (static indices, so y stays in registers)
            T tl[Q];
#pragma unroll
            for (int t = 0; t < Q; ++t) { rl[2 * Q * seg + t] = y[t]; tl[t] = T(0); }
#pragma unroll
            for (int i = 0; i < MS; ++i) {
                const bool in = i < m;
#pragma unroll
                for (int t = 0; t < Q - 1; ++t) tl[t] = in ? tl[t + 1] : tl[t];
                tl[Q - 1] = in ? y[i] : tl[Q - 1];
            }
#pragma unroll
            for (int t = 0; t < Q; ++t) rl[2 * Q * seg + Q + t] = tl[t];
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
                T acc = T(0);
                if (RK && Gsm) {
                    const T* g = Gsm + (int64_t)(2 * Q * prev + Q + t) * (N + 1);
                    for (int j = 0; j < N; ++j) acc += g[j] * rl[j];
                } else {
                    const T* g = G + (int64_t)(2 * Q * prev + Q + t) * N;
                    for (int j = 0; j < N; ++j) acc += ldg(g + j) * rl[j];
                }
                zp[t] = acc;
            }
        }
        if (has_next) {
#pragma unroll
            for (int t = 0; t < Q; ++t) {
                T acc = T(0);
                if (RK && Gsm) {
                    const T* g = Gsm + (int64_t)(2 * Q * next + t) * (N + 1);
                    for (int j = 0; j < N; ++j) acc += g[j] * rl[j];
                } else {
                    const T* g = G + (int64_t)(2 * Q * next + t) * N;
                    for (int j = 0; j < N; ++j) acc += ldg(g + j) * rl[j];
                }
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
            T tl[Q];
#pragma unroll
            for (int t = 0; t < Q; ++t) tl[t] = T(0);
#pragma unroll
            for (int i = 0; i < MS; ++i) {
                const bool in = i < m;
#pragma unroll
                for (int t = 0; t < Q - 1; ++t) tl[t] = in ? tl[t + 1] : tl[t];
                tl[Q - 1] = in ? y[i] : tl[Q - 1];
            }
#pragma unroll
            for (int t = 0; t < Q; ++t) ifc[(int64_t)(Q + t) * P.lines] = tl[t];
        }
    }
    if (XMODE) {
        __syncthreads();  // every window/closure read of the tile is done
#pragma unroll
        for (int i = 0; i < MS; ++i)
            if (i < m) tile[(off + i) * TP + lane] = y[i];
        __syncthreads();
        tile_rows<T, false, RK>(P, out, fout, tile, line0, nl, n, TP, mode, rk);
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
                else if (RK && mode == OUT_RK)
                    rk_store(*rk, rk->e0 + Lout.base + (int64_t)(off + i) * Lout.stride, double(*o - y[i]));
                else *o = *o - y[i];
            }
        }
    }
}

}  // namespace
}  // namespace cles
