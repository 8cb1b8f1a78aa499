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
// the caller's arrays are never read.

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
// clamped values are never used by a closure row).
__device__ __forceinline__ int wrap_index(int g, int n, bool periodic) {
    if (periodic) return g < 0 ? g + n : (g >= n ? g - n : g);
    return g < 0 ? 0 : (g >= n ? n - 1 : g);
}

// Cooperative copy between the CTA's x lines (contiguous rows in global
// memory) and the transposed tile: up to 32 threads per row, coalesced.
template <typename T, bool LOAD>
__device__ __forceinline__ void tile_rows(const CompactParams& P, const FieldView& v, T* g_field, T* tile, int line0,
                                          int nl, int n, int TP, int mode) {
    const int nt = blockDim.x;
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

template <typename T, int Q, int M, bool XMODE>
__global__ void __launch_bounds__(512) k_compact(const CompactParams P, const T* __restrict__ tab, const FieldView in,
                                                  const FieldView out, const int mode) {
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
    constexpr int WN = kMaxSeg + 2 * M;
    T w[WN];
#pragma unroll
    for (int j = 0; j < WN; ++j) {
        if (j < m + 2 * M) {
            const int g = wrap_index(off - M + j, n, periodic);
            if (XMODE) w[j] = tile[g * TP + lane];
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
    T y[kMaxSeg];
    const T a0 = T(P.a0);
    T ci[M];
#pragma unroll
    for (int k = 0; k < M; ++k) ci[k] = T(P.ci[k]);
#pragma unroll
    for (int i = 0; i < kMaxSeg; ++i) {
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
        for (int i = 0; i < kMaxSeg; ++i) {
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
        for (int i = 1; i < kMaxSeg; ++i)
            if (i < m) y[i] -= ldg(f0 + i) * y[i - 1];
#pragma unroll
        for (int i = 0; i < kMaxSeg; ++i)
            if (i == m - 1) y[i] *= ldg(f1 + i);
#pragma unroll
        for (int i = kMaxSeg - 2; i >= 0; --i)
            if (i < m - 1) y[i] = (y[i] - ldg(f2 + i) * y[i + 1]) * ldg(f1 + i);
    } else {
        const T* f3 = tab + P.off_f3 + (int64_t)seg * kMaxSeg;
        const T* f4 = tab + P.off_f4 + (int64_t)seg * kMaxSeg;
#pragma unroll
        for (int k = 0; k < kMaxSeg - 1; ++k) {
            if (k < m - 1) y[k + 1] -= ldg(f0 + k) * y[k];
            if (k + 2 < kMaxSeg && k < m - 2) y[k + 2] -= ldg(f1 + k) * y[k];
        }
#pragma unroll
        for (int i = kMaxSeg - 1; i >= 0; --i) {
            if (i < m) {
                T acc = y[i];
                if (i + 1 < kMaxSeg && i + 1 < m) acc -= ldg(f2 + i) * y[i + 1];
                if (i + 2 < kMaxSeg && i + 2 < m) acc -= ldg(f3 + i) * y[i + 2];
                y[i] = acc * ldg(f4 + i);
            }
        }
    }

    // ---- 4. interface solve -----------------------------------------------
    if (P.hasred) {
        const int RP = N + 1;  // pitch of the per-line interface vector
        T* rl = red + (size_t)lane * RP;
#pragma unroll
        for (int i = 0; i < kMaxSeg; ++i) {
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
        for (int i = 0; i < kMaxSeg; ++i) {
            if (i < m) {
                T acc = T(0);
#pragma unroll
                for (int t = 0; t < Q; ++t) acc += ldg(V + t * kMaxSeg + i) * zp[t] + ldg(W + t * kMaxSeg + i) * zn[t];
                y[i] -= acc;
            }
        }
    }

    // ---- 5. store ------------------------------------------------------------
    if (XMODE) {
        __syncthreads();  // every window/closure read of the tile is done
#pragma unroll
        for (int i = 0; i < kMaxSeg; ++i)
            if (i < m) tile[(off + i) * TP + lane] = y[i];
        __syncthreads();
        tile_rows<T, false>(P, out, fout, tile, line0, nl, n, TP, mode);
    } else {
        // In place (out == in) is safe: with S > 1 the interface barrier
        // separates every window read of a line from its stores, with S = 1 a
        // line belongs to one thread, and different CTAs own disjoint lines.
        if (!valid) return;
#pragma unroll
        for (int i = 0; i < kMaxSeg; ++i) {
            if (i < m) {
                T* o = fout + Lout.base + (int64_t)(off + i) * Lout.stride;
                if (mode == OUT_STORE) *o = y[i];
                else if (mode == OUT_NEGATE) *o = -y[i];
                else *o = *o - y[i];
            }
        }
    }
}

template <typename T, int Q, int M, bool X>
void launch_t(const CompactParams& P, const T* tab, const FieldView& in, const FieldView& out, int count, int mode,
              cudaStream_t st) {
    const int N = 2 * Q * P.S;
    size_t smem = 0;
    if (X) smem += sizeof(T) * (size_t)P.n * (P.LB + 1);
    if (P.hasred) smem += sizeof(T) * (size_t)P.LB * (N + 1);
    auto kern = k_compact<T, Q, M, X>;
    static thread_local int configured = 0;
    if (smem > 48 * 1024 && configured < (int)smem) {
        CLES_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        configured = (int)smem;
    }
    dim3 grid((unsigned)((P.lines + P.LB - 1) / P.LB), (unsigned)count);
    dim3 block((unsigned)(P.LB * P.S));
    kern<<<grid, block, smem, st>>>(P, tab, in, out, mode);
    count_launch();
    check_launch("k_compact");
}

template <typename T, int Q, bool X>
void dispatch_m(const CompactParams& P, const T* tab, const FieldView& in, const FieldView& out, int count, int mode,
                cudaStream_t st) {
    switch (P.M) {
        case 1: launch_t<T, Q, 1, X>(P, tab, in, out, count, mode, st); break;
        case 2: launch_t<T, Q, 2, X>(P, tab, in, out, count, mode, st); break;
        case 3: launch_t<T, Q, 3, X>(P, tab, in, out, count, mode, st); break;
        case 4: launch_t<T, Q, 4, X>(P, tab, in, out, count, mode, st); break;
        default: throw Error(CLES_EINVAL, "unsupported stencil half-width");
    }
}

template <typename T>
void dispatch(const CompactParams& P, const T* tab, const FieldView& in, const FieldView& out, int count, int mode,
              cudaStream_t st) {
    const bool X = P.dim == 0;
    if (P.q == 1) {
        if (X) dispatch_m<T, 1, true>(P, tab, in, out, count, mode, st);
        else dispatch_m<T, 1, false>(P, tab, in, out, count, mode, st);
    } else {
        if (X) dispatch_m<T, 2, true>(P, tab, in, out, count, mode, st);
        else dispatch_m<T, 2, false>(P, tab, in, out, count, mode, st);
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
    if (plan.dtype == CLES_F64) dispatch<double>(plan.P, plan.tab64, in, out, count, mode, st);
    else dispatch<float>(plan.P, plan.tab32, in, out, count, mode, st);
    if (rec >= 0) prof_end(rec, st);
}

}  // namespace cles
