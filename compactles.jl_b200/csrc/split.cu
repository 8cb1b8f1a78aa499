// Lines split across ranks: the reference's P > 1 decomposition of a compact
// operator along one dimension (src/tridiag.jl:136-170, src/banded.jl:177-214,
// src/halo.jl:143-194), one process per GPU.
//
// One application on rank r, with the exchanges done by the caller (NCCL
// send/recv and all-gather through torch.distributed, or MPI for a Julia
// host) between the calls:
//   pack      the M planes at each end of the local interior -> send buffers;
//   (send the low planes to the previous rank, the high planes to the next)
//   unpack    received planes -> the padded halo beyond each open end;
//   local     a compact kernel over the rank's rows with open ends (their
//             stencil reads that halo: the tile kernels stage it beside the
//             line, the generic kernel reads it from global memory), storing
//             the local solution y and each line's first/last q values
//             (launch_compact_split);
//   (all-gather the heads and tails of every rank)
//   reduce    per line, the previous rank's last q and the next rank's first q
//             unknowns from the precomputed rows of the reduced inverse;
//   correct   out = y - V z_prev - W z_next.
// The two exchange points are the reference's Sendrecv! halo exchange and its
// Allgather! of the interface values; nothing here waits on another rank.

#include <algorithm>

#include "cles_internal.h"

namespace cles {

namespace {

constexpr int kThreads = 256;

inline unsigned grid_for(int64_t n) {
    int64_t b = (n + kThreads - 1) / kThreads;
    if (b > 148 * 32) b = 148 * 32;
    return (unsigned)(b < 1 ? 1 : b);
}

#define GRID_STRIDE(idx, n) \
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < (n); idx += (int64_t)gridDim.x * blockDim.x)

// Element offset of index g along `dim` on line `line` (the compact kernels'
// line numbering: the other two indices, lower dimension fastest).
__device__ __forceinline__ int64_t line_elem(int dim, int nx, int ny, int64_t sy, int64_t sz, int g, int line) {
    if (dim == 0) {
        const int j = line % ny, k = line / ny;
        return g + j * sy + k * sz;
    }
    if (dim == 1) {
        const int i = line % nx, k = line / nx;
        return i + (int64_t)g * sy + k * sz;
    }
    const int i = line % nx, j = line / nx;
    return i + j * sy + (int64_t)g * sz;
}

// pack: lo[c][p][l] = f[c][p], hi[c][p][l] = f[c][n-M+p];
// unpack: f[c][-M+p] = lo[c][p][l], f[c][n+p] = hi[c][p][l].
template <typename T>
__global__ void k_split_halo(T* __restrict__ f, FieldView v, T* __restrict__ lo, T* __restrict__ hi, int dim, int nx,
                             int ny, int n, int M, int lines, int count, int lo_on, int hi_on, int pack) {
    const int64_t total = (int64_t)count * M * lines;
    GRID_STRIDE(idx, total) {
        const int line = (int)(idx % lines);
        const int64_t r = idx / lines;
        const int p = (int)(r % M);
        const int64_t comp = r / M;
        T* fc = f + comp * v.comp_stride;
        if (pack) {
            if (lo_on) lo[idx] = fc[line_elem(dim, nx, ny, v.sy, v.sz, p, line)];
            if (hi_on) hi[idx] = fc[line_elem(dim, nx, ny, v.sy, v.sz, n - M + p, line)];
        } else {
            if (lo_on) fc[line_elem(dim, nx, ny, v.sy, v.sz, p - M, line)] = lo[idx];
            if (hi_on) fc[line_elem(dim, nx, ny, v.sy, v.sz, n + p, line)] = hi[idx];
        }
    }
}

// z[c][r][l] = sum_j Gsel[r][j] * y_all[j] with y_all[2q*rank + k] =
// gath[rank][c][k][l] (src/tridiag.jl:150-159: gather, then ldiv! of the
// reduced system; only the 2q unknowns this rank needs are formed).
template <typename T>
__global__ void k_split_reduce(const T* __restrict__ gath, const T* __restrict__ Gs, T* __restrict__ z, int lines,
                               int count, int q, int ranks) {
    const int m2 = 2 * q, N = m2 * ranks;
    const int64_t total = (int64_t)count * lines;
    GRID_STRIDE(idx, total) {
        const int line = (int)(idx % lines);
        const int64_t comp = idx / lines;
        for (int r = 0; r < m2; ++r) {
            const T* g = Gs + (int64_t)r * N;
            T acc = T(0);
            for (int rr = 0; rr < ranks; ++rr)
                for (int k = 0; k < m2; ++k)
                    acc += g[m2 * rr + k] * gath[((int64_t)(rr * count + comp) * m2 + k) * lines + line];
            z[(comp * m2 + r) * lines + line] = acc;
        }
    }
}

// out -= V[:, g] z_prev + W[:, g] z_next (src/tridiag.jl:161-169,
// src/banded.jl:201-214).  Rows (j, k, comp) are taken RB at a time per
// block-stride step, threads along x: coalesced, no 64-bit division per
// element, and RB loads in flight per thread before the stores.
constexpr int RB = 4;

template <typename T, int Q>
__device__ __forceinline__ void correct_coeffs(const T* __restrict__ V, const T* __restrict__ W,
                                               const T* __restrict__ z, int dim, int nx, int ny, int nz, int n,
                                               int lines, int row, int i, T* vg, T* wg, const T*& zl) {
    const int j = row % ny;
    const int kc = row / ny;
    const int k = kc % nz, comp = kc / nz;
    const T* zc = z + (int64_t)comp * 2 * Q * lines;
    int g, line;
    if (dim == 0) { g = i; line = j + k * ny; }
    else if (dim == 1) { g = j; line = i + k * nx; }
    else { g = k; line = i + j * nx; }
#pragma unroll
    for (int t = 0; t < Q; ++t) { vg[t] = V[t * n + g]; wg[t] = W[t * n + g]; }
    zl = zc + line;
}

template <typename T, int Q, int MODE>
__global__ void k_split_correct(const T* __restrict__ loc, FieldView lv, T* __restrict__ out, FieldView v,
                                const T* __restrict__ V, const T* __restrict__ W, const T* __restrict__ z, int dim,
                                int nx, int ny, int nz, int n, int lines, int count) {
    const int rows = ny * nz * count;
    for (int r0 = blockIdx.x * RB; r0 < rows; r0 += gridDim.x * RB) {
        for (int i = threadIdx.x; i < nx; i += blockDim.x) {
            T o[RB], acc[RB], prev[RB];
            T* po[RB];
#pragma unroll
            for (int b = 0; b < RB; ++b) {
                const int row = r0 + b;
                po[b] = nullptr;
                acc[b] = T(0);
                if (row < rows) {
                    const int j = row % ny, kc = row / ny;
                    const int k = kc % nz, comp = kc / nz;
                    po[b] = out + (int64_t)comp * v.comp_stride + j * v.sy + k * v.sz + i;
                    o[b] = loc[(int64_t)comp * lv.comp_stride + j * lv.sy + k * lv.sz + i];
                    if (MODE == OUT_SUBTRACT) prev[b] = *po[b];
                    T vg[Q], wg[Q];
                    const T* zl;
                    correct_coeffs<T, Q>(V, W, z, dim, nx, ny, nz, n, lines, row, i, vg, wg, zl);
#pragma unroll
                    for (int t = 0; t < Q; ++t) acc[b] += vg[t] * zl[(int64_t)t * lines] + wg[t] * zl[(int64_t)(Q + t) * lines];
                }
            }
#pragma unroll
            for (int b = 0; b < RB; ++b) {
                if (!po[b]) continue;
                const T r = o[b] - acc[b];
                if (MODE == OUT_NEGATE) *po[b] = -r;
                else if (MODE == OUT_SUBTRACT) *po[b] = prev[b] - r;
                else *po[b] = r;
            }
        }
    }
}

// dst = src over the interior of two views of one grid shape (rows of x
// points, a block per RB rows as in the correction).
template <typename T>
__global__ void k_copy_view(const T* __restrict__ src, FieldView sv, T* __restrict__ dst, FieldView dv, int nx,
                            int ny, int nz, int count) {
    const int rows = ny * nz * count;
    for (int r0 = blockIdx.x * RB; r0 < rows; r0 += gridDim.x * RB) {
        for (int i = threadIdx.x; i < nx; i += blockDim.x) {
            T val[RB];
#pragma unroll
            for (int b = 0; b < RB; ++b) {
                const int row = r0 + b;
                if (row < rows) {
                    const int j = row % ny, kc = row / ny;
                    const int k = kc % nz, comp = kc / nz;
                    val[b] = src[(int64_t)comp * sv.comp_stride + j * sv.sy + k * sv.sz + i];
                }
            }
#pragma unroll
            for (int b = 0; b < RB; ++b) {
                const int row = r0 + b;
                if (row < rows) {
                    const int j = row % ny, kc = row / ny;
                    const int k = kc % nz, comp = kc / nz;
                    dst[(int64_t)comp * dv.comp_stride + j * dv.sy + k * dv.sz + i] = val[b];
                }
            }
        }
    }
}

inline void row_launch(int nx, int64_t rows, unsigned* nb, int* bt) {
    // a block per x row (threads cover up to 256 x points per step)
    *bt = nx >= 256 ? 256 : ((nx + 31) / 32) * 32;
    *nb = (unsigned)std::min<int64_t>((rows + RB - 1) / RB, 148 * 64);
}

template <typename T>
void halo_t(const HaloSpec& hs, const FieldView& f, void* lo, void* hi, int count, bool pack, cudaStream_t st) {
    const int64_t total = (int64_t)count * hs.M * hs.lines;
    k_split_halo<T><<<grid_for(total), kThreads, 0, st>>>(static_cast<T*>(f.base), f, static_cast<T*>(lo),
                                                          static_cast<T*>(hi), hs.dim, hs.n3[0], hs.n3[1],
                                                          hs.n3[hs.dim], hs.M, (int)hs.lines, count,
                                                          hs.lo_open ? 1 : 0, hs.hi_open ? 1 : 0, pack ? 1 : 0);
    count_launch();
    check_launch("k_split_halo");
}

template <typename T, int Q>
void correct_mode(int mode, unsigned nb, int bt, cudaStream_t st, const T* loc, const FieldView& lv, T* out,
                  const FieldView& v, const T* V, const T* W, const T* z, const SplitPlan& sp, int count) {
    const int nx = sp.n3[0], ny = sp.n3[1], nz = sp.n3[2], lines = (int)sp.lines;
    if (mode == OUT_NEGATE)
        k_split_correct<T, Q, OUT_NEGATE><<<nb, bt, 0, st>>>(loc, lv, out, v, V, W, z, sp.dim, nx, ny, nz, sp.n, lines,
                                                            count);
    else if (mode == OUT_SUBTRACT)
        k_split_correct<T, Q, OUT_SUBTRACT><<<nb, bt, 0, st>>>(loc, lv, out, v, V, W, z, sp.dim, nx, ny, nz, sp.n,
                                                              lines, count);
    else
        k_split_correct<T, Q, OUT_STORE><<<nb, bt, 0, st>>>(loc, lv, out, v, V, W, z, sp.dim, nx, ny, nz, sp.n, lines,
                                                           count);
}

template <typename T>
void correct_t(const SplitPlan& sp, const void* gathered, void* zbuf, const FieldView& loc, const FieldView& out,
               int count, int mode, cudaStream_t st) {
    const T* tab = static_cast<const T*>(sp.tab);
    const int64_t nv = (int64_t)sp.q * sp.n;
    const T* V = tab;
    const T* W = tab + nv;
    const T* Gs = tab + 2 * nv;
    const int64_t nl = (int64_t)count * sp.lines;
    k_split_reduce<T><<<grid_for(nl), kThreads, 0, st>>>(static_cast<const T*>(gathered), Gs, static_cast<T*>(zbuf),
                                                         (int)sp.lines, count, sp.q, sp.ranks);
    count_launch();
    check_launch("k_split_reduce");
    const int64_t rows = (int64_t)sp.n3[1] * sp.n3[2] * count;
    if (rows >= ((int64_t)1 << 31)) throw Error(CLES_EINVAL, "too many rows for one correction launch");
    unsigned nb;
    int bt;
    row_launch(sp.n3[0], rows, &nb, &bt);
    const T* lp = static_cast<const T*>(loc.base);
    T* op = static_cast<T*>(out.base);
    const T* z = static_cast<const T*>(zbuf);
    if (sp.q == 1) correct_mode<T, 1>(mode, nb, bt, st, lp, loc, op, out, V, W, z, sp, count);
    else correct_mode<T, 2>(mode, nb, bt, st, lp, loc, op, out, V, W, z, sp, count);
    count_launch();
    check_launch("k_split_correct");
}

}  // namespace

HaloSpec halo_spec(const SplitPlan& sp) {
    HaloSpec h;
    h.dim = sp.dim;
    for (int k = 0; k < 3; ++k) h.n3[k] = sp.n3[k];
    h.M = sp.M;
    h.lines = sp.lines;
    h.lo_open = sp.lo_open;
    h.hi_open = sp.hi_open;
    return h;
}

void halo_planes(const HaloSpec& hs, const FieldView& f, void* lo, void* hi, int count, bool pack, int dtype,
                 cudaStream_t st) {
    if (count <= 0 || hs.lines == 0 || (!hs.lo_open && !hs.hi_open)) return;
    if (dtype == CLES_F64) halo_t<double>(hs, f, lo, hi, count, pack, st);
    else halo_t<float>(hs, f, lo, hi, count, pack, st);
}

void split_halo(const SplitPlan& sp, const FieldView& f, void* lo, void* hi, int count, bool pack, cudaStream_t st) {
    halo_planes(halo_spec(sp), f, lo, hi, count, pack, sp.dtype, st);
}

void split_correct(const SplitPlan& sp, const void* gathered, void* zbuf, const FieldView& loc, const FieldView& out,
                   int count, int mode, cudaStream_t st) {
    if (count <= 0 || sp.lines == 0) return;
    if (!sp.lo_open && !sp.hi_open) {
        // one closed piece: the local solution is the answer
        if (mode == OUT_STORE && loc.base == out.base) return;
        throw Error(CLES_EINVAL, "internal: a closed piece has no correction to apply");
    }
    if (sp.dtype == CLES_F64) correct_t<double>(sp, gathered, zbuf, loc, out, count, mode, st);
    else correct_t<float>(sp, gathered, zbuf, loc, out, count, mode, st);
}

void split_correct(const SplitPlan& sp, const void* gathered, void* zbuf, const FieldView& out, int count,
                   cudaStream_t st) {
    if (count <= 0 || sp.lines == 0 || (!sp.lo_open && !sp.hi_open)) return;
    split_correct(sp, gathered, zbuf, out, out, count, OUT_STORE, st);
}

void copy_view(const FieldView& src, const FieldView& dst, const int n3[3], int count, int dtype, cudaStream_t st) {
    const int64_t rows = (int64_t)n3[1] * n3[2] * count;
    if (rows == 0 || n3[0] == 0) return;
    if (rows >= ((int64_t)1 << 31)) throw Error(CLES_EINVAL, "too many rows for one copy launch");
    unsigned nb;
    int bt;
    row_launch(n3[0], rows, &nb, &bt);
    if (dtype == CLES_F64)
        k_copy_view<double><<<nb, bt, 0, st>>>(static_cast<const double*>(src.base), src,
                                               static_cast<double*>(dst.base), dst, n3[0], n3[1], n3[2], count);
    else
        k_copy_view<float><<<nb, bt, 0, st>>>(static_cast<const float*>(src.base), src, static_cast<float*>(dst.base),
                                              dst, n3[0], n3[1], n3[2], count);
    count_launch();
    check_launch("k_copy_view");
}

}  // namespace cles
