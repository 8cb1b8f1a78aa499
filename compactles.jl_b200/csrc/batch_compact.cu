// Batched compact operators: one launch applies a directional operator to
// the lines of many grids of different sizes.
//
// A launch carries a table of per-grid plans (BatchLinePlan: the plan's
// parameters, its coefficient table and where the grid's fields sit in the
// batch arena) and a table of CTAs, each naming one plan and its first line.
// Every CTA reads its plan's parameters in place and runs the generic
// segmented spike solve of compact_body.cuh on LB lines of that grid.
// All plans of a launch share the kernel template (element type, q, M, x or
// y/z staging) and the thread count LB x S; S is a power of two per grid, so
// short lines get many lines per CTA and long lines few.  The RK update of
// the last flux-divergence direction is applied in the store with each grid's
// own dt, read from its graph-mode clock.

#include "cles_internal.h"
#include "compact_body.cuh"
#include "pointwise.h"

namespace cles {

namespace {

template <typename T, int Q, int M, bool XMODE, int MS>
__global__ void __launch_bounds__(kBatchMaxThreads) k_compact_batch(const BatchLinePlan* __restrict__ plans,
                                                        const int2* __restrict__ blocks, const T* in_base,
                                                        T* out_base, const int64_t ct, const int mode,
                                                        double* Qs, double* dus, const double A, const double B,
                                                        const int skip_idle) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int2 bk = blocks[blockIdx.x];
    // the plan is read in place through a restrict-qualified const pointer:
    // nothing the kernel stores can alias it, so its fields load once
    const BatchLinePlan* __restrict__ bp = plans + bk.x;
    const CompactParams& Ps = bp->P;
    double dt = 0.0;
    if (bp->clk) dt = bp->clk[DC_DT];
    if (skip_idle && dt == 0.0) return;   // the same for every thread of the CTA
    const int64_t off = bp->off;
    const FieldView in{const_cast<T*>(in_base) + off, ct, bp->sy, bp->sz};
    const FieldView out{out_base + off, ct, bp->sy, bp->sz};
    const int comp = blockIdx.y;
    const RkStore rk{Qs, dus, A, B, dt, (int64_t)comp * ct + off};
    compact_lines<T, Q, M, XMODE, MS, true>(Ps, static_cast<const T*>(bp->tab), in, out, mode, nullptr, bk.y,
                                                 comp, &rk, smem_raw);
}

template <typename T, int Q, int M, bool X, int MS>
void launch_k(const BatchLaunchKind& k, const BatchLinePlan* plans, const int2* blocks, int nblocks, const void* in,
              void* out, int64_t ct, int count, int mode, double* Q_, double* du, double A, double B, int skip,
              cudaStream_t st) {
    auto kern = k_compact_batch<T, Q, M, X, MS>;
    static thread_local size_t configured = 0;
    if (k.smem > 48 * 1024 && configured < k.smem) {
        CLES_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)k.smem));
        configured = k.smem;
    }
    dim3 grid((unsigned)nblocks, (unsigned)count);
    kern<<<grid, k.threads, k.smem, st>>>(plans, blocks, static_cast<const T*>(in), static_cast<T*>(out), ct, mode,
                                          Q_, du, A, B, skip);
    count_launch();
    check_launch("k_compact_batch");
}

template <typename T, int Q, int M, bool X>
void launch_ms(const BatchLaunchKind& k, const BatchLinePlan* plans, const int2* blocks, int nb, const void* in,
               void* out, int64_t ct, int count, int mode, double* Q_, double* du, double A, double B, int skip,
               cudaStream_t st) {
    switch (k.ms) {
        case 8: launch_k<T, Q, M, X, 8>(k, plans, blocks, nb, in, out, ct, count, mode, Q_, du, A, B, skip, st); break;
        case 16: launch_k<T, Q, M, X, 16>(k, plans, blocks, nb, in, out, ct, count, mode, Q_, du, A, B, skip, st); break;
        case 32: launch_k<T, Q, M, X, 32>(k, plans, blocks, nb, in, out, ct, count, mode, Q_, du, A, B, skip, st); break;
        default: throw Error(CLES_EINVAL, "batched register tile must be 8, 16 or 32 points");
    }
}

// The schemes of the library: C4 (q 1, M 1), C6 (1, 2), the C8 filter (1, 4), C10 (2, 3).
template <typename T, bool X>
void launch_x(const BatchLaunchKind& k, const BatchLinePlan* plans, const int2* blocks, int nb, const void* in,
              void* out, int64_t ct, int count, int mode, double* Q_, double* du, double A, double B, int skip,
              cudaStream_t st) {
    if (k.q == 1 && k.M == 1) launch_ms<T, 1, 1, X>(k, plans, blocks, nb, in, out, ct, count, mode, Q_, du, A, B, skip, st);
    else if (k.q == 1 && k.M == 2) launch_ms<T, 1, 2, X>(k, plans, blocks, nb, in, out, ct, count, mode, Q_, du, A, B, skip, st);
    else if (k.q == 1 && k.M == 4) launch_ms<T, 1, 4, X>(k, plans, blocks, nb, in, out, ct, count, mode, Q_, du, A, B, skip, st);
    else if (k.q == 2 && k.M == 3) launch_ms<T, 2, 3, X>(k, plans, blocks, nb, in, out, ct, count, mode, Q_, du, A, B, skip, st);
    else throw Error(CLES_EINVAL, "batched solves support the C4, C6, C10 and C8-filter stencil shapes only");
}

template <typename T>
void launch_t(const BatchLaunchKind& k, const BatchLinePlan* plans, const int2* blocks, int nb, const void* in,
              void* out, int64_t ct, int count, int mode, double* Q_, double* du, double A, double B, int skip,
              cudaStream_t st) {
    if (k.xmode) launch_x<T, true>(k, plans, blocks, nb, in, out, ct, count, mode, Q_, du, A, B, skip, st);
    else launch_x<T, false>(k, plans, blocks, nb, in, out, ct, count, mode, Q_, du, A, B, skip, st);
}

}  // namespace

size_t batch_plan_smem(const CompactParams& P, int LB, int dtype) {
    const size_t el = dtype == CLES_F64 ? sizeof(double) : sizeof(float);
    const int N = 2 * P.q * P.S;
    size_t smem = 0;
    if (P.dim == 0) smem += el * (size_t)P.n * (LB + 1);
    if (P.pcr) smem += el * (size_t)LB * 4 * P.S;
    else if (P.hasred) smem += el * ((size_t)LB * (N + 1) + (size_t)N * (N + 1));   // + the staged inverse
    return smem;
}

void launch_compact_batch(const BatchLaunchKind& kind, const BatchLinePlan* plans, const int2* blocks, int nblocks,
                          const void* in, void* out, int64_t ct, int count, int mode, double* Q, double* du, double A,
                          double B, int skip_idle, cudaStream_t st) {
    if (nblocks <= 0 || count <= 0) return;
    if (kind.dtype == CLES_F64)
        launch_t<double>(kind, plans, blocks, nblocks, in, out, ct, count, mode, Q, du, A, B, skip_idle, st);
    else
        launch_t<float>(kind, plans, blocks, nblocks, in, out, ct, count, mode, Q, du, A, B, skip_idle, st);
}

}  // namespace cles
