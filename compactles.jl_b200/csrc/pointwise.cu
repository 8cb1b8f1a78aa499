// Pointwise kernels of the RHS and the integrator (interior layout, x fastest).
//
// F is the storage type of the derived fields (double in the plain form,
// float in the mixed form); the conserved state Q and the RK register du are
// always double.  Arithmetic follows the association order of the cited
// reference lines.

#include "pointwise.h"

namespace cles {

namespace {

constexpr int kThreads = 256;

// Julia's Base.max/min on floats: a NaN operand wins.
__device__ __forceinline__ double jl_max(double x, double y) {
    if (x != x) return x;
    if (y != y) return y;
    return y > x ? y : x;
}
__device__ __forceinline__ double jl_min(double x, double y) {
    if (x != x) return x;
    if (y != y) return y;
    return y < x ? y : x;
}

// Julia's clamp(x, lo, hi): a NaN argument passes through.
__device__ __forceinline__ double jl_clamp(double x, double lo, double hi) {
    return x > hi ? hi : (x < lo ? lo : x);
}

// ---- NASA-9 species thermodynamics (src/physics.jl:298-310, 431-455) ----
__device__ __forceinline__ int n9_interval(const PhysConst& pc, int k, double T) {
    const int n = pc.nint[k];
    for (int i = 0; i < n - 1; ++i)
        if (T <= pc.Tmax[k][i]) return i;
    return n - 1;
}
__device__ __forceinline__ double n9_cp_R(const double* a, double T) {
    const double T2 = T * T;
    return a[0] / T2 + a[1] / T + a[2] + a[3] * T + a[4] * T2 + a[5] * (T2 * T) + a[6] * (T2 * T2);
}
__device__ __forceinline__ double n9_h_R(const double* a, double b1, double T) {
    const double T2 = T * T;
    return -a[0] / T + a[1] * log(T) + a[2] * T + a[3] * T2 / 2 + a[4] * (T2 * T) / 3 + a[5] * (T2 * T2) / 4 +
           a[6] * (T2 * T2 * T) / 5 + b1;
}
__device__ __forceinline__ double n9_cp(const PhysConst& pc, int k, double T) {
    return pc.Rk[k] * n9_cp_R(pc.a[k][n9_interval(pc, k, T)], T);
}
__device__ __forceinline__ double n9_h(const PhysConst& pc, int k, double T) {
    const int i = n9_interval(pc, k, T);
    return pc.Rk[k] * n9_h_R(pc.a[k][i], pc.b1[k][i], T);
}
// mixture_temperature (src/physics.jl:466-498): bounded Newton on
// sum_k Y_k e_k(T) = e, always in FP64.
__device__ double n9_temperature(const PhysConst& pc, int Ns, double e, const double* Y) {
    double e0 = 0.0, cv0 = 0.0;
    for (int k = 0; k < Ns; ++k) {
        e0 += Y[k] * pc.e_ref[k];
        cv0 += Y[k] * pc.cv_ref[k];
    }
    double T = cv0 > 0 ? jl_clamp(pc.T_guess + (e - e0) / cv0, 1e-3, 1e9) : pc.T_guess;
    for (int it = 0; it < 30; ++it) {
        double f = -e, cvm = 0.0;
        for (int k = 0; k < Ns; ++k) {
            const int i = n9_interval(pc, k, T);
            const double* a = pc.a[k][i];
            f += Y[k] * (pc.Rk[k] * n9_h_R(a, pc.b1[k][i], T) - pc.Rk[k] * T);
            cvm += Y[k] * (pc.Rk[k] * n9_cp_R(a, T) - pc.Rk[k]);
        }
        if (!(cvm > 0)) break;
        const double d = f / cvm;
        T = jl_max(T - d, 0.25 * T);
        if (fabs(d) <= 1e-14 * T) break;
    }
    return T;
}

inline unsigned grid_for(int64_t n) {
    int64_t b = (n + kThreads - 1) / kThreads;
    if (b > 148 * 64) b = 148 * 64;
    return (unsigned)(b < 1 ? 1 : b);
}

#define LAUNCH(kern, n, st, ...)                                      \
    do {                                                               \
        kern<<<grid_for(n), kThreads, 0, st>>>(__VA_ARGS__);           \
        count_launch();                                                \
        check_launch(#kern);                                           \
    } while (0)

// opt a kernel in to `bytes` of dynamic shared memory (above the 48 KB
// default) on the current device; a host call, set before every launch so
// that every device and thread sees it
template <typename K>
void set_smem_attr(K kern, size_t bytes) {
    CLES_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
}

#define GRID_STRIDE(idx, n) for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < (n); idx += (int64_t)gridDim.x * blockDim.x)

// _primitives!(::IdealMixture) (src/physics.jl:604-653) at the interior, and
// _primitives!(::Nasa9Mixture) (src/physics.jl:501-570) when N9 (a separate
// instantiation, so the ideal-gas kernel keeps its small register footprint).
// PM (batched solves): the species constants are per batch member, mc[24 m ..]
// = R_k, cv_k, cp_k (8 each) of member m = tmap[cell / 64].
template <typename F, bool N9, bool PM = false>
__global__ void k_primitives(const double* __restrict__ Q, F* __restrict__ prim, int64_t cells, int Ns, PhysConst pc,
                             int esens, const double* __restrict__ mc = nullptr, const int* __restrict__ tmap = nullptr) {
    GRID_STRIDE(I, cells) {
        const double* mcI = nullptr;
        if constexpr (PM) mcI = mc + 24 * tmap[I >> 6];
        double rho = 0.0;
        for (int sp = 0; sp < Ns; ++sp) rho += Q[I + cells * sp];
        F* out = prim + I;
        if (N9 && rho > 0) {
            const double ri = 1 / rho;
            double Y[CLES_MAX_SPECIES];
            double Rm = 0.0;
            for (int sp = 0; sp < Ns; ++sp) {
                Y[sp] = Q[I + cells * sp] * ri;
                out[cells * (P_Y0 + sp)] = F(Y[sp]);
                Rm += Y[sp] * pc.Rk[sp];
            }
            const double u = Q[I + cells * (Ns + 0)] * ri;
            const double v = Q[I + cells * (Ns + 1)] * ri;
            const double w = Q[I + cells * (Ns + 2)] * ri;
            const double e = Q[I + cells * (Ns + 3)] * ri - 0.5 * (u * u + v * v + w * w);
            const double T = n9_temperature(pc, Ns, e, Y);
            double cpm = 0.0;
            for (int sp = 0; sp < Ns; ++sp) cpm += Y[sp] * n9_cp(pc, sp, T);
            const double cvm = cpm - Rm;
            out[cells * P_RHO] = F(rho);
            out[cells * P_U] = F(u);
            out[cells * P_V] = F(v);
            out[cells * P_W] = F(w);
            out[cells * P_P] = F(rho * Rm * T);
            out[cells * P_T] = F(T);
            out[cells * P_C] = F(sqrt(jl_max((cpm / cvm) * Rm * T, 0.0)));
            out[cells * P_CP] = F(cpm);
            if (esens) {
                const double r = jl_max(rho, 1e-300);
                const double q1 = Q[I + cells * (Ns + 0)], q2 = Q[I + cells * (Ns + 1)], q3 = Q[I + cells * (Ns + 2)];
                const double ke = 0.5 * (q1 * q1 + q2 * q2 + q3 * q3) / r;
                out[cells * (P_Y0 + Ns)] = F((Q[I + cells * (Ns + 3)] - ke) / r);
            }
        } else if (rho > 0) {
            const double ri = 1 / rho;
            double Rm = 0.0, cvm = 0.0;
            for (int sp = 0; sp < Ns; ++sp) {
                const double q = Q[I + cells * sp];
                if constexpr (PM) {
                    Rm += q * mcI[sp];
                    cvm += q * mcI[8 + sp];
                } else {
                    Rm += q * pc.Rk[sp];
                    cvm += q * pc.cvk[sp];
                }
                out[cells * (P_Y0 + sp)] = F(q * ri);
            }
            Rm *= ri;
            cvm *= ri;
            const double u = Q[I + cells * (Ns + 0)] * ri;
            const double v = Q[I + cells * (Ns + 1)] * ri;
            const double w = Q[I + cells * (Ns + 2)] * ri;
            const double e = Q[I + cells * (Ns + 3)] * ri - 0.5 * (u * u + v * v + w * w);
            const double T = jl_max(e / cvm, 1e-300);
            const double p = rho * Rm * T;
            const double gm = 1 + Rm / cvm;
            out[cells * P_RHO] = F(rho);
            out[cells * P_U] = F(u);
            out[cells * P_V] = F(v);
            out[cells * P_W] = F(w);
            out[cells * P_P] = F(p);
            out[cells * P_T] = F(T);
            out[cells * P_C] = F(sqrt(gm * Rm * T));
            out[cells * P_CP] = F(cvm + Rm);
            if (esens) {
                // internal energy for the kappa* sensor (src/artificial.jl:322-330): rho floored, |m|^2/2rho
                const double r = jl_max(rho, 1e-300);
                const double q1 = Q[I + cells * (Ns + 0)], q2 = Q[I + cells * (Ns + 1)], q3 = Q[I + cells * (Ns + 2)];
                const double ke = 0.5 * (q1 * q1 + q2 * q2 + q3 * q3) / r;
                out[cells * (P_Y0 + Ns)] = F((Q[I + cells * (Ns + 3)] - ke) / r);
            }
        } else {
            out[cells * P_RHO] = F(1);
            out[cells * P_U] = F(0);
            out[cells * P_V] = F(0);
            out[cells * P_W] = F(0);
            out[cells * P_P] = F(1);
            out[cells * P_T] = F(1);
            out[cells * P_C] = F(1);
            out[cells * P_CP] = F(1);
            for (int sp = 0; sp < Ns; ++sp) out[cells * (P_Y0 + sp)] = F(sp == 0 ? 1.0 : 0.0);
            if (esens) {
                // placeholder density 1: the floor is max(1, 1e-300) = 1
                const double q1 = Q[I + cells * (Ns + 0)], q2 = Q[I + cells * (Ns + 1)], q3 = Q[I + cells * (Ns + 2)];
                const double ke = 0.5 * (q1 * q1 + q2 * q2 + q3 * q3) / 1.0;
                out[cells * (P_Y0 + Ns)] = F((Q[I + cells * (Ns + 3)] - ke) / 1.0);
            }
        }
    }
}

// |S| = sqrt(S_ij S_ij) (src/artificial.jl:287-300); g[3d+j] = d u_j / d x_d.
template <typename F>
__global__ void k_strain(const F* __restrict__ g, F* __restrict__ out, int64_t cells) {
    GRID_STRIDE(I, cells) {
        double gv[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) gv[k] = double(g[I + cells * k]);
        double ss = 0.0;
#pragma unroll
        for (int b = 0; b < 3; ++b)
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                const double Sab = 0.5 * (gv[3 * a + b] + gv[3 * b + a]);
                ss += Sab * Sab;
            }
        out[I] = F(sqrt(ss));
    }
}

// delta4_sum! (src/artificial.jl:67-94): sum_d h_d^p |(1,-4,6,-4,1) f| along d,
// periodic wrap or clamping at closed edges.
template <typename F>
__global__ void k_delta4(const F* __restrict__ f, F* __restrict__ out, Grid3 g, double w0, double w1, double w2) {
    const int64_t cells = (int64_t)g.n[0] * g.n[1] * g.n[2];
    const double wd[3] = {w0, w1, w2};
    const double D4[5] = {1.0, -4.0, 6.0, -4.0, 1.0};
    const int64_t st[3] = {1, (int64_t)g.n[0], (int64_t)g.n[0] * g.n[1]};
    GRID_STRIDE(I, cells) {
        const int i = (int)(I % g.n[0]);
        const int j = (int)((I / g.n[0]) % g.n[1]);
        const int k = (int)(I / ((int64_t)g.n[0] * g.n[1]));
        const int ijk[3] = {i, j, k};
        double o = 0.0;
        for (int d = 0; d < 3; ++d) {
            if (!g.active[d]) continue;
            const int nd = g.n[d];
            const int il = ijk[d];
            double acc = 0.0;
#pragma unroll
            for (int m = -2; m <= 2; ++m) {
                int ilm = il + m;
                if (g.periodic[d]) ilm = ilm < 0 ? ilm + nd : (ilm >= nd ? ilm - nd : ilm);
                else ilm = ilm < 0 ? 0 : (ilm >= nd ? nd - 1 : ilm);
                acc += D4[m + 2] * double(f[I + (int64_t)(ilm - il) * st[d]]);
            }
            o += wd[d] * fabs(acc);
        }
        out[I] = F(o);
    }
}

// delta4_sum! for NF fields at once, tiled: a block of 256 threads covers
// 32 x 16 (x, y) columns and walks z; each thread owns two neighbouring rows
// of one x column.  The halo'd xy planes z0-2 .. z0+kZC+1 stream through a
// ring of kRing planes in shared memory by cp.async (one commit group per
// plane); at plane z the x and y differences read plane z (the six column
// values of a thread serve both rows' y differences) and the z difference a
// register window of the thread's two columns, fed from plane z+2.  Eight
// shared-memory reads a point and field.  Accumulation order per point is
// the reference's: out = 0; for d in x, y, z: out += w_d |sum_m D4_m f|.
constexpr int kTX = kD4X, kTY = kD4Y, kZC = kD4Z;
__device__ __forceinline__ int edge_index(int i, int n, int periodic) {
    if (periodic) return i < 0 ? i + n : (i >= n ? i - n : i);
    return i < 0 ? 0 : (i >= n ? n - 1 : i);
}
constexpr int kRing = 6;
constexpr int kD4Threads = 256;
constexpr int kPlane = (kTY + 4) * (kTX + 4);
constexpr int kStage = (kPlane + kD4Threads - 1) / kD4Threads;   // staging slots a thread
static_assert(kTX * kTY == 2 * kD4Threads, "two rows a thread");
template <typename F, int NF>
constexpr size_t delta4_smem() {
    return sizeof(F) * (size_t)kRing * NF * kPlane;
}
__device__ __forceinline__ unsigned d4_smem_addr(const void* p) {
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
template <typename F>
__device__ __forceinline__ void d4_cp_async(F* dst, const F* src) {
    if constexpr (sizeof(F) == 8)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d4_smem_addr(dst)), "l"(src) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d4_smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void d4_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }

template <typename F, int NF>
__device__ __forceinline__ void delta4_tile(const F* __restrict__ f0, const F* __restrict__ f1, F* __restrict__ o0,
                                            F* __restrict__ o1, const Grid3& g, const Weights3& w0,
                                            const Weights3& w1, const int x0, const int y0, const int z0,
                                            F* __restrict__ ring) {
    constexpr int TW = kTX + 4;
    const F* fs[2] = {f0, f1};
    F* os[2] = {o0, o1};
    const Weights3 ws[2] = {w0, w1};
    const int nx = g.n[0], ny = g.n[1], nz = g.n[2];
    const int64_t sy = nx, sz = (int64_t)nx * ny;
    const int tx = threadIdx.x % kTX, ty = threadIdx.x / kTX;
    const int x = x0 + tx, ya = y0 + 2 * ty;
    const bool ins[2] = {x < nx && ya < ny, x < nx && ya + 1 < ny};
    const bool zact = g.active[2] != 0;
    const double D4[5] = {1.0, -4.0, 6.0, -4.0, 1.0};
    // this thread's staging slots of a halo'd plane: ring offset and in-plane
    // source offset (periodic wrap or clamping, as delta4_sum!)
    int64_t soff_g[kStage];
    bool sv[kStage];
#pragma unroll
    for (int s = 0; s < kStage; ++s) {
        const int idx = threadIdx.x + kD4Threads * s;
        sv[s] = idx < kPlane;
        const int hx = idx % TW, hy = idx / TW;
        const int gx = g.active[0] ? edge_index(x0 - 2 + hx, nx, g.periodic[0]) : min(x0 - 2 + hx < 0 ? 0 : x0 - 2 + hx, nx - 1);
        const int gy = g.active[1] ? edge_index(y0 - 2 + hy, ny, g.periodic[1]) : min(y0 - 2 + hy < 0 ? 0 : y0 - 2 + hy, ny - 1);
        soff_g[s] = (int64_t)gx + (int64_t)gy * sy;
    }
    const int zend = min(z0 + kZC, nz);
    // plane r of the block (r = 0 is z0 - 2) into ring slot r % kRing; planes
    // past the last one any output reads are left out (empty group)
    const int rlast = zact ? (zend - 1 + 2) - (z0 - 2) : 2;
    auto slot = [&](int r) { return ring + (size_t)(r % kRing) * NF * kPlane; };
    auto issue = [&](int r) {
        if (r <= rlast) {
            const int zz = zact ? edge_index(z0 - 2 + r, nz, g.periodic[2]) : 0;
            F* sl = slot(r);
#pragma unroll
            for (int f = 0; f < NF; ++f)
#pragma unroll
                for (int s = 0; s < kStage; ++s)
                    if (sv[s])
                        d4_cp_async(sl + f * kPlane + threadIdx.x + kD4Threads * s, fs[f] + soff_g[s] + (int64_t)zz * sz);
        }
        d4_commit();
    };
    // column offset of row t (0, 1) of this thread in a plane
    const int cofs = (2 * ty + 2) * TW + tx + 2;
    // planes 0 .. 5; the z window starts with planes 0 .. 3 (z0-2 .. z0+1)
#pragma unroll
    for (int r = 0; r < kRing; ++r) issue(r);
    F zw[NF][2][5];
    asm volatile("cp.async.wait_group 2;" ::: "memory");
    __syncthreads();
    if (zact) {
#pragma unroll
        for (int f = 0; f < NF; ++f)
#pragma unroll
            for (int q = 0; q < 4; ++q)
#pragma unroll
                for (int t = 0; t < 2; ++t) zw[f][t][q + 1] = slot(q)[f * kPlane + cofs + t * TW];
    }
    for (int z = z0; z < zend; ++z) {
        const int rz = z - z0 + 2;
        // this thread's copies of plane rz + 2 have landed (plane rz + 3 may
        // still be in flight); after the barrier everyone's have, and plane
        // rz - 2 is read by no one
        asm volatile("cp.async.wait_group 1;" ::: "memory");
        __syncthreads();
        issue(rz + 4);
        const F* pl = slot(rz);
        const F* pc = slot(rz + 2);
#pragma unroll
        for (int f = 0; f < NF; ++f) {
            const F* t0 = pl + f * kPlane;
            if (zact) {
#pragma unroll
                for (int t = 0; t < 2; ++t) {
#pragma unroll
                    for (int q = 0; q < 4; ++q) zw[f][t][q] = zw[f][t][q + 1];
                    zw[f][t][4] = pc[f * kPlane + cofs + t * TW];
                }
            }
            // the column x: tile rows 2ty .. 2ty+5 (both rows' y stencils)
            F cy[6];
#pragma unroll
            for (int k = 0; k < 6; ++k) cy[k] = t0[(2 * ty + k) * TW + tx + 2];
#pragma unroll
            for (int t = 0; t < 2; ++t) {
                if (!ins[t]) continue;
                double o = 0.0;
                if (g.active[0]) {
                    const F* row = t0 + (2 * ty + 2 + t) * TW + tx;
                    double acc = 0.0;
#pragma unroll
                    for (int m = 0; m < 5; ++m) acc += D4[m] * double(m == 2 ? cy[2 + t] : row[m]);
                    o += ws[f].w[0] * fabs(acc);
                }
                if (g.active[1]) {
                    double acc = 0.0;
#pragma unroll
                    for (int m = 0; m < 5; ++m) acc += D4[m] * double(cy[t + m]);
                    o += ws[f].w[1] * fabs(acc);
                }
                if (zact) {
                    double acc = 0.0;
#pragma unroll
                    for (int m = 0; m < 5; ++m) acc += D4[m] * double(zw[f][t][m]);
                    o += ws[f].w[2] * fabs(acc);
                }
                os[f][x + (int64_t)(ya + t) * sy + (int64_t)z * sz] = F(o);
            }
        }
    }
    asm volatile("cp.async.wait_group 0;" ::: "memory");
}

template <typename F, int NF>
__global__ void __launch_bounds__(kD4Threads) k_delta4_tiled(const F* __restrict__ f0, const F* __restrict__ f1,
                                                           F* __restrict__ o0, F* __restrict__ o1, Grid3 g,
                                                           Weights3 w0, Weights3 w1) {
    extern __shared__ __align__(16) unsigned char d4_raw[];
    delta4_tile<F, NF>(f0, f1, o0, o1, g, w0, w1, blockIdx.x * kTX, blockIdx.y * kTY, blockIdx.z * kZC,
                       reinterpret_cast<F*>(d4_raw));
}

// delta4_sum! of one or two fields on a rank's block of a decomposed grid
// (src/artificial.jl:67-94 after exchange_halos!): the same sums in the same
// order as k_delta4, with the neighbours beyond an open end of a split
// dimension read from the exchanged planes.
template <typename F, int NF>
__global__ void k_delta4_halo(const F* __restrict__ f0, const F* __restrict__ f1, F* __restrict__ o0,
                              F* __restrict__ o1, Grid3 g, Weights3 w0, Weights3 w1, Halo4 h) {
    const int64_t cells = (int64_t)g.n[0] * g.n[1] * g.n[2];
    const double D4[5] = {1.0, -4.0, 6.0, -4.0, 1.0};
    const int64_t st[3] = {1, (int64_t)g.n[0], (int64_t)g.n[0] * g.n[1]};
    const F* fs[2] = {f0, f1};
    F* os[2] = {o0, o1};
    const Weights3 ws[2] = {w0, w1};
    GRID_STRIDE(I, cells) {
        const int i = (int)(I % g.n[0]);
        const int j = (int)((I / g.n[0]) % g.n[1]);
        const int k = (int)(I / ((int64_t)g.n[0] * g.n[1]));
        const int ijk[3] = {i, j, k};
        // line index and line count of each dimension (split_halo's numbering)
        const int64_t line[3] = {j + (int64_t)k * g.n[1], i + (int64_t)k * g.n[0], i + (int64_t)j * g.n[0]};
        const int64_t lines[3] = {(int64_t)g.n[1] * g.n[2], (int64_t)g.n[0] * g.n[2], (int64_t)g.n[0] * g.n[1]};
#pragma unroll
        for (int f = 0; f < NF; ++f) {
            double o = 0.0;
            for (int d = 0; d < 3; ++d) {
                if (!g.active[d]) continue;
                const int nd = g.n[d];
                const int il = ijk[d];
                double acc = 0.0;
#pragma unroll
                for (int m = -2; m <= 2; ++m) {
                    const int ilm = il + m;
                    double v;
                    if (ilm < 0 && h.open_lo[d]) {
                        v = double(static_cast<const F*>(h.lo[d])[(int64_t)(2 * f + ilm + 2) * lines[d] + line[d]]);
                    } else if (ilm >= nd && h.open_hi[d]) {
                        v = double(static_cast<const F*>(h.hi[d])[(int64_t)(2 * f + ilm - nd) * lines[d] + line[d]]);
                    } else {
                        int e = ilm;
                        if (g.periodic[d]) e = e < 0 ? e + nd : (e >= nd ? e - nd : e);
                        else e = e < 0 ? 0 : (e >= nd ? nd - 1 : e);
                        v = double(fs[f][I + (int64_t)(e - il) * st[d]]);
                    }
                    acc += D4[m + 2] * v;
                }
                o += ws[f].w[d] * fabs(acc);
            }
            os[f][I] = F(o);
        }
    }
}

// Ducros switch (src/artificial.jl:134-147)
__device__ __forceinline__ double compression_switch(const double* gv) {
    const double div = gv[0] + gv[4] + gv[8];
    if (!(div < 0)) return 0.0;
    const double w1 = gv[3 * 1 + 2] - gv[3 * 2 + 1];
    const double w2 = gv[3 * 2 + 0] - gv[3 * 0 + 2];
    const double w3 = gv[3 * 0 + 1] - gv[3 * 1 + 0];
    return div * div / (div * div + w1 * w1 + w2 * w2 + w3 * w3 + 1e-32);
}

// mu*, beta* from the smoothed strain sensor (src/artificial.jl:306-313),
// optional gating (gate_beta!, :164-175).
template <typename F>
__global__ void k_mu_beta(const F* __restrict__ sensor, const F* __restrict__ prim, const F* __restrict__ g,
                          F* __restrict__ art, int64_t cells, double C_mu, double C_beta, int gate) {
    GRID_STRIDE(I, cells) {
        const double rs = double(prim[I + cells * P_RHO]) * jl_max(double(sensor[I]), 0.0);
        double beta = C_beta * rs;
        if (gate) {
            double gv[9];
            for (int k = 0; k < 9; ++k) gv[k] = double(g[I + cells * k]);
            beta *= compression_switch(gv);
        }
        art[I + cells * A_MU] = F(C_mu * rs);
        art[I + cells * A_BETA] = F(beta);
    }
}

// mu*, beta* (optionally gated) and kappa* from the two smoothed sensors in one
// pass (src/artificial.jl:306-313 and :334-341).
template <typename F>
__global__ void k_art_coef(const F* __restrict__ s_strain, const F* __restrict__ s_energy, const F* __restrict__ prim,
                           const F* __restrict__ g, F* __restrict__ art, int64_t cells, double C_mu, double C_beta,
                           double C_kappa, int gate) {
    GRID_STRIDE(I, cells) {
        const double rho = double(prim[I + cells * P_RHO]);
        const double rs = rho * jl_max(double(s_strain[I]), 0.0);
        double beta = C_beta * rs;
        if (gate) {
            double gv[9];
            for (int k = 0; k < 9; ++k) gv[k] = double(g[I + cells * k]);
            beta *= compression_switch(gv);
        }
        art[I + cells * A_MU] = F(C_mu * rs);
        art[I + cells * A_BETA] = F(beta);
        const double scale = rho * double(prim[I + cells * P_C]) / jl_max(double(prim[I + cells * P_T]), 2.220446049250313e-16);
        art[I + cells * A_KAPPA] = F(C_kappa * scale * jl_max(double(s_energy[I]), 0.0));
    }
}

// dilatation and switch for the :dilatation beta sensor (src/artificial.jl:208-218)
template <typename F>
__global__ void k_dilatation(const F* __restrict__ g, F* __restrict__ div, F* __restrict__ sw, int64_t cells) {
    GRID_STRIDE(I, cells) {
        double gv[9];
        for (int k = 0; k < 9; ++k) gv[k] = double(g[I + cells * k]);
        div[I] = F(gv[0] + gv[4] + gv[8]);
        sw[I] = F(compression_switch(gv));
    }
}

template <typename F>
__global__ void k_beta_dilatation(const F* __restrict__ sensor, const F* __restrict__ prim, const F* __restrict__ sw,
                                  F* __restrict__ art, int64_t cells, double C_beta) {
    GRID_STRIDE(I, cells) {
        art[I + cells * A_BETA] =
            F(C_beta * double(prim[I + cells * P_RHO]) * jl_max(double(sensor[I]), 0.0) * double(sw[I]));
    }
}

// internal energy e = (E - |m|^2/2rho)/rho with rho floored (src/artificial.jl:322-330)
template <typename F>
__global__ void k_energy(const double* __restrict__ Q, const F* __restrict__ prim, F* __restrict__ out, int64_t cells,
                         int Ns) {
    GRID_STRIDE(I, cells) {
        const double r = jl_max(double(prim[I + cells * P_RHO]), 1e-300);
        const double q1 = Q[I + cells * (Ns + 0)], q2 = Q[I + cells * (Ns + 1)], q3 = Q[I + cells * (Ns + 2)];
        const double ke = 0.5 * (q1 * q1 + q2 * q2 + q3 * q3) / r;
        out[I] = F((Q[I + cells * (Ns + 3)] - ke) / r);
    }
}

// kappa* = C_kappa (rho c / max(T, eps)) max(sensor, 0) (src/artificial.jl:334-341, src/physics.jl:155-156)
template <typename F>
__global__ void k_kappa(const F* __restrict__ sensor, const F* __restrict__ prim, F* __restrict__ art, int64_t cells,
                        double C_kappa) {
    GRID_STRIDE(I, cells) {
        const double scale = double(prim[I + cells * P_RHO]) * double(prim[I + cells * P_C]) /
                             jl_max(double(prim[I + cells * P_T]), 2.220446049250313e-16);
        art[I + cells * A_KAPPA] = F(C_kappa * scale * jl_max(double(sensor[I]), 0.0));
    }
}

// D*_k = C_D c max(sensor_k, 0) (src/artificial.jl:348-356)
template <typename F>
__global__ void k_dart(const F* __restrict__ sensor, const F* __restrict__ prim, F* __restrict__ art, int64_t cells,
                       double C_D, int sp) {
    GRID_STRIDE(I, cells) {
        art[I + cells * (A_D0 + sp)] = F(C_D * double(prim[I + cells * P_C]) * jl_max(double(sensor[I]), 0.0));
    }
}

// _assemble_fluxes! (src/rhs.jl:495-556).  gty[d*(1+Ns) + 0] = dT/dx_d,
// gty[d*(1+Ns) + 1 + k] = dY_k/dx_d; flux[d*ncons + c].
// SINGLE (one species): the species diffusion flux rho D dY (Y - 1) is zero in
// exact arithmetic (Y = 1) and below ~1e-30 of the momentum flux in FP64, so it
// is taken as 0 and dY/dx_d is neither computed nor read (gty holds dT only).
template <typename F, bool SINGLE, bool N9, bool GEO, bool PM = false>
__global__ void k_fluxes(const double* __restrict__ Q, const F* __restrict__ prim, const F* __restrict__ g,
                         const F* __restrict__ gty, const F* __restrict__ art, F* __restrict__ flux, int64_t cells,
                         int Ns, PhysConst pc, double mu0, double Pr, double Sc, Geom G,
                         const double* __restrict__ mc = nullptr, const int* __restrict__ tmap = nullptr) {
    if (SINGLE) Ns = 1;
    const int ncons = Ns + 4;
    const int gstride = SINGLE ? 1 : 1 + Ns;
    GRID_STRIDE(I, cells) {
        // curvilinear / stretched grids store A_d F_d (src/rhs.jl:670-675)
        double area[3] = {1.0, 1.0, 1.0};
        if (GEO) {
            int i, j, k;
            cell_ijk(I, G.n, i, j, k);
            const GeoPoint gp = geo_point(G, i, j, k, I);
            area[0] = gp.A[0];
            area[1] = gp.A[1];
            area[2] = gp.A[2];
        }
#define CLES_AF(v) (GEO ? __dmul_rn(ad, (v)) : (v))
        double gv[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) gv[k] = double(g[I + cells * k]);
        const double r = double(prim[I + cells * P_RHO]);
        const double uv[3] = {double(prim[I + cells * P_U]), double(prim[I + cells * P_V]), double(prim[I + cells * P_W])};
        const double p = double(prim[I + cells * P_P]);
        const double Tp = double(prim[I + cells * P_T]);
        const double E = Q[I + cells * (Ns + 3)];
        const double mu = mu0 + double(art[I + cells * A_MU]);
        const double be = double(art[I + cells * A_BETA]);
        const double ka = mu0 * double(prim[I + cells * P_CP]) / Pr + double(art[I + cells * A_KAPPA]);
        const double D0 = mu0 / (Sc * r);
        const double divu = gv[0] + gv[4] + gv[8];
        const double t11 = mu * (2 * gv[0] - (2.0 / 3.0) * divu) + be * divu;
        const double t22 = mu * (2 * gv[4] - (2.0 / 3.0) * divu) + be * divu;
        const double t33 = mu * (2 * gv[8] - (2.0 / 3.0) * divu) + be * divu;
        const double t12 = mu * (gv[1] + gv[3]);
        const double t13 = mu * (gv[2] + gv[6]);
        const double t23 = mu * (gv[5] + gv[7]);
        const double tau[3][3] = {{t11, t12, t13}, {t12, t22, t23}, {t13, t23, t33}};
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const double ud = uv[d];
            const double ad = area[d];
            const double* td = tau[d];
            const F* gd = gty + cells * (int64_t)(d * gstride);
            F* fd = flux + cells * (int64_t)(d * ncons);
            double hdiff = 0.0;
            if (SINGLE) {
                const double Yk = double(prim[I + cells * P_Y0]);
                const double f0 = r * Yk * ud;
                fd[I] = F(CLES_AF(f0));
            } else {
                double Vc = 0.0;
                for (int sp = 0; sp < Ns; ++sp)
                    Vc += (D0 + double(art[I + cells * (A_D0 + sp)])) * double(gd[I + cells * (1 + sp)]);
                for (int sp = 0; sp < Ns; ++sp) {
                    const double Dk = D0 + double(art[I + cells * (A_D0 + sp)]);
                    const double Yk = double(prim[I + cells * (P_Y0 + sp)]);
                    const double Jkd = r * (-Dk * double(gd[I + cells * (1 + sp)]) + Yk * Vc);
                    const double fk = r * Yk * ud + Jkd;
                    fd[I + cells * sp] = F(CLES_AF(fk));
                    if constexpr (PM) hdiff += mc[24 * tmap[I >> 6] + 16 + sp] * Tp * Jkd;
                    else hdiff += (N9 ? n9_h(pc, sp, Tp) : pc.cpk[sp] * Tp) * Jkd;
                }
            }
            const double m0 = r * ud * uv[0] + (d == 0 ? p : 0.0) - td[0];
            const double m1 = r * ud * uv[1] + (d == 1 ? p : 0.0) - td[1];
            const double m2 = r * ud * uv[2] + (d == 2 ? p : 0.0) - td[2];
            const double en = (E + p) * ud - (uv[0] * td[0] + uv[1] * td[1] + uv[2] * td[2]) - ka * double(gd[I]) + hdiff;
            fd[I + cells * (Ns + 0)] = F(CLES_AF(m0));
            fd[I + cells * (Ns + 1)] = F(CLES_AF(m1));
            fd[I + cells * (Ns + 2)] = F(CLES_AF(m2));
            fd[I + cells * (Ns + 3)] = F(CLES_AF(en));
        }
    }
#undef CLES_AF
}

// add_source!(::ConstantBodyForce) (src/sources.jl:42-65) for every body force
// in order; products rounded separately as in the reference.
template <typename F>
__global__ void k_body_forces(F* __restrict__ dQ, const double* __restrict__ Q, int64_t cells, int Ns, BodyForces bf) {
    GRID_STRIDE(I, cells) {
        double rho = 0.0;
        for (int sp = 0; sp < Ns; ++sp) rho += Q[I + cells * sp];
        const double q1 = Q[I + cells * Ns], q2 = Q[I + cells * (Ns + 1)], q3 = Q[I + cells * (Ns + 2)];
        double m[3] = {double(dQ[I + cells * Ns]), double(dQ[I + cells * (Ns + 1)]), double(dQ[I + cells * (Ns + 2)])};
        double e = double(dQ[I + cells * (Ns + 3)]);
        for (int f = 0; f < bf.n; ++f) {
            for (int a = 0; a < 3; ++a) m[a] = m[a] + __dmul_rn(rho, bf.g[f][a]);
            e = e + ((__dmul_rn(q1, bf.g[f][0]) + __dmul_rn(q2, bf.g[f][1])) + __dmul_rn(q3, bf.g[f][2]));
            if (sizeof(F) == 4) {
                // the stored RHS is FP32: round between sources as the stores do
                for (int a = 0; a < 3; ++a) m[a] = double(F(m[a]));
                e = double(F(e));
            }
        }
        for (int a = 0; a < 3; ++a) dQ[I + cells * (Ns + a)] = F(m[a]);
        dQ[I + cells * (Ns + 3)] = F(e);
    }
}

// Low-storage RK update (src/timestep.jl:86-95): v = A du + dt dQ; du = v; Q += B v.
template <typename F>
__global__ void k_lsrk(double* __restrict__ Q, double* __restrict__ du, const F* __restrict__ dQ, int64_t n, double A,
                       double B, double dt, const double* __restrict__ dtp) {
    if (dtp) dt = *dtp;
    GRID_STRIDE(I, n) {
        const double v = A * du[I] + dt * double(dQ[I]);
        du[I] = v;
        Q[I] += B * v;
    }
}

// The max_rate contribution of cell I (src/timestep.jl:125-175), Cartesian;
// fields are `cells` elements apart.
template <typename F>
__device__ __forceinline__ void rate_cell(const double* __restrict__ Q, const F* __restrict__ prim,
                                          const F* __restrict__ art, int64_t I, int64_t cells, int Ns,
                                          const double idx[3], const int act[3], double mu0, double Pr, double Sc,
                                          double& rate, double& rmin) {
    {
        double rq = 0.0;
        for (int sp = 0; sp < Ns; ++sp) rq += Q[I + cells * sp];
        rmin = jl_min(rmin, rq);
        const double r = double(prim[I + cells * P_RHO]);
        const double ri = 1 / r;
        const double c = double(prim[I + cells * P_C]);
        const double cp = double(prim[I + cells * P_CP]);
        const double uv[3] = {double(prim[I + cells * P_U]), double(prim[I + cells * P_V]), double(prim[I + cells * P_W])};
        double acc = 0.0, dsum = 0.0;
        for (int d = 0; d < 3; ++d) {
            if (!act[d]) continue;
            acc += (fabs(uv[d]) + c) * idx[d];
            dsum += idx[d] * idx[d];
        }
        double Dmax = mu0 / (Sc * r);
        for (int sp = 0; sp < Ns; ++sp) Dmax = jl_max(Dmax, mu0 / (Sc * r) + double(art[I + cells * (A_D0 + sp)]));
        const double nu = (mu0 + double(art[I + cells * A_MU]) + double(art[I + cells * A_BETA])) * ri +
                          (mu0 * cp / Pr + double(art[I + cells * A_KAPPA])) * ri / cp + Dmax;
        acc += 2 * nu * dsum;
        rate = jl_max(rate, acc);
    }
}

// Block max / min of (rate, rmin) into part[2 b], part[2 b + 1] (max / min are
// exact, so the order does not matter).
__device__ __forceinline__ void rate_block_reduce(double rate, double rmin, double* __restrict__ part, int b) {
    __shared__ double sr[kThreads], sm[kThreads];
    sr[threadIdx.x] = rate;
    sm[threadIdx.x] = rmin;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) {
            sr[threadIdx.x] = jl_max(sr[threadIdx.x], sr[threadIdx.x + s]);
            sm[threadIdx.x] = jl_min(sm[threadIdx.x], sm[threadIdx.x + s]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        part[2 * b] = sr[0];
        part[2 * b + 1] = sm[0];
    }
}

// max_rate per-block partials (src/timestep.jl:125-175), Cartesian.
template <typename F>
__global__ void k_rate_partial(const double* __restrict__ Q, const F* __restrict__ prim, const F* __restrict__ art,
                               double* __restrict__ part, int64_t cells, int Ns, double idx0, double idx1, double idx2,
                               int a0, int a1, int a2, double mu0, double Pr, double Sc) {
    double rate = 0.0, rmin = __longlong_as_double(0x7ff0000000000000LL);
    const double idx[3] = {idx0, idx1, idx2};
    const int act[3] = {a0, a1, a2};
    GRID_STRIDE(I, cells) rate_cell(Q, prim, art, I, cells, Ns, idx, act, mu0, Pr, Sc, rate, rmin);
    rate_block_reduce(rate, rmin, part, blockIdx.x);
}

__global__ void k_rate_final(const double* __restrict__ part, int nb, double* __restrict__ out) {
    __shared__ double sr[kThreads], sm[kThreads];
    double rate = 0.0, rmin = __longlong_as_double(0x7ff0000000000000LL);
    for (int b = threadIdx.x; b < nb; b += blockDim.x) {
        rate = jl_max(rate, part[2 * b]);
        rmin = jl_min(rmin, part[2 * b + 1]);
    }
    sr[threadIdx.x] = rate;
    sm[threadIdx.x] = rmin;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) {
            sr[threadIdx.x] = jl_max(sr[threadIdx.x], sr[threadIdx.x + s]);
            sm[threadIdx.x] = jl_min(sm[threadIdx.x], sm[threadIdx.x + s]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) { out[0] = sr[0]; out[1] = sm[0]; }
}

// Fixed-order sums (deterministic) for diagnostics: per-block partials then one block.
template <typename F>
__global__ void k_ke_partial(const double* __restrict__ Q, double* __restrict__ part, int64_t cells, int Ns) {
    __shared__ double s[kThreads];
    double acc = 0.0;
    GRID_STRIDE(I, cells) {
        double r = 0.0;
        for (int sp = 0; sp < Ns; ++sp) r += Q[I + cells * sp];
        const double q1 = Q[I + cells * (Ns + 0)], q2 = Q[I + cells * (Ns + 1)], q3 = Q[I + cells * (Ns + 2)];
        acc += 0.5 * (q1 * q1 + q2 * q2 + q3 * q3) / r;
    }
    s[threadIdx.x] = acc;
    __syncthreads();
    for (int st = blockDim.x / 2; st > 0; st >>= 1) {
        if ((int)threadIdx.x < st) s[threadIdx.x] += s[threadIdx.x + st];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = s[0];
}

// quad-weighted sum of tau:grad u and of rho (dissipation_rate, src/diagnostics.jl:354-378)
template <typename F>
__global__ void k_diss_partial(const F* __restrict__ prim, const F* __restrict__ g, const F* __restrict__ art,
                               double* __restrict__ part, Grid3 gr, double mu0, Geom Gm, int geo, unsigned foldmask) {
    __shared__ double s1[kThreads], s2[kThreads];
    const int64_t cells = (int64_t)gr.n[0] * gr.n[1] * gr.n[2];
    double a1 = 0.0, a2 = 0.0;
    GRID_STRIDE(I, cells) {
        const int i = (int)(I % gr.n[0]);
        const int j = (int)((I / gr.n[0]) % gr.n[1]);
        const int k = (int)(I / ((int64_t)gr.n[0] * gr.n[1]));
        const int ijk[3] = {i, j, k};
        // quad_weight (src/diagnostics.jl:41-49): 1/2 on a node-centred closed
        // edge, 1 on a folded (half-offset) one
        double w = 1.0;
        for (int d = 0; d < 3; ++d) {
            if (!gr.active[d] || gr.periodic[d]) continue;
            if (ijk[d] == 0 && !((foldmask >> (2 * d)) & 1u)) w *= 0.5;
            else if (ijk[d] == gr.n[d] - 1 && !((foldmask >> (2 * d + 1)) & 1u)) w *= 0.5;
        }
        // the metric Jacobian J = 1/inv_J (src/diagnostics.jl:73-75)
        const double ij = geo ? geo_point(Gm, i, j, k, I).inv_J : 1.0;
        double gv[9];
        for (int q = 0; q < 9; ++q) gv[q] = double(g[I + cells * q]);
        const double mu = mu0 + double(art[I + cells * A_MU]);
        const double be = double(art[I + cells * A_BETA]);
        const double divu = gv[0] + gv[4] + gv[8];
        double acc = 0.0;
        for (int b = 0; b < 3; ++b)
            for (int a = 0; a < 3; ++a) {
                const double tau = mu * (gv[3 * a + b] + gv[3 * b + a]) + (a == b ? (be - 2 * mu / 3) * divu : 0.0);
                acc += tau * gv[3 * a + b];
            }
        a1 += w * acc / ij;
        a2 += w * double(prim[I + cells * P_RHO]) / ij;
    }
    s1[threadIdx.x] = a1;
    s2[threadIdx.x] = a2;
    __syncthreads();
    for (int st = blockDim.x / 2; st > 0; st >>= 1) {
        if ((int)threadIdx.x < st) { s1[threadIdx.x] += s1[threadIdx.x + st]; s2[threadIdx.x] += s2[threadIdx.x + st]; }
        __syncthreads();
    }
    if (threadIdx.x == 0) { part[2 * blockIdx.x] = s1[0]; part[2 * blockIdx.x + 1] = s2[0]; }
}

__global__ void k_sum_final(const double* __restrict__ part, int nb, int width, double* __restrict__ out) {
    __shared__ double s[kThreads];
    for (int c = 0; c < width; ++c) {
        double acc = 0.0;
        for (int b = threadIdx.x; b < nb; b += blockDim.x) acc += part[(int64_t)width * b + c];
        s[threadIdx.x] = acc;
        __syncthreads();
        for (int st = blockDim.x / 2; st > 0; st >>= 1) {
            if ((int)threadIdx.x < st) s[threadIdx.x] += s[threadIdx.x + st];
            __syncthreads();
        }
        if (threadIdx.x == 0) out[c] = s[0];
        __syncthreads();
    }
}

// enforce!(::SlipWallBC) (src/boundary.jl:232-243) and a time-constant
// DirichletBC (src/problem.jl:209-221) on the wall plane of (d, side).
// The plane of face (d, side) of one grid whose fields are `cells` elements
// apart, threads t0, t0 + tstep, ... of it.
__device__ __forceinline__ void bc_plane_body(double* __restrict__ Q, const Grid3& g, const int64_t cells, int d,
                                              int side, int Ns, int kind, const BcState& st,
                                              const double* __restrict__ qface, int64_t t0, int64_t tstep) {
    const int o1 = d == 0 ? 1 : 0, o2 = d == 2 ? 1 : 2;
    const int64_t plane = (int64_t)g.n[o1] * g.n[o2];
    const int64_t stv[3] = {1, (int64_t)g.n[0], (int64_t)g.n[0] * g.n[1]};
    const int wall = side == 0 ? 0 : g.n[d] - 1;
    for (int64_t t = t0; t < plane; t += tstep) {
        const int a = (int)(t % g.n[o1]), b = (int)(t / g.n[o1]);
        const int64_t I = a * stv[o1] + b * stv[o2] + (int64_t)wall * stv[d];
        if (kind == CLES_BC_SLIPWALL) {
            double r = 0.0;
            for (int sp = 0; sp < Ns; ++sp) r += Q[I + cells * sp];
            const int mc = Ns + d;
            const double mn = Q[I + cells * mc];
            Q[I + cells * (Ns + 3)] -= 0.5 * mn * mn / r;
            Q[I + cells * mc] = 0;
        } else if (kind == CLES_BC_NOSLIP_WALL) {
            // enforce!(::NoSlipWallBC) (src/boundary.jl:245-265)
            double r = 0.0;
            for (int sp = 0; sp < Ns; ++sp) r += Q[I + cells * sp];
            const double m1 = Q[I + cells * Ns], m2 = Q[I + cells * (Ns + 1)], m3 = Q[I + cells * (Ns + 2)];
            const double ke = 0.5 * (m1 * m1 + m2 * m2 + m3 * m3) / r;
            Q[I + cells * (Ns + 3)] -= ke;
            Q[I + cells * Ns] = 0;
            Q[I + cells * (Ns + 1)] = 0;
            Q[I + cells * (Ns + 2)] = 0;
            if (st.iso) {
                // wall_internal_energy (src/boundary.jl:194-211)
                double re = 0.0;
                for (int sp = 0; sp < Ns; ++sp) re += Q[I + cells * sp] * st.ew[sp];
                Q[I + cells * (Ns + 3)] = st.ew_times_T ? re * st.Twall : re;
            }
        } else if (kind == CLES_BC_EXTRAPOLATION) {
            // enforce!(::ExtrapolationBC) (src/boundary.jl:267-278): copy the adjacent interior plane
            const int64_t J = I + (side == 0 ? stv[d] : -stv[d]);
            for (int c = 0; c < Ns + 4; ++c) Q[I + cells * c] = Q[J + cells * c];
        } else if (qface) {
            // DirichletBC(fun): the stage-time state per node ([c][plane])
            for (int c = 0; c < Ns + 4; ++c) Q[I + cells * c] = qface[c * plane + t];
        } else {
            for (int c = 0; c < Ns + 4; ++c) Q[I + cells * c] = st.q[c];
        }
    }
}

__global__ void k_bc_plane(double* __restrict__ Q, Grid3 g, int d, int side, int Ns, int kind, BcState st,
                           const double* __restrict__ qface) {
    const int64_t cells = (int64_t)g.n[0] * g.n[1] * g.n[2];
    bc_plane_body(Q, g, cells, d, side, Ns, kind, st, qface, blockIdx.x * (int64_t)blockDim.x + threadIdx.x,
                  (int64_t)gridDim.x * blockDim.x);
}

// correct_rhs!(::NSCBCOutflowBC) (src/nscbc.jl:59-157) and
// correct_rhs!(::NSCBCInflowBC) (src/nscbc.jl:220-307): LODI wave-amplitude
// corrections of dQ on one boundary plane.  Inflow targets are the constants
// of bp, or per node from tgt ([velocity 0..2, T, Y_k][plane], the stage-time
// target function's values) when tgt is set.
template <typename F, bool N9>
__global__ void k_nscbc(F* __restrict__ dQ, const F* __restrict__ prim, const F* __restrict__ g,
                        const F* __restrict__ gty, int ngty, const F* __restrict__ dpd, const F* __restrict__ dpt0,
                        const F* __restrict__ dpt1, const F* __restrict__ drd, Grid3 gr, int d, int side, int Ns,
                        PhysConst pc, NscbcParams bp, const double* __restrict__ tgt, Geom Gm, int geo) {
    const int o1 = d == 0 ? 1 : 0, o2 = d == 2 ? 1 : 2;
    const int64_t plane = (int64_t)gr.n[o1] * gr.n[o2];
    const int64_t cells = (int64_t)gr.n[0] * gr.n[1] * gr.n[2];
    const int64_t stv[3] = {1, (int64_t)gr.n[0], (int64_t)gr.n[0] * gr.n[1]};
    const int wall = side == 0 ? 0 : gr.n[d] - 1;
    const int t1 = d == 0 ? 1 : 0, t2 = d == 2 ? 1 : 2;   // transverse dims
    GRID_STRIDE(q, plane) {
        const int a = (int)(q % gr.n[o1]), b = (int)(q / gr.n[o1]);
        const int64_t I = a * stv[o1] + b * stv[o2] + (int64_t)wall * stv[d];
        auto P = [&](int slot) { return double(prim[I + cells * slot]); };
        auto G = [&](int dd, int j) { return double(g[I + cells * (3 * dd + j)]); };
        const double rho = P(P_RHO), c = P(P_C), p = P(P_P), Tp = P(P_T), cpm = P(P_CP);
        const double uv[3] = {P(P_U), P(P_V), P(P_W)};
        const double un = uv[d];
        const double Ma = fabs(un) / c;
        if (!(Ma < 1)) continue;   // supersonic: no correction
        // physical derivatives: 1/h of the normal and transverse dims
        // (1 on a uniform Cartesian grid; src/nscbc.jl:108, :125-130, :257)
        double ihd = 1.0, iht1 = 1.0, iht2 = 1.0;
        if (geo) {
            int ci, cj, ck;
            cell_ijk(I, gr.n, ci, cj, ck);
            const GeoPoint gp = geo_point(Gm, ci, cj, ck, I);
            ihd = gp.inv_h[d];
            iht1 = gp.inv_h[t1];
            iht2 = gp.inv_h[t2];
        }
        const double dpn = geo ? ihd * double(dpd[I]) : double(dpd[I]);
        const double dun = G(d, d);
        const double Rm = p / (rho * Tp);
        const double phi = cpm / Rm - 1;   // eos_phi, either mixture (src/physics.jl:142-145, 457-460)
        const double ke = 0.5 * (uv[0] * uv[0] + uv[1] * uv[1] + uv[2] * uv[2]);
        const int m0 = Ns, ie = Ns + 3;
        if (bp.kind == CLES_BC_NSCBC_OUTFLOW) {
            const double sgn = side == 1 ? -1.0 : 1.0;
            const double Lcomp = side == 1 ? (un - c) * (dpn - rho * c * dun) : (un + c) * (dpn + rho * c * dun);
            double tin = 0.0;
            if (bp.act[t1]) {
                const double ut = uv[t1];
                tin += ut * iht1 * double(dpt0[I]) + rho * c * c * G(t1, t1) + sgn * rho * c * ut * G(t1, d);
            }
            if (bp.act[t2]) {
                const double ut = uv[t2];
                tin += ut * iht2 * double(dpt1[I]) + rho * c * c * G(t2, t2) + sgn * rho * c * ut * G(t2, d);
            }
            const double bt = bp.beta_t < 0 ? Ma : bp.beta_t;
            const double K = bp.sigma * (1 - Ma * Ma) * c / bp.Lref;
            const double dL = K * (p - bp.pinf) - bt * tin - Lcomp;
            const double d1 = dL / (2 * c * c);
            const double d2 = dL / 2;
            const double d3 = sgn * dL / (2 * rho * c);
            for (int k = 0; k < Ns; ++k) dQ[I + cells * k] = F(double(dQ[I + cells * k]) - P(P_Y0 + k) * d1);
            for (int aa = 0; aa < 3; ++aa)
                dQ[I + cells * (m0 + aa)] =
                    F(double(dQ[I + cells * (m0 + aa)]) - (uv[aa] * d1 + (aa == d ? rho * d3 : 0.0)));
            dQ[I + cells * ie] = F(double(dQ[I + cells * ie]) - (ke * d1 + phi * d2 + rho * un * d3));
        } else {
            const bool low = side == 0;
            const double drn = geo ? ihd * double(drd[I]) : double(drd[I]);
            const double K = c / bp.Lref;
            const double L1c = (un - c) * (dpn - rho * c * dun);
            const double L5c = (un + c) * (dpn + rho * c * dun);
            const double L2c = un * (c * c * drn - dpn);
            double uT[3] = {bp.u[0], bp.u[1], bp.u[2]}, TT = bp.T;
            if (tgt) {
                for (int aa = 0; aa < 3; ++aa) uT[aa] = tgt[aa * plane + q];
                TT = tgt[3 * plane + q];
            }
            auto YT = [&](int k) { return tgt ? tgt[(4 + k) * plane + q] : bp.Y[k]; };
            const double rel = bp.eta_u * rho * c * c * (1 - Ma * Ma) / bp.Lref * (un - uT[d]);
            const double dL1 = low ? 0.0 : (-rel - L1c);
            const double dL5 = low ? (rel - L5c) : 0.0;
            const double dL2 = bp.eta_T * rho * (c * c * c) * (TT - Tp) / (bp.Lref * Tp) - L2c;
            const double d1 = dL2 / (c * c) + (dL5 + dL1) / (2 * c * c);
            const double d2 = (dL5 + dL1) / 2;
            const double d3 = (dL5 - dL1) / (2 * rho * c);
            const double d4 = bp.eta_t * K * (uv[t1] - uT[t1]) - un * G(d, t1);
            const double d5 = bp.eta_t * K * (uv[t2] - uT[t2]) - un * G(d, t2);
            const double cvm = cpm - Rm;
            double sphiY = 0.0;
            for (int k = 0; k < Ns; ++k) {
                const double Yk = P(P_Y0 + k);
                const double gY = ngty > 1 ? double(gty[I + cells * (d * ngty + 1 + k)]) : 0.0;
                const double dLs = bp.eta_Y * K * (Yk - YT(k)) - un * gY;
                dQ[I + cells * k] = F(double(dQ[I + cells * k]) - (Yk * d1 + rho * dLs));
                // eos_dphi_dY (src/physics.jl:147-152, 462-470)
                const double cvk = N9 ? n9_cp(pc, k, Tp) - pc.Rk[k] : pc.cvk[k];
                sphiY += (cvk * Rm - pc.Rk[k] * cvm) / (Rm * Rm) * dLs;
            }
            for (int aa = 0; aa < 3; ++aa) {
                const double extra = aa == d ? rho * d3 : (aa == t1 ? rho * d4 : rho * d5);
                dQ[I + cells * (m0 + aa)] = F(double(dQ[I + cells * (m0 + aa)]) - (uv[aa] * d1 + extra));
            }
            dQ[I + cells * ie] = F(double(dQ[I + cells * ie]) -
                                   (ke * d1 + phi * d2 + p * sphiY + rho * (un * d3 + uv[t1] * d4 + uv[t2] * d5)));
        }
    }
}

__global__ void k_gather_interior(const double* __restrict__ padded, double* __restrict__ interior, int n0, int n1,
                                  int n2, int p0, int p1, int p2) {
    const int64_t cells = (int64_t)n0 * n1 * n2;
    const int64_t F0 = n0 + 2 * p0, F1 = n1 + 2 * p1;
    GRID_STRIDE(I, cells) {
        const int64_t i = I % n0, r = I / n0;
        const int64_t j = r % n1, k = r / n1;
        interior[I] = padded[(i + p0) + F0 * ((j + p1) + F1 * (k + p2))];
    }
}

template <typename F>
__global__ void k_convert(const double* __restrict__ a, F* __restrict__ b, int64_t n) {
    GRID_STRIDE(I, n) b[I] = F(a[I]);
}

template <typename F>
__global__ void k_to_double(const F* __restrict__ a, double* __restrict__ b, int64_t n) {
    GRID_STRIDE(I, n) b[I] = double(a[I]);
}

// Device clock of the graph-mode run loop (one thread).  clk layout: see
// DeviceClock in pointwise.h.  Before the step: dt from the reduced rate
// (predicted_dt without prediction or growth cap), the check_step floors
// (src/stepcontrol.jl:184-204), dt_seen, and the tfinal clip
// (src/timestep.jl:288-352).
__device__ __forceinline__ void clock_before_body(double* __restrict__ clk, const double rate, const double rmin,
                                                  const ClockConst& c) {
    if (clk[DC_FAILURE] != 0.0 || clk[DC_DONE] != 0.0) { clk[DC_DT] = 0.0; return; }
    double dt = c.cfl / rate;
    int f = 0;
    if (!isfinite(dt)) f = CLES_FAIL_NONFINITE;
    else if (!(rmin > 0)) f = CLES_FAIL_NEGATIVE_DENSITY;
    else if (!(dt > 5.391247e-44)) f = CLES_FAIL_PLANCK;
    else if (!(dt >= c.dt_min)) f = CLES_FAIL_DT_MIN;
    else if (c.dt_min_ratio > 0 && clk[DC_DT_SEEN] > 0 && !(dt >= c.dt_min_ratio * clk[DC_DT_SEEN])) f = CLES_FAIL_DT_COLLAPSE;
    clk[DC_RATE] = rate;
    clk[DC_RHO_MIN] = rmin;
    if (f) { clk[DC_FAILURE] = f; clk[DC_DT] = 0.0; return; }
    clk[DC_DT_SEEN] = jl_max(clk[DC_DT_SEEN], dt);
    clk[DC_DT] = jl_min(dt, c.tfinal - clk[DC_T]);
}
__global__ void k_clock_before(double* __restrict__ clk, const double* __restrict__ rate_rmin, ClockConst c) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    clock_before_body(clk, rate_rmin[0], rate_rmin[1], c);
}
// After the step: t += dt, step += 1, done when the run! loop condition fails.
__device__ __forceinline__ void clock_after_body(double* __restrict__ clk, const ClockConst& c) {
    if (clk[DC_FAILURE] != 0.0 || clk[DC_DONE] != 0.0) return;
    clk[DC_T] += clk[DC_DT];
    clk[DC_STEP] += 1.0;
    if (!(clk[DC_T] < c.tfinal) || !(clk[DC_STEP] < c.nmax)) clk[DC_DONE] = 1.0;
}
__global__ void k_clock_after(double* __restrict__ clk, ClockConst c) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    clock_after_body(clk, c);
}

// ---- batched forms over the grids of a batch --------------------------------
template <typename F, int NF>
__global__ void __launch_bounds__(kD4Threads) k_delta4_batch(const F* __restrict__ f0, const F* __restrict__ f1,
                                                           F* __restrict__ o0, F* __restrict__ o1, int p0, int p1,
                                                           const BatchGrid* __restrict__ grids,
                                                           const BatchTile* __restrict__ tiles) {
    extern __shared__ __align__(16) unsigned char d4_raw[];
    const BatchTile t = tiles[blockIdx.x];
    const BatchGrid& G = grids[t.grid];
    Weights3 w0, w1;
    for (int d = 0; d < 3; ++d) {
        w0.w[d] = p0 == 2 ? G.h[d] * G.h[d] : G.h[d];
        w1.w[d] = p1 == 2 ? G.h[d] * G.h[d] : G.h[d];
    }
    delta4_tile<F, NF>(f0 + G.off, f1 ? f1 + G.off : nullptr, o0 + G.off, o1 ? o1 + G.off : nullptr, G.g, w0, w1,
                       t.x0, t.y0, t.z0, reinterpret_cast<F*>(d4_raw));
}

template <typename F>
__global__ void k_rate_batch_partial(const double* __restrict__ Q, const F* __restrict__ prim,
                                     const F* __restrict__ art, const BatchGrid* __restrict__ grids,
                                     const BatchChunk* __restrict__ chunks, double* __restrict__ part, int64_t ct,
                                     int Ns, double mu0, double Pr, double Sc) {
    const BatchChunk ch = chunks[blockIdx.x];
    const BatchGrid& G = grids[ch.grid];
    double idx[3];
    int act[3];
    for (int d = 0; d < 3; ++d) { idx[d] = 1.0 / G.h[d]; act[d] = G.g.active[d]; }
    double rate = 0.0, rmin = __longlong_as_double(0x7ff0000000000000LL);
    const int64_t end = min(ch.c0 + (int64_t)kBatchChunk, G.cells);
    for (int64_t c = ch.c0 + threadIdx.x; c < end; c += blockDim.x)
        rate_cell(Q, prim, art, G.off + c, ct, Ns, idx, act, mu0, Pr, Sc, rate, rmin);
    rate_block_reduce(rate, rmin, part, blockIdx.x);
}

// One block per grid: the grid's max / min over its chunk partials, then its clock_before.
__global__ void k_rate_batch_final(const double* __restrict__ part, const int* __restrict__ chunk_first,
                                   const BatchGrid* __restrict__ grids) {
    const int g = blockIdx.x;
    double rate = 0.0, rmin = __longlong_as_double(0x7ff0000000000000LL);
    for (int b = chunk_first[g] + threadIdx.x; b < chunk_first[g + 1]; b += blockDim.x) {
        rate = jl_max(rate, part[2 * b]);
        rmin = jl_min(rmin, part[2 * b + 1]);
    }
    __shared__ double out[2];
    // the same tree as k_rate_final, into out[]
    rate_block_reduce(rate, rmin, out, 0);
    __syncthreads();
    if (threadIdx.x == 0) clock_before_body(grids[g].clk, out[0], out[1], grids[g].cc);
}

__global__ void k_bc_batch(double* __restrict__ Q, const BatchGrid* __restrict__ grids,
                           const BatchFace* __restrict__ faces, int64_t ct, int Ns) {
    const BatchFace& f = faces[blockIdx.x];
    const BatchGrid& G = grids[f.grid];
    bc_plane_body(Q + G.off, G.g, ct, f.d, f.side, Ns, f.kind, f.st, nullptr, threadIdx.x, blockDim.x);
}

// The LSRK update of the members flagged in need[] (whose last divergence did
// not apply it), each with its own dt; fields are ct elements apart.
template <typename F>
__global__ void k_lsrk_batch(double* __restrict__ Q, double* __restrict__ du, const F* __restrict__ dQ, int64_t ct,
                             int ncons, const int* __restrict__ tmap, const BatchGrid* __restrict__ grids,
                             const int* __restrict__ need, double A, double B) {
    GRID_STRIDE(I, ct) {
        const int g = tmap[I >> 6];
        if (!need[g]) continue;
        const double dt = grids[g].clk[DC_DT];
        for (int c = 0; c < ncons; ++c) {
            const int64_t e = I + ct * c;
            const double v = A * du[e] + dt * double(dQ[e]);
            du[e] = v;
            Q[e] += B * v;
        }
    }
}

__global__ void k_clock_after_batch(const BatchGrid* __restrict__ grids, int G) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g < G) clock_after_body(grids[g].clk, grids[g].cc);
}

}  // namespace

void clock_before(double* clk, const double* rate_rmin, const ClockConst& c, cudaStream_t st) {
    k_clock_before<<<1, 32, 0, st>>>(clk, rate_rmin, c);
    count_launch();
    check_launch("k_clock_before");
}
template <typename F>
void BatchOps<F>::delta4(const F* f0, const F* f1, F* o0, F* o1, int p0, int p1, const BatchGrid* grids,
                         const BatchTile* tiles, int ntiles, int64_t, cudaStream_t st) {
    if (ntiles <= 0) return;
    if (f1) {
        constexpr size_t sm = delta4_smem<F, 2>();
        set_smem_attr(k_delta4_batch<F, 2>, sm);
        k_delta4_batch<F, 2><<<ntiles, kD4Threads, sm, st>>>(f0, f1, o0, o1, p0, p1, grids, tiles);
    } else {
        constexpr size_t sm = delta4_smem<F, 1>();
        set_smem_attr(k_delta4_batch<F, 1>, sm);
        k_delta4_batch<F, 1><<<ntiles, kD4Threads, sm, st>>>(f0, f1, o0, o1, p0, p1, grids, tiles);
    }
    count_launch();
    check_launch("k_delta4_batch");
}
template <typename F>
void BatchOps<F>::rate_clock(const double* Q, const F* prim, const F* art, const BatchGrid* grids, int G,
                             const BatchChunk* chunks, int nchunks, const int* chunk_first, double* part,
                             int64_t ct, int Ns, double mu0, double Pr, double Sc, cudaStream_t st) {
    k_rate_batch_partial<F><<<nchunks, kThreads, 0, st>>>(Q, prim, art, grids, chunks, part, ct, Ns, mu0, Pr, Sc);
    count_launch();
    check_launch("k_rate_batch_partial");
    k_rate_batch_final<<<G, kThreads, 0, st>>>(part, chunk_first, grids);
    count_launch();
    check_launch("k_rate_batch_final");
}
template <typename F>
void BatchOps<F>::primitives(const double* Q, F* prim, int64_t ct, int Ns, const PhysConst& pc, int esens,
                             const double* mc, const int* tmap, cudaStream_t st) {
    LAUNCH((k_primitives<F, false, true>), ct, st, Q, prim, ct, Ns, pc, esens, mc, tmap);
}
template <typename F>
void BatchOps<F>::fluxes(const double* Q, const F* prim, const F* g, const F* gty, const F* art, F* flux, int64_t ct,
                         int Ns, const PhysConst& pc, double mu0, double Pr, double Sc, const double* mc,
                         const int* tmap, cudaStream_t st) {
    const Geom G{};
    if (Ns == 1)
        LAUNCH((k_fluxes<F, true, false, false>), ct, st, Q, prim, g, gty, art, flux, ct, Ns, pc, mu0, Pr, Sc, G,
               nullptr, nullptr);
    else
        LAUNCH((k_fluxes<F, false, false, false, true>), ct, st, Q, prim, g, gty, art, flux, ct, Ns, pc, mu0, Pr, Sc,
               G, mc, tmap);
}
template <typename F>
void BatchOps<F>::lsrk(double* Q, double* du, const F* dQ, int64_t ct, int ncons, const int* tmap,
                       const BatchGrid* grids, const int* need, double A, double B, cudaStream_t st) {
    LAUNCH(k_lsrk_batch<F>, ct, st, Q, du, dQ, ct, ncons, tmap, grids, need, A, B);
}
template struct BatchOps<double>;
template struct BatchOps<float>;

void batch_bc(double* Q, const BatchGrid* grids, const BatchFace* faces, int nfaces, int64_t ct, int Ns,
              cudaStream_t st) {
    if (nfaces <= 0) return;
    k_bc_batch<<<nfaces, kThreads, 0, st>>>(Q, grids, faces, ct, Ns);
    count_launch();
    check_launch("k_bc_batch");
}
void batch_clock_after(const BatchGrid* grids, int G, cudaStream_t st) {
    k_clock_after_batch<<<(G + 127) / 128, 128, 0, st>>>(grids, G);
    count_launch();
    check_launch("k_clock_after_batch");
}

void clock_after(double* clk, const ClockConst& c, cudaStream_t st) {
    k_clock_after<<<1, 32, 0, st>>>(clk, c);
    count_launch();
    check_launch("k_clock_after");
}

// ------------------------------------------------------------- launchers ----

template <typename F>
void Pointwise<F>::primitives(const double* Q, F* prim, int64_t cells, int Ns, const PhysConst& pc, cudaStream_t st,
                              int esens) {
    if (pc.eos == CLES_EOS_NASA9) LAUNCH((k_primitives<F, true>), cells, st, Q, prim, cells, Ns, pc, esens, nullptr, nullptr);
    else LAUNCH((k_primitives<F, false>), cells, st, Q, prim, cells, Ns, pc, esens, nullptr, nullptr);
}
template <typename F>
void Pointwise<F>::delta4_tiled(const F* f0, const F* f1, F* o0, F* o1, const Grid3& g, const double w0[3],
                                const double w1[3], cudaStream_t st) {
    dim3 grid((unsigned)((g.n[0] + kTX - 1) / kTX), (unsigned)((g.n[1] + kTY - 1) / kTY),
              (unsigned)((g.n[2] + kZC - 1) / kZC));
    Weights3 a{{w0[0], w0[1], w0[2]}}, b{{0.0, 0.0, 0.0}};
    if (f1) {
        b = Weights3{{w1[0], w1[1], w1[2]}};
        constexpr size_t sm = delta4_smem<F, 2>();
        set_smem_attr(k_delta4_tiled<F, 2>, sm);
        k_delta4_tiled<F, 2><<<grid, kD4Threads, sm, st>>>(f0, f1, o0, o1, g, a, b);
    } else {
        constexpr size_t sm = delta4_smem<F, 1>();
        set_smem_attr(k_delta4_tiled<F, 1>, sm);
        k_delta4_tiled<F, 1><<<grid, kD4Threads, sm, st>>>(f0, nullptr, o0, nullptr, g, a, b);
    }
    count_launch();
    check_launch("k_delta4_tiled");
}
template <typename F>
void Pointwise<F>::delta4_halo(const F* f0, const F* f1, F* o0, F* o1, const Grid3& g, const double w0[3],
                               const double w1[3], const Halo4& h, cudaStream_t st) {
    const int64_t cells = (int64_t)g.n[0] * g.n[1] * g.n[2];
    Weights3 a{{w0[0], w0[1], w0[2]}}, b{{0.0, 0.0, 0.0}};
    if (f1) {
        b = Weights3{{w1[0], w1[1], w1[2]}};
        LAUNCH((k_delta4_halo<F, 2>), cells, st, f0, f1, o0, o1, g, a, b, h);
    } else {
        LAUNCH((k_delta4_halo<F, 1>), cells, st, f0, nullptr, o0, nullptr, g, a, b, h);
    }
}
template <typename F>
void Pointwise<F>::art_coef(const F* s_strain, const F* s_energy, const F* prim, const F* g, F* art, int64_t cells,
                            double C_mu, double C_beta, double C_kappa, int gate, cudaStream_t st) {
    LAUNCH(k_art_coef<F>, cells, st, s_strain, s_energy, prim, g, art, cells, C_mu, C_beta, C_kappa, gate);
}
template <typename F>
void Pointwise<F>::strain(const F* g, F* out, int64_t cells, cudaStream_t st) {
    LAUNCH(k_strain<F>, cells, st, g, out, cells);
}
template <typename F>
void Pointwise<F>::delta4(const F* f, F* out, const Grid3& g, const double wd[3], cudaStream_t st) {
    const int64_t cells = (int64_t)g.n[0] * g.n[1] * g.n[2];
    LAUNCH(k_delta4<F>, cells, st, f, out, g, wd[0], wd[1], wd[2]);
}
template <typename F>
void Pointwise<F>::mu_beta(const F* sensor, const F* prim, const F* g, F* art, int64_t cells, double C_mu,
                           double C_beta, int gate, cudaStream_t st) {
    LAUNCH(k_mu_beta<F>, cells, st, sensor, prim, g, art, cells, C_mu, C_beta, gate);
}
template <typename F>
void Pointwise<F>::dilatation(const F* g, F* div, F* sw, int64_t cells, cudaStream_t st) {
    LAUNCH(k_dilatation<F>, cells, st, g, div, sw, cells);
}
template <typename F>
void Pointwise<F>::beta_dilatation(const F* sensor, const F* prim, const F* sw, F* art, int64_t cells, double C_beta,
                                   cudaStream_t st) {
    LAUNCH(k_beta_dilatation<F>, cells, st, sensor, prim, sw, art, cells, C_beta);
}
template <typename F>
void Pointwise<F>::energy(const double* Q, const F* prim, F* out, int64_t cells, int Ns, cudaStream_t st) {
    LAUNCH(k_energy<F>, cells, st, Q, prim, out, cells, Ns);
}
template <typename F>
void Pointwise<F>::kappa(const F* sensor, const F* prim, F* art, int64_t cells, double C_kappa, cudaStream_t st) {
    LAUNCH(k_kappa<F>, cells, st, sensor, prim, art, cells, C_kappa);
}
template <typename F>
void Pointwise<F>::dart(const F* sensor, const F* prim, F* art, int64_t cells, double C_D, int sp, cudaStream_t st) {
    LAUNCH(k_dart<F>, cells, st, sensor, prim, art, cells, C_D, sp);
}
template <typename F>
void Pointwise<F>::fluxes(const double* Q, const F* prim, const F* g, const F* gty, const F* art, F* flux,
                          int64_t cells, int Ns, const PhysConst& pc, double mu0, double Pr, double Sc,
                          cudaStream_t st) {
    const Geom G{};
    if (Ns == 1)
        LAUNCH((k_fluxes<F, true, false, false>), cells, st, Q, prim, g, gty, art, flux, cells, Ns, pc, mu0, Pr, Sc, G, nullptr, nullptr);
    else if (pc.eos == CLES_EOS_NASA9)
        LAUNCH((k_fluxes<F, false, true, false>), cells, st, Q, prim, g, gty, art, flux, cells, Ns, pc, mu0, Pr, Sc, G, nullptr, nullptr);
    else
        LAUNCH((k_fluxes<F, false, false, false>), cells, st, Q, prim, g, gty, art, flux, cells, Ns, pc, mu0, Pr, Sc, G, nullptr, nullptr);
}
template <typename F>
void Pointwise<F>::fluxes_geo(const double* Q, const F* prim, const F* g, const F* gty, const F* art, F* flux,
                              int64_t cells, int Ns, const PhysConst& pc, double mu0, double Pr, double Sc,
                              const Geom& G, cudaStream_t st) {
    if (Ns == 1)
        LAUNCH((k_fluxes<F, true, false, true>), cells, st, Q, prim, g, gty, art, flux, cells, Ns, pc, mu0, Pr, Sc, G, nullptr, nullptr);
    else if (pc.eos == CLES_EOS_NASA9)
        LAUNCH((k_fluxes<F, false, true, true>), cells, st, Q, prim, g, gty, art, flux, cells, Ns, pc, mu0, Pr, Sc, G, nullptr, nullptr);
    else
        LAUNCH((k_fluxes<F, false, false, true>), cells, st, Q, prim, g, gty, art, flux, cells, Ns, pc, mu0, Pr, Sc, G, nullptr, nullptr);
}
template <typename F>
void Pointwise<F>::body_forces(F* dQ, const double* Q, int64_t cells, int Ns, const BodyForces& bf, cudaStream_t st) {
    LAUNCH(k_body_forces<F>, cells, st, dQ, Q, cells, Ns, bf);
}
template <typename F>
void Pointwise<F>::lsrk(double* Q, double* du, const F* dQ, int64_t n, double A, double B, double dt, cudaStream_t st,
                        const double* dtp) {
    LAUNCH(k_lsrk<F>, n, st, Q, du, dQ, n, A, B, dt, dtp);
}
template <typename F>
void Pointwise<F>::rate(const double* Q, const F* prim, const F* art, double* part, double* out, int64_t cells, int Ns,
                        const double idx[3], const int act[3], double mu0, double Pr, double Sc, cudaStream_t st) {
    const unsigned nb = grid_for(cells);
    k_rate_partial<F><<<nb, kThreads, 0, st>>>(Q, prim, art, part, cells, Ns, idx[0], idx[1], idx[2], act[0], act[1],
                                               act[2], mu0, Pr, Sc);
    count_launch();
    check_launch("k_rate_partial");
    k_rate_final<<<1, kThreads, 0, st>>>(part, (int)nb, out);
    count_launch();
    check_launch("k_rate_final");
}
void rate_final(const double* part, int nb, double* out, cudaStream_t st) {
    k_rate_final<<<1, kThreads, 0, st>>>(part, nb, out);
    count_launch();
    check_launch("k_rate_final");
}
template <typename F>
void Pointwise<F>::kinetic(const double* Q, double* part, double* out, int64_t cells, int Ns, cudaStream_t st) {
    const unsigned nb = grid_for(cells);
    k_ke_partial<F><<<nb, kThreads, 0, st>>>(Q, part, cells, Ns);
    count_launch();
    check_launch("k_ke_partial");
    k_sum_final<<<1, kThreads, 0, st>>>(part, (int)nb, 1, out);
    count_launch();
    check_launch("k_sum_final");
}
template <typename F>
void Pointwise<F>::dissipation(const F* prim, const F* g, const F* art, double* part, double* out, const Grid3& gr,
                               double mu0, cudaStream_t st, const Geom* G, unsigned foldmask) {
    const int64_t cells = (int64_t)gr.n[0] * gr.n[1] * gr.n[2];
    const unsigned nb = grid_for(cells);
    k_diss_partial<F><<<nb, kThreads, 0, st>>>(prim, g, art, part, gr, mu0, G ? *G : Geom{}, G ? 1 : 0, foldmask);
    count_launch();
    check_launch("k_diss_partial");
    k_sum_final<<<1, kThreads, 0, st>>>(part, (int)nb, 2, out);
    count_launch();
    check_launch("k_sum_final");
}
template <typename F>
void Pointwise<F>::convert(const double* a, F* b, int64_t n, cudaStream_t st) {
    LAUNCH(k_convert<F>, n, st, a, b, n);
}
template <typename F>
void Pointwise<F>::to_double(const F* a, double* b, int64_t n, cudaStream_t st) {
    LAUNCH(k_to_double<F>, n, st, a, b, n);
}

void bc_plane(double* Q, const Grid3& g, int d, int side, int Ns, int kind, const BcState& s, cudaStream_t st,
              const double* qface) {
    const int o1 = d == 0 ? 1 : 0, o2 = d == 2 ? 1 : 2;
    const int64_t plane = (int64_t)g.n[o1] * g.n[o2];
    k_bc_plane<<<grid_for(plane), kThreads, 0, st>>>(Q, g, d, side, Ns, kind, s, qface);
    count_launch();
    check_launch("k_bc_plane");
}

template <typename F>
void Pointwise<F>::nscbc(F* dQ, const F* prim, const F* g, const F* gty, int ngty, const F* dpd, const F* dpt0,
                         const F* dpt1, const F* drd, const Grid3& gr, int d, int side, int Ns, const PhysConst& pc,
                         const NscbcParams& bp, cudaStream_t st, const double* tgt, const Geom* G) {
    const Geom G0 = G ? *G : Geom{};
    const int geo = G ? 1 : 0;
    const int o1 = d == 0 ? 1 : 0, o2 = d == 2 ? 1 : 2;
    const int64_t plane = (int64_t)gr.n[o1] * gr.n[o2];
    if (pc.eos == CLES_EOS_NASA9)
        k_nscbc<F, true><<<grid_for(plane), kThreads, 0, st>>>(dQ, prim, g, gty, ngty, dpd, dpt0, dpt1, drd, gr, d, side,
                                                               Ns, pc, bp, tgt, G0, geo);
    else
        k_nscbc<F, false><<<grid_for(plane), kThreads, 0, st>>>(dQ, prim, g, gty, ngty, dpd, dpt0, dpt1, drd, gr, d,
                                                                side, Ns, pc, bp, tgt, G0, geo);
    count_launch();
    check_launch("k_nscbc");
}

void gather_interior(const double* padded, double* interior, const int n[3], const int pad[3], cudaStream_t st) {
    const int64_t cells = (int64_t)n[0] * n[1] * n[2];
    k_gather_interior<<<grid_for(cells), kThreads, 0, st>>>(padded, interior, n[0], n[1], n[2], pad[0], pad[1], pad[2]);
    count_launch();
    check_launch("k_gather_interior");
}

int64_t rate_partials(int64_t cells) { return (int64_t)grid_for(cells); }

template struct Pointwise<double>;
template struct Pointwise<float>;

}  // namespace cles
