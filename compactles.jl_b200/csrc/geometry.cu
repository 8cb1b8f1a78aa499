// Curvilinear and stretched grids (src/metric.jl, src/folds.jl, the general
// path of compute_rhs! at src/rhs.jl:650-687 and max_rate at
// src/timestep.jl:125-200).
//
// The geometry is carried as per-dimension node tables (Geom); each kernel
// recomputes J, A_d, 1/h_d and 1/r of its cell with geo_point, so no 3-D
// geometry array is streamed.  Products that the reference rounds separately
// are written with __dmul_rn so they are not contracted into an FMA.

#include "pointwise.h"

namespace cles {

namespace {

constexpr int kThreads = 256;

inline unsigned grid_for(int64_t n) {
    int64_t b = (n + kThreads - 1) / kThreads;
    if (b > 148 * 64) b = 148 * 64;
    return (unsigned)(b < 1 ? 1 : b);
}

#define GRID_STRIDE(idx, n) \
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < (n); idx += (int64_t)gridDim.x * blockDim.x)

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

// compute_primitives_and_gradients! tail (src/rhs.jl:596-604): each active
// dim's coordinate derivatives times 1/h_d, collapsed dims zero, then the
// additive curvature terms of metric_correct_gradients! (src/metric.jl:181-221).
// g[3 d + j] = d u_j / d x_d.
template <typename F>
__global__ void k_metric_grad(F* __restrict__ g, const F* __restrict__ prim, Geom G, Grid3 gr, int64_t cells) {
    GRID_STRIDE(I, cells) {
        int i, j, k;
        cell_ijk(I, gr.n, i, j, k);
        const GeoPoint p = geo_point(G, i, j, k, I);
        double gv[9];
#pragma unroll
        for (int d = 0; d < 3; ++d)
#pragma unroll
            for (int c = 0; c < 3; ++c)
                gv[3 * d + c] = gr.active[d] ? __dmul_rn(double(g[I + cells * (3 * d + c)]), p.inv_h[d]) : 0.0;
        if (G.metric == CLES_METRIC_CYLINDRICAL) {
            const double ir = p.inv_r;
            gv[3] = gv[3] - __dmul_rn(double(prim[I + cells * P_V]), ir);
            gv[4] = gv[4] + __dmul_rn(double(prim[I + cells * P_U]), ir);
        } else if (G.metric == CLES_METRIC_SPHERICAL) {
            const double ir = p.inv_r, ctr = p.cotr;
            const double ur = double(prim[I + cells * P_U]), ut = double(prim[I + cells * P_V]),
                         up = double(prim[I + cells * P_W]);
            gv[3] = gv[3] - __dmul_rn(ut, ir);
            gv[4] = gv[4] + __dmul_rn(ur, ir);
            gv[6] = gv[6] - __dmul_rn(up, ir);
            gv[7] = gv[7] - __dmul_rn(up, ctr);
            gv[8] = gv[8] + (__dmul_rn(ur, ir) + __dmul_rn(ut, ctr));
        }
#pragma unroll
        for (int e = 0; e < 9; ++e) g[I + cells * e] = F(gv[e]);
    }
}

// _scale_grad! (src/rhs.jl:477-483) of `count` fields per active dim
template <typename F>
__global__ void k_scale_grad(F* __restrict__ f, int count, Geom G, Grid3 gr, int64_t cells) {
    GRID_STRIDE(I, cells) {
        int i, j, k;
        cell_ijk(I, gr.n, i, j, k);
        const GeoPoint p = geo_point(G, i, j, k, I);
        for (int d = 0; d < 3; ++d) {
            if (!gr.active[d]) continue;
            for (int c = 0; c < count; ++c) {
                F* q = f + I + cells * ((int64_t)d * count + c);
                *q = F(__dmul_rn(double(*q), p.inv_h[d]));
            }
        }
    }
}

// _Pi (src/metric.jl:225-233): Pi_ab = rho u_a u_b + p delta_ab - tau_ab
template <typename F>
__device__ __forceinline__ double metric_pi(const F* prim, const F* g, const F* art, double mu0, int64_t I,
                                            int64_t cells, int a, int b) {
    const double mu = mu0 + double(art[I + cells * A_MU]);
    const double be = double(art[I + cells * A_BETA]);
    const double divu = double(g[I]) + double(g[I + cells * 4]) + double(g[I + cells * 8]);
    double tau = __dmul_rn(mu, double(g[I + cells * (3 * a + b)]) + double(g[I + cells * (3 * b + a)]));
    tau = tau + (a == b ? __dmul_rn(be - 2 * mu / 3, divu) : 0.0);
    const double uv[3] = {double(prim[I + cells * P_U]), double(prim[I + cells * P_V]), double(prim[I + cells * P_W])};
    return __dmul_rn(__dmul_rn(double(prim[I + cells * P_RHO]), uv[a]), uv[b]) +
           (a == b ? double(prim[I + cells * P_P]) : 0.0) - tau;
}

// The general flux-divergence path of compute_rhs! (src/rhs.jl:669-683):
// dQ_c = 0; dQ_c -= inv_J D_d(A_d F_dc) for d = 1, 2, 3; then
// add_metric_sources! (src/metric.jl:235-269) on the momentum components.
template <typename F>
__global__ void k_metric_div(F* __restrict__ dQ, const F* __restrict__ fd, int ncons, int Ns,
                             const F* __restrict__ prim, const F* __restrict__ g, const F* __restrict__ art,
                             double mu0, Geom G, Grid3 gr, int64_t cells) {
    GRID_STRIDE(I, cells) {
        int i, j, k;
        cell_ijk(I, gr.n, i, j, k);
        const GeoPoint p = geo_point(G, i, j, k, I);
        double mom[3] = {0.0, 0.0, 0.0};
        for (int c = 0; c < ncons; ++c) {
            double acc = 0.0;
            for (int d = 0; d < 3; ++d)
                if (gr.active[d]) acc = acc - __dmul_rn(p.inv_J, double(fd[I + cells * ((int64_t)d * ncons + c)]));
            if (c >= Ns && c < Ns + 3) mom[c - Ns] = acc;
            else dQ[I + cells * c] = F(acc);
        }
        const double ir = p.inv_r;
        if (G.metric == CLES_METRIC_CYLINDRICAL) {
            mom[0] = mom[0] + __dmul_rn(ir, metric_pi(prim, g, art, mu0, I, cells, 1, 1));
            mom[1] = mom[1] - __dmul_rn(ir, metric_pi(prim, g, art, mu0, I, cells, 1, 0));
        } else if (G.metric == CLES_METRIC_SPHERICAL) {
            const double ctr = p.cotr;
            const double Ptt = metric_pi(prim, g, art, mu0, I, cells, 1, 1);
            const double Ppp = metric_pi(prim, g, art, mu0, I, cells, 2, 2);
            mom[0] = mom[0] + __dmul_rn(ir, Ptt + Ppp);
            mom[1] = mom[1] + (__dmul_rn(-ir, metric_pi(prim, g, art, mu0, I, cells, 1, 0)) + __dmul_rn(ctr, Ppp));
            mom[2] = mom[2] + (__dmul_rn(-ir, metric_pi(prim, g, art, mu0, I, cells, 2, 0)) -
                               __dmul_rn(ctr, metric_pi(prim, g, art, mu0, I, cells, 2, 1)));
        }
        for (int a = 0; a < 3; ++a) dQ[I + cells * (Ns + a)] = F(mom[a]);
    }
}

// max_rate per-block partials (src/timestep.jl:125-175) with the inverse
// physical spacing inv_h_d / h_d and curvature_rate (src/timestep.jl:185-200).
template <typename F>
__global__ void k_rate_partial_geo(const double* __restrict__ Q, const F* __restrict__ prim,
                                   const F* __restrict__ art, double* __restrict__ part, int Ns, double h0, double h1,
                                   double h2, double mu0, double Pr, double Sc, Geom G, Grid3 gr, int64_t cells) {
    double rate = 0.0, rmin = __longlong_as_double(0x7ff0000000000000LL);
    const double hh[3] = {h0, h1, h2};
    GRID_STRIDE(I, cells) {
        int i, j, k;
        cell_ijk(I, gr.n, i, j, k);
        const GeoPoint p = geo_point(G, i, j, k, I);
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
            if (!gr.active[d]) continue;
            const double idx = p.inv_h[d] / hh[d];
            acc = acc + __dmul_rn(fabs(uv[d]) + c, idx);
            dsum = dsum + __dmul_rn(idx, idx);
        }
        double crate = 0.0;
        if (G.metric == CLES_METRIC_CYLINDRICAL) {
            if (!gr.active[1]) crate = __dmul_rn(fabs(uv[1]), p.inv_r);
        } else if (G.metric == CLES_METRIC_SPHERICAL) {
            if (!gr.active[1]) crate = crate + __dmul_rn(fabs(uv[1]), p.inv_r);
            if (!gr.active[2]) crate = crate + __dmul_rn(fabs(uv[2]), p.inv_r + fabs(p.cotr));
        }
        acc = acc + crate;
        double Dmax = mu0 / (Sc * r);
        for (int sp = 0; sp < Ns; ++sp) Dmax = jl_max(Dmax, mu0 / (Sc * r) + double(art[I + cells * (A_D0 + sp)]));
        const double nu = __dmul_rn(mu0 + double(art[I + cells * A_MU]) + double(art[I + cells * A_BETA]), ri) +
                          __dmul_rn(mu0 * cp / Pr + double(art[I + cells * A_KAPPA]), ri) / cp + Dmax;
        acc = acc + __dmul_rn(2 * nu, dsum);
        rate = jl_max(rate, acc);
    }
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
        part[2 * blockIdx.x] = sr[0];
        part[2 * blockIdx.x + 1] = sm[0];
    }
}

// Partner slot of interior cell c under the on-rank pairing.
__device__ __forceinline__ int64_t pair_partner(const PairParams& pp, int c[3]) {
    if (pp.pdim >= 0) {
        const int half = pp.n[pp.pdim] / 2;
        c[pp.pdim] = c[pp.pdim] < half ? c[pp.pdim] + half : c[pp.pdim] - half;
    }
    if (pp.revdim >= 0) c[pp.revdim] = pp.n[pp.revdim] - 1 - c[pp.revdim];
    return c[0] + (int64_t)pp.n[0] * (c[1] + (int64_t)pp.n[1] * c[2]);
}

// Full-grid index of half-grid cell J (the sd extent halved) and of its partner.
__device__ __forceinline__ void pair_cell(const PairParams& pp, int64_t J, int64_t& I, int64_t& Mx) {
    int nh[3] = {pp.n[0], pp.n[1], pp.n[2]};
    nh[pp.sd] /= 2;
    int c[3];
    cell_ijk(J, nh, c[0], c[1], c[2]);
    I = c[0] + (int64_t)pp.n[0] * (c[1] + (int64_t)pp.n[1] * c[2]);
    Mx = pair_partner(pp, c);
}

// pair_forward! on-rank branch (src/folds.jl:169-190) over `count` fields
// (stride fs): for each canonical slot x (lower half of sd) and its partner
// Mx: w[x] = (f[x] + s f[Mx]) / 2, w[Mx] = (f[x] - s f[Mx]) / 2.
template <typename T>
__global__ void k_pair_forward(const T* __restrict__ f, T* __restrict__ w, PairParams pp, double sg, int64_t half,
                               int64_t fs) {
    const T* fc = f + fs * blockIdx.y;
    T* wc = w + fs * blockIdx.y;
    GRID_STRIDE(J, half) {
        int64_t I, Mx;
        pair_cell(pp, J, I, Mx);
        const double a = double(fc[I]), b = sg * double(fc[Mx]);
        wc[I] = T(0.5 * (a + b));
        wc[Mx] = T(0.5 * (a - b));
    }
}

// pair_backward! on-rank branch (src/folds.jl:224-243) in place: out holds
// the even result on the canonical half and the odd result on the partner
// half; out[x] = Re + Ro, out[Mx] = s (Re - Ro).
template <typename T>
__global__ void k_pair_backward(T* out, PairParams pp, double sg, int64_t half, int64_t fs) {
    T* oc = out + fs * blockIdx.y;
    GRID_STRIDE(J, half) {
        int64_t I, Mx;
        pair_cell(pp, J, I, Mx);
        const double Re = double(oc[I]), Ro = double(oc[Mx]);
        oc[I] = T(Re + Ro);
        oc[Mx] = T(sg * (Re - Ro));
    }
}

__global__ void k_geo_area(double* __restrict__ out, int d, Geom G, int64_t cells) {
    GRID_STRIDE(I, cells) {
        int i, j, k;
        cell_ijk(I, G.n, i, j, k);
        out[I] = geo_point(G, i, j, k, I).A[d];
    }
}

// gcl_cotr! (src/metric.jl:154-170): cot(theta)/r = inv_J D_theta(A_theta)
__global__ void k_geo_gcl(double* __restrict__ cotr, const double* __restrict__ dA, Geom G, int64_t cells) {
    Geom G0 = G;
    G0.cotr = nullptr;
    GRID_STRIDE(I, cells) {
        int i, j, k;
        cell_ijk(I, G.n, i, j, k);
        cotr[I] = __dmul_rn(geo_point(G0, i, j, k, I).inv_J, dA[I]);
    }
}

}  // namespace

template <typename F>
void MetricOps<F>::metric_grad(F* g, const F* prim, const Geom& G, const Grid3& gr, cudaStream_t st) {
    const int64_t cells = (int64_t)gr.n[0] * gr.n[1] * gr.n[2];
    k_metric_grad<F><<<grid_for(cells), kThreads, 0, st>>>(g, prim, G, gr, cells);
    count_launch();
    check_launch("k_metric_grad");
}
template <typename F>
void MetricOps<F>::scale_grad(F* f, int count, const Geom& G, const Grid3& gr, cudaStream_t st) {
    const int64_t cells = (int64_t)gr.n[0] * gr.n[1] * gr.n[2];
    k_scale_grad<F><<<grid_for(cells), kThreads, 0, st>>>(f, count, G, gr, cells);
    count_launch();
    check_launch("k_scale_grad");
}
template <typename F>
void MetricOps<F>::metric_div(F* dQ, const F* fd, int ncons, int Ns, const F* prim, const F* g, const F* art,
                              double mu0, const Geom& G, const Grid3& gr, cudaStream_t st) {
    const int64_t cells = (int64_t)gr.n[0] * gr.n[1] * gr.n[2];
    k_metric_div<F><<<grid_for(cells), kThreads, 0, st>>>(dQ, fd, ncons, Ns, prim, g, art, mu0, G, gr, cells);
    count_launch();
    check_launch("k_metric_div");
}
template <typename F>
void MetricOps<F>::rate_geo(const double* Q, const F* prim, const F* art, double* part, double* out, int Ns,
                            const double h[3], double mu0, double Pr, double Sc, const Geom& G, const Grid3& gr,
                            cudaStream_t st) {
    const int64_t cells = (int64_t)gr.n[0] * gr.n[1] * gr.n[2];
    const unsigned nb = grid_for(cells);
    k_rate_partial_geo<F><<<nb, kThreads, 0, st>>>(Q, prim, art, part, Ns, h[0], h[1], h[2], mu0, Pr, Sc, G, gr,
                                                   cells);
    count_launch();
    check_launch("k_rate_partial_geo");
    rate_final(part, (int)nb, out, st);
}

template <typename T>
void pair_forward(const T* f, T* w, int count, int64_t fs, const PairParams& pp, int sig, cudaStream_t st) {
    const int64_t half = (int64_t)pp.n[0] * pp.n[1] * pp.n[2] / 2;
    const dim3 grid(grid_for(half), (unsigned)count);
    k_pair_forward<T><<<grid, kThreads, 0, st>>>(f, w, pp, (double)sig, half, fs);
    count_launch();
    check_launch("k_pair_forward");
}
template <typename T>
void pair_backward(T* out, int count, int64_t fs, const PairParams& pp, int sig, cudaStream_t st) {
    const int64_t half = (int64_t)pp.n[0] * pp.n[1] * pp.n[2] / 2;
    const dim3 grid(grid_for(half), (unsigned)count);
    k_pair_backward<T><<<grid, kThreads, 0, st>>>(out, pp, (double)sig, half, fs);
    count_launch();
    check_launch("k_pair_backward");
}

void geo_area(double* out, int d, const Geom& G, cudaStream_t st) {
    const int64_t cells = (int64_t)G.n[0] * G.n[1] * G.n[2];
    k_geo_area<<<grid_for(cells), kThreads, 0, st>>>(out, d, G, cells);
    count_launch();
    check_launch("k_geo_area");
}
void geo_gcl(double* cotr, const double* dA, const Geom& G, cudaStream_t st) {
    const int64_t cells = (int64_t)G.n[0] * G.n[1] * G.n[2];
    k_geo_gcl<<<grid_for(cells), kThreads, 0, st>>>(cotr, dA, G, cells);
    count_launch();
    check_launch("k_geo_gcl");
}

template struct MetricOps<double>;
template struct MetricOps<float>;
template void pair_forward<double>(const double*, double*, int, int64_t, const PairParams&, int, cudaStream_t);
template void pair_forward<float>(const float*, float*, int, int64_t, const PairParams&, int, cudaStream_t);
template void pair_backward<double>(double*, int, int64_t, const PairParams&, int, cudaStream_t);
template void pair_backward<float>(float*, int, int64_t, const PairParams&, int, cudaStream_t);

}  // namespace cles
