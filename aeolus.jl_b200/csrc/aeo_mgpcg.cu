// aeo_mgpcg.cu -- multigrid-preconditioned conjugate gradients for
// div(c grad phi) = b on a uniform grid (the cut-cell pressure solve).
//
// The algorithm is the reference's MGPreconditionedCG (src/Multigrid.jl:
// 551-967, pcg! in src/Backends.jl:1511-1589): CG on the FP64 operator with
// face coefficients, deflated for a singular operator (periodic / Neumann
// axes), preconditioned by one V-cycle of red-black Gauss-Seidel (nu1 / nu2
// sweeps), full-weighting restriction, trilinear prolongation and face
// coefficients coarsened by four-face means, with a long RB-GS smoothing on
// the coarsest level.
//
// GPU design:
//   * the whole solve is one CUDA graph: a prologue, a conditional WHILE node
//     whose body is one CG iteration (operator, update, V-cycle, reductions,
//     direction), and the final mean shift.  The loop condition is set on the
//     device by the last kernel of each iteration (converged, breakdown, or
//     the iteration cap), so no host round trip happens between iterations
//     and the loop always ends by the cap;
//   * every reduction is FP64 and deterministic: fixed grids, per-block
//     partials, and the last block to finish folds the partials in a fixed
//     order and computes the scalars (alpha, beta, the means, the status) in
//     device memory;
//   * levels are interior-only arrays; halos are index maps (periodic wrap,
//     Neumann mirror), exact for the even dimensions of every level that is
//     not the coarsest;
//   * the coarsest level runs all its sweeps in one thread block with its
//     arrays in shared memory, each colour pass computed before it is
//     written, which is the reference's halo-copy semantics at any parity;
//   * the first half-sweep of a level that starts from zero is pointwise
//     (every neighbour is zero), so it is fused with the zeroing and with
//     the mean projection of the level's right-hand side;
//   * the fine residual is never stored: it is formed inside the restriction.
//   * the mean projections the reference applies to phi after smoothing and
//     prolongation shift phi by a constant; RB-GS, the residual and the
//     prolongation commute with constant shifts and the CG deflation removes
//     the mean of z, so they are omitted; the projections of every
//     right-hand side are kept.
#include <cuda_runtime.h>

#include <cfloat>
#include <cmath>
#include <cstring>
#include <new>
#include <string>
#include <type_traits>
#include <vector>

#include "../../include/aeolus_b200_mgpcg.h"

namespace {

constexpr int TPB = 256;
constexpr int RED_BLOCKS = 592;        // 4 x 148 SMs: the fixed grid of every FP64 reduction
constexpr int COARSE_THREADS = 1024;
constexpr int COARSE_MAX_CELLS = 16384;
constexpr int COARSE_PER_THREAD = COARSE_MAX_CELLS / COARSE_THREADS;
constexpr int MAX_LEVELS = 24;

template <typename R> struct Eps;
template <> struct Eps<double> { static __device__ __host__ double v() { return DBL_EPSILON; } };
template <> struct Eps<float> { static __device__ __host__ float v() { return FLT_EPSILON; } };

struct Bc { int x, y, z; };            // 0 periodic, 1 Neumann

// Device scalars of one solve.  Written only by last blocks of reductions
// and read by every block of the next kernels.
struct PcgState {
    double tol, n;
    double mb, bnorm, rz, pAp, alpha, beta, m, mr, rnorm, curvature, mx, rel;
    int iters, maxit, status, done;
    int project, flexible;
    unsigned counter;
};

template <typename R> struct Level {
    int nx, ny, nz;
    long long n;
    R ix2, iy2, iz2;
    R* phi;
    R* b;
    const R* cx;                        // nullptr: constant-coefficient Laplacian
    const R* cy;
    const R* cz;
    double* bmean;                      // mean of b to subtract before use (device scalar)
};

__device__ __forceinline__ int wm(int i, int n, int bc) { return i > 0 ? i - 1 : (bc == 0 ? n - 1 : 0); }
__device__ __forceinline__ int wp(int i, int n, int bc) { return i < n - 1 ? i + 1 : (bc == 0 ? 0 : n - 1); }

// Neighbour and face indices of cell (i, j, k) of an nx x ny x nz level.
struct Idx {
    long long q, xm, xp, ym, yp, zm, zp, cx, cy;
    long long sy, sz;                   // cy north offset (nx), cz top offset (nx*ny)
};

__device__ __forceinline__ Idx make_idx(int i, int j, int k, int nx, int ny, int nz, Bc bc) {
    Idx d;
    long long row = (long long)nx * ((long long)j + (long long)ny * k);
    d.q = row + i;
    d.xm = row + wm(i, nx, bc.x);
    d.xp = row + wp(i, nx, bc.x);
    long long pl = (long long)nx * ny * k;
    d.ym = pl + (long long)nx * wm(j, ny, bc.y) + i;
    d.yp = pl + (long long)nx * wp(j, ny, bc.y) + i;
    long long cj = (long long)nx * j + i;
    d.zm = (long long)nx * ny * wm(k, nz, bc.z) + cj;
    d.zp = (long long)nx * ny * wp(k, nz, bc.z) + cj;
    d.cx = (long long)i + (long long)(nx + 1) * ((long long)j + (long long)ny * k);
    d.cy = (long long)i + (long long)nx * ((long long)j + (long long)(ny + 1) * k);
    d.sy = nx;
    d.sz = (long long)nx * ny;
    return d;
}

// _Aphi of _ConstOp / _VarOp (src/Multigrid.jl:174-193) in the value type V
// with coefficients of type C.
template <typename V, typename C>
__device__ __forceinline__ V aphi(const V* f, const Idx& d, const C* cx, const C* cy, const C* cz, V ix2, V iy2,
                                  V iz2) {
    V c = f[d.q];
    if (cx == nullptr)
        return (f[d.xp] - V(2) * c + f[d.xm]) * ix2 + (f[d.yp] - V(2) * c + f[d.ym]) * iy2 +
               (f[d.zp] - V(2) * c + f[d.zm]) * iz2;
    V fxp = V(cx[d.cx + 1]), fxm = V(cx[d.cx]);
    V fyp = V(cy[d.cy + d.sy]), fym = V(cy[d.cy]);
    V fzp = V(cz[d.q + d.sz]), fzm = V(cz[d.q]);
    return (fxp * (f[d.xp] - c) - fxm * (c - f[d.xm])) * ix2 + (fyp * (f[d.yp] - c) - fym * (c - f[d.ym])) * iy2 +
           (fzp * (f[d.zp] - c) - fzm * (c - f[d.zm])) * iz2;
}

// One RB-GS update of cell d (src/Multigrid.jl:311-336); false: a fully
// blocked cell (|diag| < eps), left unchanged.
template <typename R>
__device__ __forceinline__ bool gs_value(const R* f, R bval, const Idx& d, const Level<R>& L, R* out) {
    R off, diag;
    if (L.cx == nullptr) {
        diag = -R(2) * (L.ix2 + L.iy2 + L.iz2);
        off = (f[d.xp] + f[d.xm]) * L.ix2 + (f[d.yp] + f[d.ym]) * L.iy2 + (f[d.zp] + f[d.zm]) * L.iz2;
    } else {
        R fxp = L.cx[d.cx + 1], fxm = L.cx[d.cx];
        R fyp = L.cy[d.cy + d.sy], fym = L.cy[d.cy];
        R fzp = L.cz[d.q + d.sz], fzm = L.cz[d.q];
        diag = -((fxp + fxm) * L.ix2 + (fyp + fym) * L.iy2 + (fzp + fzm) * L.iz2);
        if (fabs(diag) < Eps<R>::v()) return false;
        off = (fxp * f[d.xp] + fxm * f[d.xm]) * L.ix2 + (fyp * f[d.yp] + fym * f[d.ym]) * L.iy2 +
              (fzp * f[d.zp] + fzm * f[d.zm]) * L.iz2;
    }
    *out = (bval - off) / diag;
    return true;
}

// The diagonal alone (first half-sweep from zero: every neighbour is zero)
template <typename R>
__device__ __forceinline__ bool gs_diag(const Idx& d, const Level<R>& L, R* diag) {
    if (L.cx == nullptr) {
        *diag = -R(2) * (L.ix2 + L.iy2 + L.iz2);
        return true;
    }
    R fxp = L.cx[d.cx + 1], fxm = L.cx[d.cx];
    R fyp = L.cy[d.cy + d.sy], fym = L.cy[d.cy];
    R fzp = L.cz[d.q + d.sz], fzm = L.cz[d.q];
    *diag = -((fxp + fxm) * L.ix2 + (fyp + fym) * L.iy2 + (fzp + fzm) * L.iz2);
    return !(fabs(*diag) < Eps<R>::v());
}

// ---------------------------------------------------------------- reductions

__device__ __forceinline__ double warp_sum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// Block sum of K values, valid in thread 0; fixed order (deterministic).
template <int K>
__device__ __forceinline__ void block_sum(double (&v)[K]) {
    __shared__ double sh[K][32];
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31, nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int q = 0; q < K; ++q) v[q] = warp_sum(v[q]);
    if (l == 0)
#pragma unroll
        for (int q = 0; q < K; ++q) sh[q][w] = v[q];
    __syncthreads();
    if (w == 0) {
#pragma unroll
        for (int q = 0; q < K; ++q) v[q] = warp_sum(l < nw ? sh[q][l] : 0.0);
    }
    __syncthreads();
}

// Stores this block's partials; the last block to arrive folds all of them
// in block order and returns true with the totals in thread 0's `tot`.
template <int K>
__device__ bool reduce_last(double (&v)[K], double* part, unsigned* counter, double (&tot)[K]) {
    __shared__ bool last;
    block_sum<K>(v);
    const int nb = gridDim.x;
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < K; ++q) part[q * nb + blockIdx.x] = v[q];
        __threadfence();
        unsigned t = atomicAdd(counter, 1u);
        last = (t == (unsigned)nb - 1);
    }
    __syncthreads();
    if (!last) return false;
    __threadfence();
    double a[K];
#pragma unroll
    for (int q = 0; q < K; ++q) a[q] = 0.0;
    for (int b = threadIdx.x; b < nb; b += blockDim.x)
#pragma unroll
        for (int q = 0; q < K; ++q) a[q] += __ldcg(&part[q * nb + b]);
    block_sum<K>(a);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < K; ++q) tot[q] = a[q];
        *counter = 0u;
    }
    return true;
}

// ------------------------------------------------------------ CG kernels
// (pcg!/_pcg!, src/Backends.jl:1526-1589; definite = :negative)

// sum of a -> S->mb (mode 0) or S->mx (mode 1), divided by n when the mean is projected
__global__ void pcg_mean_kernel(const double* __restrict__ a, long long n, PcgState* S, double* part, int mode) {
    double v[1] = {0.0};
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
        v[0] += a[q];
    double t[1];
    if (reduce_last<1>(v, part, &S->counter, t) && threadIdx.x == 0) {
        double m = S->project ? t[0] / S->n : 0.0;
        if (mode == 0) S->mb = m; else S->mx = m;
    }
}

// r = b - mb (zero guess), x = 0; reduces (|b - mb|^2, sum r); zero rhs ends the solve
__global__ void pcg_init_kernel(const double* __restrict__ b, double* __restrict__ r, double* __restrict__ x,
                                long long n, PcgState* S, double* part) {
    const double mb = S->mb;
    double v[2] = {0.0, 0.0};
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        double bv = b[q] - mb;
        r[q] = bv;
        x[q] = 0.0;
        v[0] += bv * bv;
        v[1] += bv;
    }
    double t[2];
    if (reduce_last<2>(v, part, &S->counter, t) && threadIdx.x == 0) {
        S->bnorm = sqrt(t[0]);
        S->mr = S->project ? t[1] / S->n : 0.0;
        S->iters = 0;
        S->curvature = nan("");
        S->rz = 0.0;
        S->alpha = S->beta = 0.0;
        if (S->bnorm == 0.0) {
            S->status = AEO_MG_ZERO_RHS;
            S->done = 3;
        } else {
            S->status = AEO_MG_MAXIT;
            S->done = 0;
        }
    }
}

// Ap = A p with p.Ap; the last block forms alpha or flags a breakdown
template <typename C>
__global__ void pcg_apply_kernel(const double* __restrict__ p, double* __restrict__ Ap, const C* cx, const C* cy,
                                 const C* cz, int nx, int ny, int nz, Bc bc, double ix2, double iy2, double iz2,
                                 PcgState* S, double* part, int standalone) {
    if (!standalone && S->done) return;
    const long long n = (long long)nx * ny * nz;
    double v[1] = {0.0};
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        int i = (int)(q % nx);
        long long t = q / nx;
        int j = (int)(t % ny), k = (int)(t / ny);
        Idx d = make_idx(i, j, k, nx, ny, nz, bc);
        double a = aphi<double, C>(p, d, cx, cy, cz, ix2, iy2, iz2);
        Ap[q] = a;
        v[0] += p[q] * a;
    }
    double t[1];
    if (reduce_last<1>(v, part, &S->counter, t) && threadIdx.x == 0 && !standalone) {
        double pAp = t[0];
        S->pAp = pAp;
        S->curvature = pAp;
        if (!(fabs(pAp) > DBL_EPSILON * fabs(S->rz))) {
            S->status = AEO_MG_BREAKDOWN;
            S->done = 2;
        } else {
            S->alpha = S->rz / pAp;
        }
    }
}

// x += alpha p, r -= alpha Ap; reduces (r.r, sum r); convergence test
__global__ void pcg_update_kernel(double* __restrict__ x, double* __restrict__ r, const double* __restrict__ p,
                                  const double* __restrict__ Ap, long long n, PcgState* S, double* part) {
    if (S->done) return;
    const double alpha = S->alpha;
    double v[2] = {0.0, 0.0};
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        x[q] = x[q] + alpha * p[q];
        double rv = r[q] - alpha * Ap[q];
        r[q] = rv;
        v[0] += rv * rv;
        v[1] += rv;
    }
    double t[2];
    if (reduce_last<2>(v, part, &S->counter, t) && threadIdx.x == 0) {
        S->iters += 1;
        S->rnorm = sqrt(t[0]);
        S->mr = S->project ? t[1] / S->n : 0.0;
        if (S->rnorm <= S->tol * S->bnorm) {
            S->status = AEO_MG_CONVERGED;
            S->done = 1;
        }
    }
}

// after z = M r: (r.r, r.z, sum z, sum r, z.Ap, sum Ap); the deflation mean
// m = sum z / n, (r.z) -= m sum r, and beta
template <typename Z>
__global__ void pcg_rz_kernel(const double* __restrict__ r, const Z* __restrict__ z, const double* __restrict__ Ap,
                              long long n, PcgState* S, double* part, int first) {
    if (S->done) return;
    const bool flex = S->flexible && !first;
    double v[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        double rv = r[q], zv = double(z[q]);
        v[0] += rv * rv;
        v[1] += rv * zv;
        v[2] += zv;
        v[3] += rv;
        if (flex) {
            double a = Ap[q];
            v[4] += zv * a;
            v[5] += a;
        }
    }
    double t[6];
    if (reduce_last<6>(v, part, &S->counter, t) && threadIdx.x == 0) {
        double m = S->project ? t[2] / S->n : 0.0;
        double rzn = t[1];
        if (S->project) rzn -= m * t[3];
        S->m = m;
        if (first) {
            S->rz = rzn;
            S->beta = 0.0;
            S->rnorm = sqrt(t[0]);
            if (S->rnorm <= S->tol * S->bnorm) {
                S->status = AEO_MG_CONVERGED;
                S->done = 1;
            }
        } else {
            if (flex) {
                double zAp = t[4] - (S->project ? m * t[5] : 0.0);
                S->beta = -S->alpha * zAp / S->rz;
            } else {
                S->beta = rzn / S->rz;
            }
            S->rz = rzn;
        }
    }
}

// p = (z - m) + beta p  (p = z - m on the first pass)
template <typename Z>
__global__ void pcg_dir_kernel(double* __restrict__ p, const Z* __restrict__ z, long long n, const PcgState* S,
                               int first) {
    if (S->done) return;
    const double m = S->m, beta = S->beta;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
        p[q] = first ? double(z[q]) - m : (double(z[q]) - m) + beta * p[q];
}

__global__ void pcg_cond_kernel(PcgState* S, cudaGraphConditionalHandle h, int mode) {
    // mode 0: CG (continue while running and below the iteration cap);
    // mode 1: multigrid cycles (continue while above tol and below the cap)
    unsigned go = (S->done == 0 && S->iters < S->maxit) ? 1u : 0u;
    if (mode == 0 && S->done == 0 && S->iters >= S->maxit) S->status = AEO_MG_MAXIT;
    cudaGraphSetConditional(h, go);
}

__global__ void shift_kernel(double* __restrict__ x, long long n, const PcgState* S) {
    const double m = S->mx;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
        x[q] = x[q] - m;
}

// ------------------------------------------------------- multigrid kernels

// The first half-sweep of a level whose phi starts at zero: one thread per
// pair of cells (2ih, 2ih+1) of a row.  b <- b - mean (the projection of
// the level's right-hand side; level 0 takes b from the FP64 residual
// r - mean r), phi <- (b - 0)/diag on colour-0 cells, 0 on colour-1 cells.
template <typename R>
__global__ void mg_first_kernel(Level<R> L, Bc bc, const double* __restrict__ r0, const double* mr0, const int* done) {
    if (*done) return;
    const int half = L.nx >> 1;
    const long long total = (long long)half * L.ny * L.nz;
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= total) return;
    int ih = (int)(t % half);
    long long rest = t / half;
    int j = (int)(rest % L.ny), k = (int)(rest / L.ny);
    const double m0 = r0 ? *mr0 : 0.0;
    const R m = r0 ? R(0) : R(*L.bmean);
#pragma unroll
    for (int s = 0; s < 2; ++s) {
        int i = 2 * ih + s;
        long long q = (long long)L.nx * ((long long)j + (long long)L.ny * k) + i;
        R bv = r0 ? R(r0[q] - m0) : L.b[q] - m;
        L.b[q] = bv;
        R out = R(0);
        if (((i + j + k) & 1) == 0) {
            Idx d = make_idx(i, j, k, L.nx, L.ny, L.nz, bc);
            R diag;
            if (gs_diag<R>(d, L, &diag)) out = (bv - R(0)) / diag;
        }
        L.phi[q] = out;
    }
}

// One colour pass of red-black Gauss-Seidel over an even-nx level.
template <typename R>
__global__ void mg_rbgs_kernel(Level<R> L, Bc bc, int colour, const int* done) {
    if (done && *done) return;
    const int half = L.nx >> 1;
    const long long total = (long long)half * L.ny * L.nz;
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= total) return;
    int ih = (int)(t % half);
    long long rest = t / half;
    int j = (int)(rest % L.ny), k = (int)(rest / L.ny);
    int i = 2 * ih + ((j + k + colour) & 1);
    Idx d = make_idx(i, j, k, L.nx, L.ny, L.nz, bc);
    R v;
    if (gs_value<R>(L.phi, L.b[d.q], d, L, &v)) L.phi[d.q] = v;
}

// Coarse b = mean of the eight fine residuals b - A phi (src/Multigrid.jl:
// 380-406, formed here without storing the fine residual); the last block
// stores the coarse mean that the coarse level subtracts before use.
template <typename R>
__global__ void mg_restrict_kernel(Level<R> F, Level<R> Cl, Bc bc, double* part, unsigned* counter, const int* done) {
    if (done && *done) return;
    const long long nc = Cl.n;
    double v[1] = {0.0};
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nc; t += (long long)gridDim.x * blockDim.x) {
        int I = (int)(t % Cl.nx);
        long long rest = t / Cl.nx;
        int J = (int)(rest % Cl.ny), K = (int)(rest / Cl.ny);
        R s = R(0);
#pragma unroll
        for (int dk = 0; dk < 2; ++dk)
#pragma unroll
            for (int dj = 0; dj < 2; ++dj)
#pragma unroll
                for (int di = 0; di < 2; ++di) {
                    Idx d = make_idx(2 * I + di, 2 * J + dj, 2 * K + dk, F.nx, F.ny, F.nz, bc);
                    R rr = F.b[d.q] - aphi<R, R>(F.phi, d, F.cx, F.cy, F.cz, F.ix2, F.iy2, F.iz2);
                    s += rr;
                }
        R bc_ = s * R(0.125);
        Cl.b[t] = bc_;
        v[0] += double(bc_);
    }
    double tot[1];
    if (reduce_last<1>(v, part, counter, tot) && threadIdx.x == 0) *Cl.bmean = tot[0] / double(nc);
}

// phi_fine += trilinear (3/4, 1/4) interpolation of phi_coarse
// (src/Multigrid.jl:412-455), the eight terms in the reference's order.
template <typename R>
__global__ void mg_prolong_kernel(Level<R> F, Level<R> Cl, Bc bc, const int* done) {
    if (done && *done) return;
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= F.n) return;
    int i = (int)(t % F.nx);
    long long rest = t / F.nx;
    int j = (int)(rest % F.ny), k = (int)(rest / F.ny);
    int Ih = i >> 1, Jh = j >> 1, Kh = k >> 1;
    int Ix = (i & 1) ? wp(Ih, Cl.nx, bc.x) : wm(Ih, Cl.nx, bc.x);
    int Jy = (j & 1) ? wp(Jh, Cl.ny, bc.y) : wm(Jh, Cl.ny, bc.y);
    int Kz = (k & 1) ? wp(Kh, Cl.nz, bc.z) : wm(Kh, Cl.nz, bc.z);
    const R n_ = R(3) / R(4), f_ = R(1) / R(4);
    const long long sx = 1, sy = Cl.nx, sz = (long long)Cl.nx * Cl.ny;
    const R* P = Cl.phi;
    long long hhh = Ih * sx + Jh * sy + Kh * sz;
    R acc = R(0);
    acc += (n_ * n_ * n_) * P[hhh];
    acc += (f_ * n_ * n_) * P[Ix * sx + Jh * sy + Kh * sz];
    acc += (n_ * f_ * n_) * P[Ih * sx + Jy * sy + Kh * sz];
    acc += (f_ * f_ * n_) * P[Ix * sx + Jy * sy + Kh * sz];
    acc += (n_ * n_ * f_) * P[Ih * sx + Jh * sy + Kz * sz];
    acc += (f_ * n_ * f_) * P[Ix * sx + Jh * sy + Kz * sz];
    acc += (n_ * f_ * f_) * P[Ih * sx + Jy * sy + Kz * sz];
    acc += (f_ * f_ * f_) * P[Ix * sx + Jy * sy + Kz * sz];
    F.phi[t] += acc;
}

// The coarsest level: phi = 0, b -= mean, then `sweeps` RB-GS sweeps, all
// in one block (_solve_coarsest!, src/Multigrid.jl:681-685).  Arrays are
// staged in shared memory when they fit.  Each colour pass computes every
// new value before any is written, the semantics of the reference's halo
// copy even where a periodic wrap joins two cells of one colour.
template <typename R>
__global__ void __launch_bounds__(COARSE_THREADS) mg_coarsest_kernel(Level<R> L, Bc bc, int sweeps, int staged,
                                                                    const double* __restrict__ r0, const double* mr0,
                                                                    const int* done) {
    if (done && *done) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int nx = L.nx, ny = L.ny, nz = L.nz;
    const int n = (int)L.n;
    const int ncx = (nx + 1) * ny * nz, ncy = nx * (ny + 1) * nz, ncz = nx * ny * (nz + 1);
    Level<R> S = L;
    if (staged) {
        R* base = reinterpret_cast<R*>(smem_raw);
        S.phi = base;
        S.b = base + n;
        if (L.cx) {
            R* c = base + 2 * n;
            for (int q = threadIdx.x; q < ncx; q += blockDim.x) c[q] = L.cx[q];
            for (int q = threadIdx.x; q < ncy; q += blockDim.x) c[ncx + q] = L.cy[q];
            for (int q = threadIdx.x; q < ncz; q += blockDim.x) c[ncx + ncy + q] = L.cz[q];
            S.cx = c;
            S.cy = c + ncx;
            S.cz = c + ncx + ncy;
        }
    }
    const double m0 = r0 ? *mr0 : 0.0;
    const R m = r0 ? R(0) : R(*L.bmean);
    for (int q = threadIdx.x; q < n; q += blockDim.x) {
        S.b[q] = r0 ? R(r0[q] - m0) : L.b[q] - m;
        S.phi[q] = R(0);
    }
    __syncthreads();
    R nv[COARSE_PER_THREAD];
    for (int sw = 0; sw < sweeps; ++sw)
        for (int colour = 0; colour < 2; ++colour) {
#pragma unroll
            for (int s = 0; s < COARSE_PER_THREAD; ++s) {
                int q = threadIdx.x + s * COARSE_THREADS;
                nv[s] = R(0);
                if (q < n) {
                    int i = q % nx, j = (q / nx) % ny, k = q / (nx * ny);
                    Idx d = make_idx(i, j, k, nx, ny, nz, bc);
                    R v = S.phi[q];
                    if (((i + j + k) & 1) == colour) gs_value<R>(S.phi, S.b[q], d, S, &v);
                    nv[s] = v;
                }
            }
            __syncthreads();
#pragma unroll
            for (int s = 0; s < COARSE_PER_THREAD; ++s) {
                int q = threadIdx.x + s * COARSE_THREADS;
                if (q < n) S.phi[q] = nv[s];
            }
            __syncthreads();
        }
    if (staged)
        for (int q = threadIdx.x; q < n; q += blockDim.x) L.phi[q] = S.phi[q];
}

// Level-0 right-hand side for the standalone cycles: b0 = r - mean(r)
template <typename R>
__global__ void mg_load_kernel(Level<R> L, const double* __restrict__ r0, const double* mr0) {
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= L.n) return;
    L.b[t] = R(r0[t] - *mr0);
    L.phi[t] = R(0);
}

// relative residual of the standalone cycles (_residual_norm!,
// src/Multigrid.jl:780-785): |r - mean r| / |b| from sum r and sum r^2
template <typename R>
__global__ void mg_resnorm_kernel(Level<R> L, Bc bc, PcgState* S, double* part) {
    if (S->done) return;
    double v[2] = {0.0, 0.0};
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < L.n; t += (long long)gridDim.x * blockDim.x) {
        int i = (int)(t % L.nx);
        long long rest = t / L.nx;
        int j = (int)(rest % L.ny), k = (int)(rest / L.ny);
        Idx d = make_idx(i, j, k, L.nx, L.ny, L.nz, bc);
        double rr = double(L.b[t] - aphi<R, R>(L.phi, d, L.cx, L.cy, L.cz, L.ix2, L.iy2, L.iz2));
        v[0] += rr;
        v[1] += rr * rr;
    }
    double tot[2];
    if (reduce_last<2>(v, part, &S->counter, tot) && threadIdx.x == 0) {
        double ss = tot[1];
        if (S->project) ss -= tot[0] * (tot[0] / S->n);
        S->iters += 1;
        S->rel = sqrt(fmax(ss, 0.0)) / S->bnorm;
        S->rnorm = S->rel;
        if (S->rel < S->tol) {
            S->status = AEO_MG_CONVERGED;
            S->done = 1;
        }
    }
}

// phi0 -> x (FP64) after the cycles; the mean removed by shift_kernel
template <typename R>
__global__ void mg_store_kernel(Level<R> L, double* __restrict__ x) {
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= L.n) return;
    x[t] = double(L.phi[t]);
}

// |b0| of the standalone cycles; zero rhs ends before the first cycle
template <typename R>
__global__ void mg_bnorm_kernel(Level<R> L, PcgState* S, double* part) {
    double v[1] = {0.0};
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < L.n; t += (long long)gridDim.x * blockDim.x) {
        double bv = double(L.b[t]);
        v[0] += bv * bv;
    }
    double tot[1];
    if (reduce_last<1>(v, part, &S->counter, tot) && threadIdx.x == 0) {
        S->bnorm = sqrt(tot[0]);
        S->iters = 0;
        S->rel = 1.0;
        S->curvature = nan("");
        if (S->bnorm == 0.0) {
            S->status = AEO_MG_ZERO_RHS;
            S->done = 3;
        } else {
            S->status = AEO_MG_MAXIT;
            S->done = 0;
        }
    }
}

// ------------------------------------------------------------- host side

int blocks_for(long long n) { return (int)((n + TPB - 1) / TPB); }

struct MgBase {
    aeo_mg_config cfg{};
    std::string err;
    virtual ~MgBase() {}
    void fail(const std::string& m) { err = m; }
    virtual aeo_status init(const double* cx, const double* cy, const double* cz) = 0;
    virtual aeo_status solve(const double* b, double* x, bool device, aeo_mg_stats* st) = 0;
    virtual aeo_status cycles(const double* b, double* x, aeo_mg_stats* st) = 0;
    virtual aeo_status apply(const double* x, double* out) = 0;
    virtual aeo_status precondition(const double* r, double* z) = 0;
    virtual aeo_status profile(int what, int reps, double* ms) = 0;
    virtual int nlevels() const = 0;
    virtual void level_dims(int l, int32_t* d) const = 0;
    virtual int launches_per_iteration() const = 0;
};

#define CK(call)                                                                         \
    do {                                                                                 \
        cudaError_t e_ = (call);                                                         \
        if (e_ != cudaSuccess) {                                                         \
            fail(std::string(#call) + ": " + cudaGetErrorString(e_));                    \
            return AEO_ERR_CUDA;                                                         \
        }                                                                                \
    } while (0)

#define CKL()                                                                            \
    do {                                                                                 \
        cudaError_t e_ = cudaGetLastError();                                             \
        if (e_ != cudaSuccess) {                                                         \
            fail(std::string("kernel launch: ") + cudaGetErrorString(e_));               \
            return AEO_ERR_CUDA;                                                         \
        }                                                                                \
    } while (0)

// Four-face means of the face coefficients (_restrict_coeff,
// src/Multigrid.jl:465-496), on the host in FP64 at set-up.
void restrict_coeff(int nx, int ny, int nz, const std::vector<double>& cx, const std::vector<double>& cy,
                    const std::vector<double>& cz, int cnx, int cny, int cnz, std::vector<double>& Cx,
                    std::vector<double>& Cy, std::vector<double>& Cz) {
    auto mn = [](int a, int b) { return a < b ? a : b; };
    const int sx1 = nx + 1, sx2 = ny, sx3 = nz, sy1 = nx, sy2 = ny + 1, sy3 = nz, sz1 = nx, sz2 = ny, sz3 = nz + 1;
    Cx.assign((size_t)(cnx + 1) * cny * cnz, 0.0);
    Cy.assign((size_t)cnx * (cny + 1) * cnz, 0.0);
    Cz.assign((size_t)cnx * cny * (cnz + 1), 0.0);
    auto fx = [&](int i, int j, int k) { return cx[(size_t)(i - 1) + (size_t)sx1 * ((size_t)(j - 1) + (size_t)sx2 * (k - 1))]; };
    auto fy = [&](int i, int j, int k) { return cy[(size_t)(i - 1) + (size_t)sy1 * ((size_t)(j - 1) + (size_t)sy2 * (k - 1))]; };
    auto fz = [&](int i, int j, int k) { return cz[(size_t)(i - 1) + (size_t)sz1 * ((size_t)(j - 1) + (size_t)sz2 * (k - 1))]; };
    for (int K = 1; K <= cnz; ++K)
        for (int J = 1; J <= cny; ++J)
            for (int I = 1; I <= cnx + 1; ++I) {
                int i = 2 * I - 1;
                double s = 0;
                for (int dk = 0; dk <= 1; ++dk)
                    for (int dj = 0; dj <= 1; ++dj) s += fx(mn(i, sx1), mn(2 * J - 1 + dj, sx2), mn(2 * K - 1 + dk, sx3));
                Cx[(size_t)(I - 1) + (size_t)(cnx + 1) * ((size_t)(J - 1) + (size_t)cny * (K - 1))] = s * 0.25;
            }
    for (int K = 1; K <= cnz; ++K)
        for (int J = 1; J <= cny + 1; ++J)
            for (int I = 1; I <= cnx; ++I) {
                int j = 2 * J - 1;
                double s = 0;
                for (int dk = 0; dk <= 1; ++dk)
                    for (int di = 0; di <= 1; ++di) s += fy(mn(2 * I - 1 + di, sy1), mn(j, sy2), mn(2 * K - 1 + dk, sy3));
                Cy[(size_t)(I - 1) + (size_t)cnx * ((size_t)(J - 1) + (size_t)(cny + 1) * (K - 1))] = s * 0.25;
            }
    for (int K = 1; K <= cnz + 1; ++K)
        for (int J = 1; J <= cny; ++J)
            for (int I = 1; I <= cnx; ++I) {
                int k = 2 * K - 1;
                double s = 0;
                for (int dj = 0; dj <= 1; ++dj)
                    for (int di = 0; di <= 1; ++di) s += fz(mn(2 * I - 1 + di, sz1), mn(2 * J - 1 + dj, sz2), mn(k, sz3));
                Cz[(size_t)(I - 1) + (size_t)cnx * ((size_t)(J - 1) + (size_t)cny * (K - 1))] = s * 0.25;
            }
}

template <typename R, typename CT>
struct Mg : MgBase {
    cudaStream_t st = nullptr, st_body = nullptr;
    Bc bc{0, 0, 0};
    int nl = 0;
    long long n = 0;
    Level<R> L[MAX_LEVELS];
    std::vector<void*> allocs;
    const CT *ocx = nullptr, *ocy = nullptr, *ocz = nullptr;   // operator coefficients (FP64 or exact FP32)
    double *b = nullptr, *x = nullptr, *r = nullptr, *p = nullptr, *Ap = nullptr;
    double* part = nullptr;
    double* bmeans = nullptr;      // one device scalar per level
    PcgState* S = nullptr;
    PcgState* hS = nullptr;        // pinned host copy
    int* dzero = nullptr;          // a device flag that stays 0 (kernels run outside a solve)
    int coarse_staged = 0;
    size_t coarse_smem = 0;
    cudaGraphExec_t g_solve = nullptr, g_cycles = nullptr, g_pc = nullptr;
    int body_launches = 0;

    ~Mg() override {
        if (st) cudaStreamSynchronize(st);
        if (g_solve) cudaGraphExecDestroy(g_solve);
        if (g_cycles) cudaGraphExecDestroy(g_cycles);
        if (g_pc) cudaGraphExecDestroy(g_pc);
        for (void* a : allocs) cudaFree(a);
        if (hS) cudaFreeHost(hS);
        if (st) cudaStreamDestroy(st);
        if (st_body) cudaStreamDestroy(st_body);
    }

    template <typename T>
    aeo_status dalloc(T** ptr, size_t count) {
        void* a = nullptr;
        CK(cudaMalloc(&a, sizeof(T) * (count ? count : 1)));
        allocs.push_back(a);
        *ptr = reinterpret_cast<T*>(a);
        return AEO_OK;
    }

    int nlevels() const override { return nl; }
    void level_dims(int l, int32_t* d) const override {
        d[0] = L[l].nx;
        d[1] = L[l].ny;
        d[2] = L[l].nz;
    }
    int launches_per_iteration() const override { return body_launches; }

    aeo_status init(const double* cx, const double* cy, const double* cz) override {
        bc = {cfg.bc_x, cfg.bc_y, cfg.bc_z};
        CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        CK(cudaStreamCreateWithFlags(&st_body, cudaStreamNonBlocking));
        const bool coeff = cx != nullptr;
        int nx = cfg.nx, ny = cfg.ny, nz = cfg.nz;
        double dx = cfg.dx, dy = cfg.dy, dz = cfg.dz;
        n = (long long)nx * ny * nz;
        std::vector<double> hx, hy, hz;
        if (coeff) {
            hx.assign(cx, cx + (size_t)(nx + 1) * ny * nz);
            hy.assign(cy, cy + (size_t)nx * (ny + 1) * nz);
            hz.assign(cz, cz + (size_t)nx * ny * (nz + 1));
        }
        // the operator's coefficients: FP64, or FP32 when every value is exactly representable
        if (coeff) {
            bool exact = sizeof(CT) == sizeof(double);
            if (!exact) {
                exact = true;
                for (const std::vector<double>* v : {&hx, &hy, &hz})
                    for (double a : *v)
                        if (double(float(a)) != a) { exact = false; break; }
                if (!exact) {
                    fail("internal: FP32 operator coefficients requested for inexact values");
                    return AEO_ERR_STATE;
                }
            }
            CT *ax, *ay, *az;
            if (aeo_status s = dalloc(&ax, hx.size())) return s;
            if (aeo_status s = dalloc(&ay, hy.size())) return s;
            if (aeo_status s = dalloc(&az, hz.size())) return s;
            std::vector<CT> t;
            t.assign(hx.begin(), hx.end());
            CK(cudaMemcpy(ax, t.data(), sizeof(CT) * t.size(), cudaMemcpyHostToDevice));
            t.assign(hy.begin(), hy.end());
            CK(cudaMemcpy(ay, t.data(), sizeof(CT) * t.size(), cudaMemcpyHostToDevice));
            t.assign(hz.begin(), hz.end());
            CK(cudaMemcpy(az, t.data(), sizeof(CT) * t.size(), cudaMemcpyHostToDevice));
            ocx = ax; ocy = ay; ocz = az;
        }
        // the hierarchy (src/Multigrid.jl:572-591)
        if (aeo_status s = dalloc(&bmeans, MAX_LEVELS)) return s;
        CK(cudaMemset(bmeans, 0, sizeof(double) * MAX_LEVELS));
        std::vector<double> Cx, Cy, Cz;
        while (true) {
            Level<R>& V = L[nl];
            V.nx = nx; V.ny = ny; V.nz = nz;
            V.n = (long long)nx * ny * nz;
            V.ix2 = R(1) / (R(dx) * R(dx));   // one(T) / dx^2 (src/Multigrid.jl:162-164)
            V.iy2 = R(1) / (R(dy) * R(dy));
            V.iz2 = R(1) / (R(dz) * R(dz));
            if (aeo_status s = dalloc(&V.phi, V.n)) return s;
            if (aeo_status s = dalloc(&V.b, V.n)) return s;
            V.bmean = bmeans + nl;
            V.cx = V.cy = V.cz = nullptr;
            if (coeff) {
                if (nl == 0 && std::is_same<R, CT>::value) {
                    V.cx = reinterpret_cast<const R*>(ocx);
                    V.cy = reinterpret_cast<const R*>(ocy);
                    V.cz = reinterpret_cast<const R*>(ocz);
                } else {
                    R *ax, *ay, *az;
                    if (aeo_status s = dalloc(&ax, hx.size())) return s;
                    if (aeo_status s = dalloc(&ay, hy.size())) return s;
                    if (aeo_status s = dalloc(&az, hz.size())) return s;
                    std::vector<R> t(hx.begin(), hx.end());
                    CK(cudaMemcpy(ax, t.data(), sizeof(R) * t.size(), cudaMemcpyHostToDevice));
                    t.assign(hy.begin(), hy.end());
                    CK(cudaMemcpy(ay, t.data(), sizeof(R) * t.size(), cudaMemcpyHostToDevice));
                    t.assign(hz.begin(), hz.end());
                    CK(cudaMemcpy(az, t.data(), sizeof(R) * t.size(), cudaMemcpyHostToDevice));
                    V.cx = ax; V.cy = ay; V.cz = az;
                }
            }
            ++nl;
            bool cxo = nx % 2 == 0 && nx / 2 >= cfg.min_size;
            bool cyo = ny % 2 == 0 && ny / 2 >= cfg.min_size;
            bool czo = nz % 2 == 0 && nz / 2 >= cfg.min_size;
            if (!(cxo && cyo && czo) || nl == MAX_LEVELS) break;
            int cnx = nx / 2, cny = ny / 2, cnz = nz / 2;
            if (coeff) {
                restrict_coeff(nx, ny, nz, hx, hy, hz, cnx, cny, cnz, Cx, Cy, Cz);
                hx.swap(Cx); hy.swap(Cy); hz.swap(Cz);
            }
            nx = cnx; ny = cny; nz = cnz;
            dx *= 2; dy *= 2; dz *= 2;
        }
        const Level<R>& C = L[nl - 1];
        if (C.n > COARSE_MAX_CELLS) {
            fail("coarsest multigrid level has " + std::to_string(C.n) + " cells, above the " +
                 std::to_string(COARSE_MAX_CELLS) + " one block solves: give nx, ny, nz more factors of two");
            return AEO_ERR_ARGUMENT;
        }
        size_t cb = sizeof(R) * (2 * (size_t)C.n + (coeff ? (size_t)(C.nx + 1) * C.ny * C.nz +
                                                          (size_t)C.nx * (C.ny + 1) * C.nz +
                                                          (size_t)C.nx * C.ny * (C.nz + 1) : 0));
        coarse_staged = cb <= 200 * 1024;
        coarse_smem = coarse_staged ? cb : 0;
        if (coarse_smem > 48 * 1024)
            CK(cudaFuncSetAttribute(mg_coarsest_kernel<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)coarse_smem));
        if (aeo_status s = dalloc(&b, n)) return s;
        if (aeo_status s = dalloc(&x, n)) return s;
        if (aeo_status s = dalloc(&r, n)) return s;
        if (aeo_status s = dalloc(&p, n)) return s;
        if (aeo_status s = dalloc(&Ap, n)) return s;
        if (aeo_status s = dalloc(&part, (size_t)RED_BLOCKS * 8)) return s;
        if (aeo_status s = dalloc(&S, 1)) return s;
        if (aeo_status s = dalloc(&dzero, 1)) return s;
        CK(cudaMemset(dzero, 0, sizeof(int)));
        CK(cudaMallocHost(&hS, sizeof(PcgState)));
        PcgState h0{};
        h0.tol = cfg.tol;
        h0.n = double(n);
        h0.maxit = cfg.maxit;
        h0.project = (cfg.bc_x == 0 || cfg.bc_x == 1) && (cfg.bc_y == 0 || cfg.bc_y == 1) &&
                     (cfg.bc_z == 0 || cfg.bc_z == 1);
        h0.flexible = cfg.flexible;
        CK(cudaMemcpy(S, &h0, sizeof(PcgState), cudaMemcpyHostToDevice));
        CK(cudaMemset(part, 0, sizeof(double) * RED_BLOCKS * 8));
        return AEO_OK;
    }

    // ---- launch helpers (stream s) ----
    aeo_status launch_apply(cudaStream_t s, const double* in, double* out, int standalone) {
        const double ix2 = 1.0 / (cfg.dx * cfg.dx), iy2 = 1.0 / (cfg.dy * cfg.dy), iz2 = 1.0 / (cfg.dz * cfg.dz);
        pcg_apply_kernel<CT><<<RED_BLOCKS, TPB, 0, s>>>(in, out, ocx, ocy, ocz, cfg.nx, cfg.ny, cfg.nz, bc, ix2, iy2,
                                                        iz2, S, part, standalone);
        CKL();
        return AEO_OK;
    }

    int vcycle_launches() const {
        int c = 1;   // coarsest
        for (int l = 0; l < nl - 1; ++l) c += 2 * cfg.nu1 + 2 * cfg.nu2 + 2;
        return c;
    }

    // One V-cycle from phi = 0 with level-0 right-hand side r0 - mean (mg_vcycle!,
    // src/Multigrid.jl:706-739).  from_zero = false: level 0 keeps its phi and b
    // (the standalone cycles).
    aeo_status launch_vcycle(cudaStream_t s, const double* r0, bool from_zero, const int* done) {
        const double* mr = &S->mr;
        if (nl == 1) {
            if (!from_zero) {
                fail("internal: standalone cycles on a one-level hierarchy");
                return AEO_ERR_STATE;
            }
            mg_coarsest_kernel<R><<<1, COARSE_THREADS, coarse_smem, s>>>(L[0], bc, cfg.coarse_sweeps, coarse_staged,
                                                                         r0, mr, done);
            CKL();
            return AEO_OK;
        }
        for (int l = 0; l < nl - 1; ++l) {
            Level<R>& F = L[l];
            const int hb = blocks_for((long long)(F.nx / 2) * F.ny * F.nz);
            int sw0 = 0;
            if (l > 0 || from_zero) {
                mg_first_kernel<R><<<hb, TPB, 0, s>>>(F, bc, l == 0 ? r0 : nullptr, mr, done);
                CKL();
                mg_rbgs_kernel<R><<<hb, TPB, 0, s>>>(F, bc, 1, done);
                CKL();
                sw0 = 1;
            }
            for (int sw = sw0; sw < cfg.nu1; ++sw)
                for (int c = 0; c < 2; ++c) {
                    mg_rbgs_kernel<R><<<hb, TPB, 0, s>>>(F, bc, c, done);
                    CKL();
                }
            Level<R>& Cl = L[l + 1];
            int rb = blocks_for(Cl.n);
            if (rb > RED_BLOCKS) rb = RED_BLOCKS;
            mg_restrict_kernel<R><<<rb, TPB, 0, s>>>(F, Cl, bc, part, &S->counter, done);
            CKL();
        }
        Level<R>& C = L[nl - 1];
        mg_coarsest_kernel<R><<<1, COARSE_THREADS, coarse_smem, s>>>(C, bc, cfg.coarse_sweeps, coarse_staged, nullptr,
                                                                     mr, done);
        CKL();
        for (int l = nl - 2; l >= 0; --l) {
            Level<R>& F = L[l];
            mg_prolong_kernel<R><<<blocks_for(F.n), TPB, 0, s>>>(F, L[l + 1], bc, done);
            CKL();
            const int hb = blocks_for((long long)(F.nx / 2) * F.ny * F.nz);
            for (int sw = 0; sw < cfg.nu2; ++sw)
                for (int c = 0; c < 2; ++c) {
                    mg_rbgs_kernel<R><<<hb, TPB, 0, s>>>(F, bc, c, done);
                    CKL();
                }
        }
        return AEO_OK;
    }

    // the preconditioned residual z: level-0 phi, or r itself for plain CG
    aeo_status launch_rz_dir(cudaStream_t s, int first) {
        if (cfg.precond == AEO_PC_VCYCLE) {
            pcg_rz_kernel<R><<<RED_BLOCKS, TPB, 0, s>>>(r, L[0].phi, Ap, n, S, part, first);
            CKL();
            pcg_dir_kernel<R><<<RED_BLOCKS, TPB, 0, s>>>(p, L[0].phi, n, S, first);
        } else {
            pcg_rz_kernel<double><<<RED_BLOCKS, TPB, 0, s>>>(r, r, Ap, n, S, part, first);
            CKL();
            pcg_dir_kernel<double><<<RED_BLOCKS, TPB, 0, s>>>(p, r, n, S, first);
        }
        CKL();
        return AEO_OK;
    }

    // The conditional handle of the graph being captured on `st` (value 0 at
    // every launch until a kernel sets it).
    aeo_status make_handle(cudaGraphConditionalHandle* hdl) {
        cudaStreamCaptureStatus cs;
        cudaGraph_t g = nullptr;
        CK(cudaStreamGetCaptureInfo(st, &cs, nullptr, &g, nullptr, nullptr));
        if (cs != cudaStreamCaptureStatusActive) {
            fail("internal: stream is not capturing");
            return AEO_ERR_STATE;
        }
        CK(cudaGraphConditionalHandleCreate(hdl, g, 0, cudaGraphCondAssignDefault));
        return AEO_OK;
    }

    // Adds a WHILE node on `hdl` to the graph being captured on `st`, captures
    // `body` into its body graph on st_body, and continues the capture after it.
    template <typename F>
    aeo_status capture_while(cudaGraphConditionalHandle hdl, F body) {
        cudaStreamCaptureStatus cs;
        cudaGraph_t g = nullptr;
        const cudaGraphNode_t* deps = nullptr;
        size_t ndeps = 0;
        CK(cudaStreamGetCaptureInfo(st, &cs, nullptr, &g, &deps, &ndeps));
        if (cs != cudaStreamCaptureStatusActive) {
            fail("internal: stream is not capturing");
            return AEO_ERR_STATE;
        }
        cudaGraphNodeParams cp = {};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = hdl;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t node;
        std::vector<cudaGraphNode_t> dv(deps, deps + ndeps);
        CK(cudaGraphAddNode(&node, g, dv.data(), dv.size(), &cp));
        cudaGraph_t bodyg = cp.conditional.phGraph_out[0];
        CK(cudaStreamBeginCaptureToGraph(st_body, bodyg, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
        aeo_status bs = body(st_body);
        cudaGraph_t out = nullptr;
        cudaError_t e = cudaStreamEndCapture(st_body, &out);
        if (bs) return bs;
        if (e != cudaSuccess) {
            fail(std::string("cudaStreamEndCapture(body): ") + cudaGetErrorString(e));
            return AEO_ERR_CUDA;
        }
        CK(cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies));
        return AEO_OK;
    }

    aeo_status end_capture(cudaGraphExec_t* ex, aeo_status s) {
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(st, &g);
        if (s) {
            if (g) cudaGraphDestroy(g);
            return s;
        }
        if (e != cudaSuccess) {
            fail(std::string("cudaStreamEndCapture: ") + cudaGetErrorString(e));
            return AEO_ERR_CUDA;
        }
        cudaError_t e2 = cudaGraphInstantiate(ex, g, 0);
        cudaGraphDestroy(g);
        if (e2 != cudaSuccess) {
            fail(std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e2));
            return AEO_ERR_CUDA;
        }
        return AEO_OK;
    }

    // The solve graph: prologue, WHILE(one CG iteration), mean shift.  The
    // loop's condition is set by pcg_cond_kernel before the loop and at the
    // end of every iteration.
    aeo_status build_solve() {
        CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed));
        aeo_status s = [&]() -> aeo_status {
            cudaGraphConditionalHandle hdl;
            if (aeo_status q = make_handle(&hdl)) return q;
            pcg_mean_kernel<<<RED_BLOCKS, TPB, 0, st>>>(b, n, S, part, 0);
            CKL();
            pcg_init_kernel<<<RED_BLOCKS, TPB, 0, st>>>(b, r, x, n, S, part);
            CKL();
            if (cfg.precond == AEO_PC_VCYCLE)
                if (aeo_status q = launch_vcycle(st, r, true, &S->done)) return q;
            if (aeo_status q = launch_rz_dir(st, 1)) return q;
            pcg_cond_kernel<<<1, 1, 0, st>>>(S, hdl, 0);
            CKL();
            if (aeo_status q = capture_while(hdl, [&](cudaStream_t sb) -> aeo_status {
                    int c0 = 0;
                    if (aeo_status q2 = launch_apply(sb, p, Ap, 0)) return q2;
                    pcg_update_kernel<<<RED_BLOCKS, TPB, 0, sb>>>(x, r, p, Ap, n, S, part);
                    CKL();
                    c0 += 2;
                    if (cfg.precond == AEO_PC_VCYCLE) {
                        if (aeo_status q2 = launch_vcycle(sb, r, true, &S->done)) return q2;
                        c0 += vcycle_launches();
                    }
                    if (aeo_status q2 = launch_rz_dir(sb, 0)) return q2;
                    pcg_cond_kernel<<<1, 1, 0, sb>>>(S, hdl, 0);
                    CKL();
                    body_launches = c0 + 3;
                    return AEO_OK;
                }))
                return q;
            if (S_project()) {
                pcg_mean_kernel<<<RED_BLOCKS, TPB, 0, st>>>(x, n, S, part, 1);
                CKL();
                shift_kernel<<<RED_BLOCKS, TPB, 0, st>>>(x, n, S);
                CKL();
            }
            return AEO_OK;
        }();
        return end_capture(&g_solve, s);
    }

    bool S_project() const {
        return (cfg.bc_x == 0 || cfg.bc_x == 1) && (cfg.bc_y == 0 || cfg.bc_y == 1) && (cfg.bc_z == 0 || cfg.bc_z == 1);
    }

    aeo_status stats_out(aeo_mg_stats* o, bool relative) {
        CK(cudaMemcpyAsync(hS, S, sizeof(PcgState), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        if (o) {
            o->iterations = hS->iters;
            o->status = hS->status;
            o->residual = relative ? hS->rel : hS->rnorm;
            o->bnorm = hS->bnorm;
            o->curvature = hS->curvature;
            if (hS->status == AEO_MG_ZERO_RHS) o->residual = 0.0;
        }
        return AEO_OK;
    }

    aeo_status solve(const double* bin, double* xout, bool device, aeo_mg_stats* o) override {
        if (!g_solve)
            if (aeo_status s = build_solve()) return s;
        CK(cudaMemcpyAsync(b, bin, sizeof(double) * n, device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st));
        CK(cudaGraphLaunch(g_solve, st));
        CK(cudaMemcpyAsync(xout, x, sizeof(double) * n, device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, st));
        return stats_out(o, false);
    }

    aeo_status build_cycles() {
        if (nl == 1) {
            fail("standalone multigrid cycles need at least two levels");
            return AEO_ERR_ARGUMENT;
        }
        CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed));
        aeo_status s = [&]() -> aeo_status {
            cudaGraphConditionalHandle hdl;
            if (aeo_status q = make_handle(&hdl)) return q;
            pcg_mean_kernel<<<RED_BLOCKS, TPB, 0, st>>>(b, n, S, part, 0);
            CKL();
            mg_load_kernel_launch(st);
            CKL();
            mg_bnorm_kernel<R><<<RED_BLOCKS, TPB, 0, st>>>(L[0], S, part);
            CKL();
            pcg_cond_kernel<<<1, 1, 0, st>>>(S, hdl, 1);
            CKL();
            if (aeo_status q = capture_while(hdl, [&](cudaStream_t sb) -> aeo_status {
                    if (aeo_status q2 = launch_vcycle(sb, nullptr, false, &S->done)) return q2;
                    mg_resnorm_kernel<R><<<RED_BLOCKS, TPB, 0, sb>>>(L[0], bc, S, part);
                    CKL();
                    pcg_cond_kernel<<<1, 1, 0, sb>>>(S, hdl, 1);
                    CKL();
                    return AEO_OK;
                }))
                return q;
            mg_store_kernel<R><<<blocks_for(n), TPB, 0, st>>>(L[0], x);
            CKL();
            if (S_project()) {
                pcg_mean_kernel<<<RED_BLOCKS, TPB, 0, st>>>(x, n, S, part, 1);
                CKL();
                shift_kernel<<<RED_BLOCKS, TPB, 0, st>>>(x, n, S);
                CKL();
            }
            return AEO_OK;
        }();
        return end_capture(&g_cycles, s);
    }

    void mg_load_kernel_launch(cudaStream_t s) {
        // b0 = b - mean(b) (the loaded right-hand side, _load_rhs!), phi0 = 0
        mg_load_kernel<R><<<blocks_for(n), TPB, 0, s>>>(L[0], b, &S->mb);
    }

    aeo_status cycles(const double* bin, double* xout, aeo_mg_stats* o) override {
        if (!g_cycles)
            if (aeo_status s = build_cycles()) return s;
        CK(cudaMemcpyAsync(b, bin, sizeof(double) * n, cudaMemcpyHostToDevice, st));
        CK(cudaGraphLaunch(g_cycles, st));
        CK(cudaMemcpyAsync(xout, x, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
        return stats_out(o, true);
    }

    aeo_status apply(const double* xin, double* out) override {
        CK(cudaMemcpyAsync(p, xin, sizeof(double) * n, cudaMemcpyHostToDevice, st));
        if (aeo_status s = launch_apply(st, p, Ap, 1)) return s;
        CK(cudaMemcpyAsync(out, Ap, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        return AEO_OK;
    }

    // z = M r: the load of r with its mean (as the solve's prologue), one cycle,
    // then z - mean(z) on the host side of the copy
    aeo_status precondition(const double* rin, double* zout) override {
        if (cfg.precond != AEO_PC_VCYCLE) {
            std::memcpy(zout, rin, sizeof(double) * n);
        } else {
            CK(cudaMemcpyAsync(b, rin, sizeof(double) * n, cudaMemcpyHostToDevice, st));
            pcg_mean_kernel<<<RED_BLOCKS, TPB, 0, st>>>(b, n, S, part, 0);
            CKL();
            pcg_init_kernel<<<RED_BLOCKS, TPB, 0, st>>>(b, r, x, n, S, part);
            CKL();
            // pcg_init stored mean(r) in S->mr; the cycle runs even for a zero r
            if (aeo_status s = launch_vcycle(st, r, true, dzero)) return s;
            std::vector<R> hz((size_t)n);
            CK(cudaMemcpyAsync(hz.data(), L[0].phi, sizeof(R) * n, cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            for (long long q = 0; q < n; ++q) zout[q] = double(hz[q]);
        }
        if (S_project()) {
            double s = 0;
            for (long long q = 0; q < n; ++q) s += zout[q];
            s /= double(n);
            for (long long q = 0; q < n; ++q) zout[q] -= s;
        }
        return AEO_OK;
    }

    aeo_status profile(int what, int reps, double* ms) override {
        if (what == 0 && !g_solve) {
            fail("profile: no solve has run yet");
            return AEO_ERR_STATE;
        }
        cudaEvent_t e0, e1;
        CK(cudaEventCreate(&e0));
        CK(cudaEventCreate(&e1));
        int* dz = dzero;
        auto run = [&]() -> aeo_status {
            switch (what) {
            case 0: CK(cudaGraphLaunch(g_solve, st)); return AEO_OK;
            case 1: {
                Level<R>& F = L[0];
                if (F.nx % 2) { fail("profile: odd finest nx"); return AEO_ERR_ARGUMENT; }
                mg_rbgs_kernel<R><<<blocks_for((long long)(F.nx / 2) * F.ny * F.nz), TPB, 0, st>>>(F, bc, 0, dz);
                CKL();
                return AEO_OK;
            }
            case 2: return launch_apply(st, p, Ap, 1);
            case 3: return launch_vcycle(st, r, true, dz);
            default: fail("profile: unknown part"); return AEO_ERR_ARGUMENT;
            }
        };
        for (int w = 0; w < 3; ++w)
            if (aeo_status s = run()) return s;
        CK(cudaEventRecord(e0, st));
        for (int i = 0; i < reps; ++i)
            if (aeo_status s = run()) return s;
        CK(cudaEventRecord(e1, st));
        CK(cudaEventSynchronize(e1));
        float t = 0;
        CK(cudaEventElapsedTime(&t, e0, e1));
        *ms = double(t) / (reps > 0 ? reps : 1);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        return AEO_OK;
    }
};

std::string g_mg_error;

}  // namespace

struct aeo_mg {
    MgBase* core;
};

extern "C" {

aeo_status aeo_mg_create(const aeo_mg_config* c, const double* cx, const double* cy, const double* cz, aeo_mg** out) {
    if (!out) { g_mg_error = "out is NULL"; return AEO_ERR_ARGUMENT; }
    *out = nullptr;
    if (!c) { g_mg_error = "config is NULL"; return AEO_ERR_ARGUMENT; }
    if (c->nx < 1 || c->ny < 1 || c->nz < 1) { g_mg_error = "grid dimensions must be positive"; return AEO_ERR_ARGUMENT; }
    if (!(c->dx > 0) || !(c->dy > 0) || !(c->dz > 0)) { g_mg_error = "spacings must be positive"; return AEO_ERR_ARGUMENT; }
    for (int b : {c->bc_x, c->bc_y, c->bc_z})
        if (b != AEO_MG_PERIODIC && b != AEO_MG_NEUMANN) {
            g_mg_error = "unsupported BC (use periodic or Neumann, src/Multigrid.jl:62-66)";
            return AEO_ERR_ARGUMENT;
        }
    if ((cx == nullptr) != (cy == nullptr) || (cx == nullptr) != (cz == nullptr)) {
        g_mg_error = "give all three face coefficient arrays or none";
        return AEO_ERR_ARGUMENT;
    }
    if (c->precision != AEO_PREC_FP64 && c->precision != AEO_PREC_FP32_MIXED) { g_mg_error = "unknown precision"; return AEO_ERR_ARGUMENT; }
    if (c->precond != AEO_PC_IDENTITY && c->precond != AEO_PC_VCYCLE) { g_mg_error = "unknown preconditioner"; return AEO_ERR_ARGUMENT; }
    if (!(c->tol >= 0) || c->maxit < 0 || c->nu1 < 1 || c->nu2 < 0 || c->coarse_sweeps < 0 || c->min_size < 1) {
        g_mg_error = "invalid tol / maxit / sweep counts (nu1 >= 1)";
        return AEO_ERR_ARGUMENT;
    }
    long long ncell = (long long)c->nx * c->ny * c->nz;
    if (ncell > (1LL << 31)) { g_mg_error = "grid above 2^31 cells"; return AEO_ERR_ARGUMENT; }
    if (cudaSetDevice(c->device) != cudaSuccess) { g_mg_error = "cudaSetDevice failed"; return AEO_ERR_CUDA; }
    bool exact32 = false;
    if (c->precision == AEO_PREC_FP32_MIXED && cx) {
        exact32 = true;
        const long long nxs = (long long)(c->nx + 1) * c->ny * c->nz, nys = (long long)c->nx * (c->ny + 1) * c->nz,
                        nzs = (long long)c->nx * c->ny * (c->nz + 1);
        for (long long q = 0; q < nxs && exact32; ++q) exact32 = double(float(cx[q])) == cx[q];
        for (long long q = 0; q < nys && exact32; ++q) exact32 = double(float(cy[q])) == cy[q];
        for (long long q = 0; q < nzs && exact32; ++q) exact32 = double(float(cz[q])) == cz[q];
    }
    MgBase* m = nullptr;
    if (c->precision == AEO_PREC_FP64) m = new (std::nothrow) Mg<double, double>();
    else if (exact32) m = new (std::nothrow) Mg<float, float>();
    else m = new (std::nothrow) Mg<float, double>();
    if (!m) { g_mg_error = "out of host memory"; return AEO_ERR_CUDA; }
    m->cfg = *c;
    if (aeo_status s = m->init(cx, cy, cz)) {
        g_mg_error = m->err;
        delete m;
        return s;
    }
    aeo_mg* h = new (std::nothrow) aeo_mg;
    if (!h) { delete m; g_mg_error = "out of host memory"; return AEO_ERR_CUDA; }
    h->core = m;
    *out = h;
    return AEO_OK;
}

aeo_status aeo_mg_destroy(aeo_mg* h) {
    if (!h) return AEO_OK;
    cudaSetDevice(h->core->cfg.device);
    delete h->core;
    delete h;
    return AEO_OK;
}

#define MG_ENTER(h)                                                    \
    if (!h) return AEO_ERR_ARGUMENT;                                   \
    if (cudaSetDevice(h->core->cfg.device) != cudaSuccess) {           \
        h->core->fail("cudaSetDevice failed");                         \
        return AEO_ERR_CUDA;                                           \
    }

aeo_status aeo_mg_levels(aeo_mg* h, int32_t* nlevels, int32_t* dims) {
    MG_ENTER(h);
    if (nlevels) *nlevels = h->core->nlevels();
    if (dims)
        for (int l = 0; l < h->core->nlevels(); ++l) h->core->level_dims(l, dims + 3 * l);
    return AEO_OK;
}

aeo_status aeo_mg_solve(aeo_mg* h, const double* b, double* x, aeo_mg_stats* st) {
    MG_ENTER(h);
    if (!b || !x) { h->core->fail("b and x must not be NULL"); return AEO_ERR_ARGUMENT; }
    return h->core->solve(b, x, false, st);
}

aeo_status aeo_mg_solve_device(aeo_mg* h, const double* b, double* x, aeo_mg_stats* st) {
    MG_ENTER(h);
    if (!b || !x) { h->core->fail("b and x must not be NULL"); return AEO_ERR_ARGUMENT; }
    return h->core->solve(b, x, true, st);
}

aeo_status aeo_mg_vcycle_solve(aeo_mg* h, const double* b, double* x, aeo_mg_stats* st) {
    MG_ENTER(h);
    if (!b || !x) { h->core->fail("b and x must not be NULL"); return AEO_ERR_ARGUMENT; }
    return h->core->cycles(b, x, st);
}

aeo_status aeo_mg_apply(aeo_mg* h, const double* x, double* out) {
    MG_ENTER(h);
    if (!x || !out) { h->core->fail("x and out must not be NULL"); return AEO_ERR_ARGUMENT; }
    return h->core->apply(x, out);
}

aeo_status aeo_mg_precondition(aeo_mg* h, const double* r, double* z) {
    MG_ENTER(h);
    if (!r || !z) { h->core->fail("r and z must not be NULL"); return AEO_ERR_ARGUMENT; }
    return h->core->precondition(r, z);
}

aeo_status aeo_mg_profile(aeo_mg* h, int32_t what, int32_t reps, double* ms) {
    MG_ENTER(h);
    if (!ms || reps < 1) { h->core->fail("profile: ms NULL or reps < 1"); return AEO_ERR_ARGUMENT; }
    return h->core->profile(what, reps, ms);
}

int32_t aeo_mg_launches_per_iteration(const aeo_mg* h) { return h ? h->core->launches_per_iteration() : 0; }

const char* aeo_mg_last_error(const aeo_mg* h) { return h ? h->core->err.c_str() : g_mg_error.c_str(); }

}  // extern "C"
