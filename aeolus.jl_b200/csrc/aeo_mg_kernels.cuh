// aeo_mg_kernels.cuh -- device code of the multigrid-preconditioned CG
// (included by aeo_mgpcg.cu).  Indices are 32-bit (levels below 2^30
// cells); stencil kernels run on 3-D grids (x lanes, y rows, z planes), the
// reduction kernels on a fixed grid that loops over rows, so no kernel
// divides a 64-bit index.
#pragma once

#include <cuda_runtime.h>

#include <cfloat>

namespace mgk {

constexpr int TPB = 256;
constexpr int RED_BLOCKS = 1184;       // 8 x 148 SMs (2048 threads an SM): the fixed grid of every FP64 reduction
constexpr int COARSE_THREADS = 1024;
constexpr int COARSE_MAX_CELLS = 16384;
// Programmatic dependent launch: a kernel launched with the programmatic
// stream serialisation attribute may start while the kernel before it is
// finishing; it waits here, before its first read of anything an earlier
// kernel wrote, for that kernel's completion and memory (a no-op when the
// launch had no such attribute).
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

constexpr int RB_X = 32, RB_Y = 8;     // block of the 3-D stencil grids

enum { MG_CONVERGED = 0, MG_MAXIT = 1, MG_BREAKDOWN = 2, MG_ZERO_RHS = 3 };

template <typename R> struct Eps;
template <> struct Eps<double> { static __device__ __host__ double v() { return DBL_EPSILON; } };
template <> struct Eps<float> { static __device__ __host__ float v() { return FLT_EPSILON; } };

struct Bc { int x, y, z; };            // 0 periodic, 1 Neumann

// Device scalars of one solve, written by last blocks of reductions.
struct PcgState {
    double tol, n;
    double mb, bnorm, rz, pAp, alpha, beta, m, mr, rnorm, curvature, mx, rel;
    int iters, maxit, status, done;
    int project, flexible;
    unsigned counter;
    // learned preconditioner: in use (learned), at set-up (learned_init), the
    // iteration it was dropped at (-1: never), slow iterations in a row, the
    // previous residual norm and the stagnation ratio
    int learned, learned_init, fallback_at, slow;
    double rprev, stag;
};

// Face coefficients of one level: value arrays, or one-byte codes into a
// table of the level's distinct values (exact: the table holds the values
// themselves), or none (the constant-coefficient Laplacian).
template <typename V> struct Coef {
    const V* cx = nullptr;
    const V* cy = nullptr;
    const V* cz = nullptr;
    const unsigned char* kx = nullptr;
    const unsigned char* ky = nullptr;
    const unsigned char* kz = nullptr;
    const V* tab = nullptr;
    __host__ __device__ bool var() const { return cx != nullptr || kx != nullptr; }
    __device__ __forceinline__ V x(int i) const { return kx ? __ldg(tab + kx[i]) : cx[i]; }
    __device__ __forceinline__ V y(int i) const { return ky ? __ldg(tab + ky[i]) : cy[i]; }
    __device__ __forceinline__ V z(int i) const { return kz ? __ldg(tab + kz[i]) : cz[i]; }
};

template <typename R> struct Level {
    int nx, ny, nz, n;
    R ix2, iy2, iz2;
    R* phi;
    R* b;
    R* r;                               // residual (every level but the coarsest)
    Coef<R> c;
    double* bmean;                      // mean of b to subtract before use (device scalar)
};

__device__ __forceinline__ int wm(int i, int n, int bc) { return i > 0 ? i - 1 : (bc == 0 ? n - 1 : 0); }
__device__ __forceinline__ int wp(int i, int n, int bc) { return i < n - 1 ? i + 1 : (bc == 0 ? 0 : n - 1); }

// Neighbour and face indices of cell (i, j, k); halos as index maps
// (periodic wrap, Neumann mirror = the cell itself).
struct Idx {
    int q, xm, xp, ym, yp, zm, zp, cx, cy, sy, sz;
};

__device__ __forceinline__ Idx make_idx(int i, int j, int k, int nx, int ny, int nz, Bc bc) {
    Idx d;
    const int pl = nx * ny;
    const int row = pl * k + nx * j;
    d.q = row + i;
    d.xm = row + wm(i, nx, bc.x);
    d.xp = row + wp(i, nx, bc.x);
    d.ym = pl * k + nx * wm(j, ny, bc.y) + i;
    d.yp = pl * k + nx * wp(j, ny, bc.y) + i;
    d.zm = pl * wm(k, nz, bc.z) + nx * j + i;
    d.zp = pl * wp(k, nz, bc.z) + nx * j + i;
    d.cx = i + (nx + 1) * (j + ny * k);
    d.cy = i + nx * (j + (ny + 1) * k);
    d.sy = nx;
    d.sz = pl;
    return d;
}

// _Aphi of _ConstOp / _VarOp (src/Multigrid.jl:174-193) in the value type V.
template <typename V, typename C>
__device__ __forceinline__ V aphi(const V* f, const Idx& d, const Coef<C>& cf, V ix2, V iy2, V iz2) {
    V c = f[d.q];
    if (!cf.var())
        return (f[d.xp] - V(2) * c + f[d.xm]) * ix2 + (f[d.yp] - V(2) * c + f[d.ym]) * iy2 +
               (f[d.zp] - V(2) * c + f[d.zm]) * iz2;
    V fxp = V(cf.x(d.cx + 1)), fxm = V(cf.x(d.cx));
    V fyp = V(cf.y(d.cy + d.sy)), fym = V(cf.y(d.cy));
    V fzp = V(cf.z(d.q + d.sz)), fzm = V(cf.z(d.q));
    return (fxp * (f[d.xp] - c) - fxm * (c - f[d.xm])) * ix2 + (fyp * (f[d.yp] - c) - fym * (c - f[d.ym])) * iy2 +
           (fzp * (f[d.zp] - c) - fzm * (c - f[d.zm])) * iz2;
}

// The coefficient form of a level, as a kernel template parameter: the
// constant-coefficient Laplacian, one-byte codes into the level's value
// table (staged in shared memory), or per-face values.
enum { CF_CONST = 0, CF_CODES = 1, CF_VALUES = 2 };

template <typename R, int CF>
__device__ __forceinline__ R face_coef(const R* vals, const unsigned char* codes, const R* stab, int f) {
    // read-only for every kernel that takes them: the non-coherent path, which
    // the compiler may also schedule ahead of the kernel's own stores
    if (CF == CF_CODES) return stab[__ldg(codes + f)];
    return __ldg(vals + f);
}

// The six neighbours of cell q = (i, j, k): the interior steps, or at a
// boundary the periodic wrap / the Neumann mirror (the cell itself) -- the
// maps of make_idx, formed from q with adds and selects.
struct Nbr {
    int xm, xp, ym, yp, zm, zp;
};
__device__ __forceinline__ Nbr nbr_of(int q, int i, int j, int k, int nx, int ny, int nz, int pl, Bc bc) {
    Nbr n;
    n.xm = i > 0 ? q - 1 : (bc.x == 0 ? q + nx - 1 : q);
    n.xp = i < nx - 1 ? q + 1 : (bc.x == 0 ? q - (nx - 1) : q);
    n.ym = j > 0 ? q - nx : (bc.y == 0 ? q + (ny - 1) * nx : q);
    n.yp = j < ny - 1 ? q + nx : (bc.y == 0 ? q - (ny - 1) * nx : q);
    n.zm = k > 0 ? q - pl : (bc.z == 0 ? q + (nz - 1) * pl : q);
    n.zp = k < nz - 1 ? q + pl : (bc.z == 0 ? q - (nz - 1) * pl : q);
    return n;
}

// the smoother's division: IEEE in FP64 (the reference's arithmetic); the
// FP32 cycle (a preconditioner of FP64 CG) divides with the fast reciprocal
// (within 2 ulp)
__device__ __forceinline__ double gs_div(double a, double b) { return a / b; }
__device__ __forceinline__ float gs_div(float a, float b) { return __fdividef(a, b); }

// One RB-GS update (src/Multigrid.jl:311-336) from the six neighbour values
// and face coefficients; false for a fully blocked cell (|diag| < eps),
// which keeps its value.
template <typename R, int CF>
__device__ __forceinline__ bool gs_vals(R nxp, R nxm, R nyp, R nym, R nzp, R nzm, R fxp, R fxm, R fyp, R fym, R fzp,
                                        R fzm, R bval, R ix2, R iy2, R iz2, R* out) {
    if (CF == CF_CONST) {
        const R diag = -R(2) * (ix2 + iy2 + iz2);
        const R off = (nxp + nxm) * ix2 + (nyp + nym) * iy2 + (nzp + nzm) * iz2;
        *out = gs_div(bval - off, diag);
        return true;
    }
    const R diag = -((fxp + fxm) * ix2 + (fyp + fym) * iy2 + (fzp + fzm) * iz2);
    if (fabs(diag) < Eps<R>::v()) return false;
    const R off = (fxp * nxp + fxm * nxm) * ix2 + (fyp * nyp + fym * nym) * iy2 + (fzp * nzp + fzm * nzm) * iz2;
    *out = gs_div(bval - off, diag);
    return true;
}

template <typename R>
__device__ __forceinline__ bool gs_diag(const Idx& d, const Level<R>& L, R* diag) {
    if (!L.c.var()) {
        *diag = -R(2) * (L.ix2 + L.iy2 + L.iz2);
        return true;
    }
    R fxp = L.c.x(d.cx + 1), fxm = L.c.x(d.cx);
    R fyp = L.c.y(d.cy + d.sy), fym = L.c.y(d.cy);
    R fzp = L.c.z(d.q + d.sz), fzm = L.c.z(d.q);
    *diag = -((fxp + fxm) * L.ix2 + (fyp + fym) * L.iy2 + (fzp + fzm) * L.iz2);
    return !(fabs(*diag) < Eps<R>::v());
}

// ---------------------------------------------------------------- reductions

__device__ __forceinline__ int tid() { return threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z); }
__device__ __forceinline__ int nthreads() { return blockDim.x * blockDim.y * blockDim.z; }

__device__ __forceinline__ double warp_sum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// Block sum of K values, valid in thread 0; fixed order (deterministic).
template <int K>
__device__ __forceinline__ void block_sum(double (&v)[K]) {
    __shared__ double sh[K][32];
    const int t = tid(), w = t >> 5, l = t & 31, nw = (nthreads() + 31) >> 5;
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
// in block order and returns true with the totals in thread 0.
template <int K>
__device__ bool reduce_last(double (&v)[K], double* part, unsigned* counter, double (&tot)[K]) {
    __shared__ bool last;
    block_sum<K>(v);
    const int nb = gridDim.x * gridDim.y * gridDim.z;
    const int bid = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
    if (tid() == 0) {
#pragma unroll
        for (int q = 0; q < K; ++q) part[q * nb + bid] = v[q];
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
    for (int b = tid(); b < nb; b += nthreads())
#pragma unroll
        for (int q = 0; q < K; ++q) a[q] += __ldcg(&part[q * nb + b]);
    block_sum<K>(a);
    if (tid() == 0) {
#pragma unroll
        for (int q = 0; q < K; ++q) tot[q] = a[q];
        *counter = 0u;
    }
    return true;
}

// ------------------------------------------------------------ CG kernels
// (pcg!/_pcg!, src/Backends.jl:1526-1589; definite = :negative).  Vector
// kernels: 1-D grid-stride over the n cells on RED_BLOCKS blocks.

#define GRID_STRIDE(q, n) for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < (n); q += gridDim.x * blockDim.x)

// sum of a -> S->mb (mode 0) or S->mx (mode 1), over n when the mean is projected
__global__ void pcg_mean_kernel(const double* __restrict__ a, int n, PcgState* S, double* part, int mode) {
    double v[1] = {0.0};
    GRID_STRIDE(q, n) v[0] += a[q];
    double t[1];
    if (reduce_last<1>(v, part, &S->counter, t) && tid() == 0) {
        double m = S->project ? t[0] / S->n : 0.0;
        if (mode == 0) S->mb = m; else S->mx = m;
    }
}

// r = b - mb (zero guess), x = 0; (|b - mb|^2, sum r); a zero rhs ends the solve
__global__ void pcg_init_kernel(const double* __restrict__ b, double* __restrict__ r, double* __restrict__ x, int n,
                                PcgState* S, double* part) {
    const double mb = S->mb;
    double v[2] = {0.0, 0.0};
    GRID_STRIDE(q, n) {
        double bv = b[q] - mb;
        r[q] = bv;
        x[q] = 0.0;
        v[0] += bv * bv;
        v[1] += bv;
    }
    double t[2];
    if (reduce_last<2>(v, part, &S->counter, t) && tid() == 0) {
        S->bnorm = sqrt(t[0]);
        S->mr = S->project ? t[1] / S->n : 0.0;
        S->iters = 0;
        S->curvature = nan("");
        S->rz = 0.0;
        S->alpha = S->beta = 0.0;
        S->learned = S->learned_init;
        S->fallback_at = -1;
        S->slow = 0;
        if (S->bnorm == 0.0) {
            S->status = MG_ZERO_RHS;
            S->done = 3;
        } else {
            S->status = MG_MAXIT;
            S->done = 0;
        }
    }
}

// Ap = A p with p.Ap; the last block forms alpha or flags a breakdown.
// Block (32, 8): lanes along x, warps over rows, rows looped on a fixed grid.
// The coefficient form is a template parameter (codes: the table, padded to
// 256 entries, staged in shared memory); the arithmetic of aphi in FP64.
template <typename C, int CF>
__global__ void __launch_bounds__(RB_X * RB_Y) pcg_apply_kernel(const double* __restrict__ p, double* __restrict__ Ap,
                                                               Coef<C> cf, int nx, int ny, int nz, Bc bc, double ix2,
                                                               double iy2, double iz2, PcgState* S, double* part,
                                                               int standalone) {
    pdl_wait();
    __shared__ double stab[CF == CF_CODES ? 256 : 1];
    if (!standalone && S->done) return;
    if (CF == CF_CODES) {
        for (int q = tid(); q < 256; q += nthreads()) stab[q] = double(cf.tab[q]);
        __syncthreads();
    }
    double v[1] = {0.0};
    const int nrows = ny * nz, pl = nx * ny;
    for (int row = blockIdx.x * blockDim.y + threadIdx.y; row < nrows; row += gridDim.x * blockDim.y) {
        const int j = row % ny, k = row / ny;
        for (int i = threadIdx.x; i < nx; i += blockDim.x) {
            const int q = i + nx * row;
            const Nbr n = nbr_of(q, i, j, k, nx, ny, nz, pl, bc);
            // p and the coefficients are read-only here: the non-coherent path
            const double c = __ldg(p + q);
            const double pxp = __ldg(p + n.xp), pxm = __ldg(p + n.xm), pyp = __ldg(p + n.yp), pym = __ldg(p + n.ym);
            const double pzp = __ldg(p + n.zp), pzm = __ldg(p + n.zm);
            double a;
            if (CF == CF_CONST) {
                a = (pxp - 2.0 * c + pxm) * ix2 + (pyp - 2.0 * c + pym) * iy2 + (pzp - 2.0 * c + pzm) * iz2;
            } else {
                const int fx = q + j + ny * k, fy = q + nx * k;
                const double fxm = CF == CF_CODES ? stab[__ldg(cf.kx + fx)] : double(__ldg(cf.cx + fx));
                const double fxp = CF == CF_CODES ? stab[__ldg(cf.kx + fx + 1)] : double(__ldg(cf.cx + fx + 1));
                const double fym = CF == CF_CODES ? stab[__ldg(cf.ky + fy)] : double(__ldg(cf.cy + fy));
                const double fyp = CF == CF_CODES ? stab[__ldg(cf.ky + fy + nx)] : double(__ldg(cf.cy + fy + nx));
                const double fzm = CF == CF_CODES ? stab[__ldg(cf.kz + q)] : double(__ldg(cf.cz + q));
                const double fzp = CF == CF_CODES ? stab[__ldg(cf.kz + q + pl)] : double(__ldg(cf.cz + q + pl));
                a = (fxp * (pxp - c) - fxm * (c - pxm)) * ix2 + (fyp * (pyp - c) - fym * (c - pym)) * iy2 +
                    (fzp * (pzp - c) - fzm * (c - pzm)) * iz2;
            }
            Ap[q] = a;
            v[0] += c * a;
        }
    }
    double t[1];
    if (reduce_last<1>(v, part, &S->counter, t) && tid() == 0 && !standalone) {
        double pAp = t[0];
        S->pAp = pAp;
        S->curvature = pAp;
        if (!(fabs(pAp) > DBL_EPSILON * fabs(S->rz))) {
            S->status = MG_BREAKDOWN;
            S->done = 2;
        } else {
            S->alpha = S->rz / pAp;
        }
    }
}

// x += alpha p, r -= alpha Ap; (r.r, sum r); the convergence test
__global__ void pcg_update_kernel(double* __restrict__ x, double* __restrict__ r, const double* __restrict__ p,
                                  const double* __restrict__ Ap, int n, PcgState* S, double* part) {
    pdl_wait();
    if (S->done) return;
    const double alpha = S->alpha;
    double v[2] = {0.0, 0.0};
    GRID_STRIDE(q, n) {
        x[q] = x[q] + alpha * p[q];
        double rv = r[q] - alpha * Ap[q];
        r[q] = rv;
        v[0] += rv * rv;
        v[1] += rv;
    }
    double t[2];
    if (reduce_last<2>(v, part, &S->counter, t) && tid() == 0) {
        S->iters += 1;
        S->rnorm = sqrt(t[0]);
        S->mr = S->project ? t[1] / S->n : 0.0;
        if (S->rnorm <= S->tol * S->bnorm) {
            S->status = MG_CONVERGED;
            S->done = 1;
        }
    }
}

// after z = M r: (r.r, r.z, sum z, sum r, z.Ap, sum Ap); the deflation mean
// m = sum z / n, (r.z) -= m sum r, and beta (Polak-Ribiere when flexible)
template <typename Z>
__global__ void pcg_rz_kernel(const double* __restrict__ r, const Z* __restrict__ z, const double* __restrict__ Ap,
                              int n, PcgState* S, double* part, int first) {
    pdl_wait();
    if (S->done) return;
    const bool flex = S->flexible && !first;
    double v[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    GRID_STRIDE(q, n) {
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
    if (reduce_last<6>(v, part, &S->counter, t) && tid() == 0) {
        double m = S->project ? t[2] / S->n : 0.0;
        double rzn = t[1];
        if (S->project) rzn -= m * t[3];
        S->m = m;
        if (first) {
            S->rz = rzn;
            S->beta = 0.0;
            S->rnorm = sqrt(t[0]);
            S->rprev = S->rnorm;
            if (S->rnorm <= S->tol * S->bnorm) {
                S->status = MG_CONVERGED;
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
__global__ void pcg_dir_kernel(double* __restrict__ p, const Z* __restrict__ z, int n, const PcgState* S, int first) {
    pdl_wait();
    if (S->done) return;
    const double m = S->m, beta = S->beta;
    GRID_STRIDE(q, n) p[q] = first ? double(z[q]) - m : (double(z[q]) - m) + beta * p[q];
}

// z = r / diag(A), the Jacobi preconditioner (1/diag precomputed; 0 on a
// fully blocked cell)
__global__ void pcg_jacobi_kernel(double* __restrict__ z, const double* __restrict__ r,
                                  const double* __restrict__ invd, int n, const PcgState* S) {
    pdl_wait();
    if (S->done) return;
    GRID_STRIDE(q, n) z[q] = r[q] * invd[q];
}

// the loop condition of the WHILE node: mode 0 CG, mode 1 multigrid cycles
__global__ void pcg_cond_kernel(PcgState* S, cudaGraphConditionalHandle h, int mode) {
    unsigned go = (S->done == 0 && S->iters < S->maxit) ? 1u : 0u;
    if (mode == 0 && S->done == 0 && S->iters >= S->maxit) S->status = MG_MAXIT;
    cudaGraphSetConditional(h, go);
}

// The preconditioner of the next application (the IF node's value): the
// learned network while it keeps the residual falling; from the second
// iteration in a row whose residual fell by less than the stagnation ratio
// on, the multigrid cycle for the rest of the solve.
__global__ void pcg_select_kernel(PcgState* S, cudaGraphConditionalHandle h) {
    if (S->done == 0 && S->learned) {
        if (S->rnorm > S->stag * S->rprev) {
            if (++S->slow >= 2) {
                S->learned = 0;
                S->fallback_at = S->iters;
            }
        } else {
            S->slow = 0;
        }
    }
    S->rprev = S->rnorm;
    cudaGraphSetConditional(h, (S->done == 0 && S->learned) ? 1u : 0u);
}

// the iterate and residual after `iters` updates into slot iters of the
// history (residual -> error training pairs of the plain solve)
__global__ void pcg_harvest_kernel(const double* __restrict__ x, const double* __restrict__ r, double* __restrict__ hx,
                                   double* __restrict__ hr, int n, int cap, const PcgState* S) {
    const int slot = S->iters;
    if (slot >= cap) return;
    GRID_STRIDE(q, n) {
        hx[(size_t)slot * n + q] = x[q];
        hr[(size_t)slot * n + q] = r[q];
    }
}

__global__ void shift_kernel(double* __restrict__ x, int n, const PcgState* S) {
    const double m = S->mx;
    GRID_STRIDE(q, n) x[q] = x[q] - m;
}

// ------------------------------------------------------- multigrid kernels
// 3-D grids: x lanes over half-rows (RB) or cells, y over rows j, z over planes k.

// The first half-sweep of a level whose phi starts at zero: every neighbour
// is zero, so colour-0 cells take (b - 0)/diag, colour-1 cells stay 0.
// Fused with the zeroing and with the mean projection of the level's
// right-hand side (level 0 takes it from the FP64 residual r - mean r).
// One thread per pair of cells (2ih, 2ih+1).
template <typename R>
__global__ void mg_first_kernel(Level<R> L, Bc bc, const double* __restrict__ r0, const double* mr0, const int* done) {
    pdl_wait();
    if (*done) return;
    const int ih = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.z;
    if (ih >= (L.nx >> 1) || j >= L.ny) return;
    const double m0 = r0 ? *mr0 : 0.0;
    const R m = r0 ? R(0) : R(*L.bmean);
#pragma unroll
    for (int s = 0; s < 2; ++s) {
        const int i = 2 * ih + s;
        const int q = L.nx * (j + L.ny * k) + i;
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

// One colour pass of red-black Gauss-Seidel over an even-nx level.  A
// thread owns an x-pair of cells and marches RB_K levels up their column:
// the pair is one vector load per level and stays in registers as the
// z-neighbours of the next level and the x-neighbour of the updated cell
// (the pair's other cell), so an update loads the pair above, the x
// neighbour outside the pair, the two y neighbours, b and its face
// coefficients; every neighbour is of the other colour, so the pass has no
// order.  The coefficient form is a template parameter (codes: the level's
// table, padded to 256 entries, staged in shared memory); K = 1 on levels too
// small to fill the GPU with K-level columns.

template <typename R> struct Vec2;
template <> struct Vec2<float> { using T = float2; };
template <> struct Vec2<double> { using T = double2; };

template <typename R, int CF, int RB_K>
__global__ void __launch_bounds__(RB_X * RB_Y) mg_rbgs_kernel(Level<R> L, Bc bc, int colour, const int* done) {
    pdl_wait();
    __shared__ R stab[CF == CF_CODES ? 256 : 1];
    if (*done) return;
    if (CF == CF_CODES) {
        for (int q = tid(); q < 256; q += nthreads()) stab[q] = L.c.tab[q];
        __syncthreads();
    }
    using V2 = typename Vec2<R>::T;
    const int ih = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k0 = blockIdx.z * RB_K;
    const int nx = L.nx, ny = L.ny, nz = L.nz, pl = nx * ny;
    if (ih >= (nx >> 1) || j >= ny) return;
    const int i0 = 2 * ih, row0 = i0 + nx * j;
    // in-plane neighbours outside the pair (-1 / 0: the Neumann mirror, the cell itself)
    const int xl = i0 > 0 ? row0 - 1 : (bc.x == 0 ? row0 + nx - 1 : -1);
    const int xr = i0 + 2 < nx ? row0 + 2 : (bc.x == 0 ? row0 + 2 - nx : -1);
    const int dym = j > 0 ? -nx : (bc.y == 0 ? (ny - 1) * nx : 0);
    const int dyp = j < ny - 1 ? nx : (bc.y == 0 ? -(ny - 1) * nx : 0);
    const R* __restrict__ f = L.phi;
    // the coefficient codes / values and b through restrict pointers: no store
    // of this kernel (phi's colour) touches them, so the loads of the levels
    // ahead need not wait for the stores of the levels before (the byte codes
    // could alias phi as far as the compiler knows)
    const unsigned char* __restrict__ ckx = L.c.kx;
    const unsigned char* __restrict__ cky = L.c.ky;
    const unsigned char* __restrict__ ckz = L.c.kz;
    const R* __restrict__ ccx = L.c.cx;
    const R* __restrict__ ccy = L.c.cy;
    const R* __restrict__ ccz = L.c.cz;
    const R* __restrict__ bb = L.b;
    // phi through the non-coherent path as well: a colour pass reads only the
    // other colour's cells and the cells this thread itself writes (before it
    // writes them), so no value read here changes during the pass
    auto pair_at = [&](int k) { return __ldg(reinterpret_cast<const V2*>(f + (size_t)k * pl + row0)); };
    V2 pc = pair_at(k0);
    V2 pm = k0 > 0 ? pair_at(k0 - 1) : (bc.z == 0 ? pair_at(nz - 1) : pc);
#pragma unroll
    for (int kk = 0; kk < RB_K; ++kk) {
        const int k = k0 + kk;
        if (k >= nz) break;
        const V2 pp = k + 1 < nz ? pair_at(k + 1) : (bc.z == 0 ? pair_at(0) : pc);
        const int a = (j + k + colour) & 1;   // the pair's cell of this colour
        const int q = k * pl + row0 + a;
        const R c = a ? pc.y : pc.x;
        const R nxm = a ? pc.x : (xl >= 0 ? __ldg(f + k * pl + xl) : c);
        const R nxp = a ? (xr >= 0 ? __ldg(f + k * pl + xr) : c) : pc.y;
        const R nym = dym ? __ldg(f + q + dym) : c;
        const R nyp = dyp ? __ldg(f + q + dyp) : c;
        const R nzm = a ? pm.y : pm.x, nzp = a ? pp.y : pp.x;
        R fxp = R(0), fxm = R(0), fyp = R(0), fym = R(0), fzp = R(0), fzm = R(0);
        if (CF != CF_CONST) {
            const int fx = q + j + ny * k, fy = q + nx * k;   // (nx+1)(j + ny k) + i, nx(j + (ny+1) k) + i
            fxm = face_coef<R, CF>(ccx, ckx, stab, fx);
            fxp = face_coef<R, CF>(ccx, ckx, stab, fx + 1);
            fym = face_coef<R, CF>(ccy, cky, stab, fy);
            fyp = face_coef<R, CF>(ccy, cky, stab, fy + nx);
            fzm = face_coef<R, CF>(ccz, ckz, stab, q);
            fzp = face_coef<R, CF>(ccz, ckz, stab, q + pl);
        }
        R v;
        if (gs_vals<R, CF>(nxp, nxm, nyp, nym, nzp, nzm, fxp, fxm, fyp, fym, fzp, fzm, __ldg(bb + q), L.ix2, L.iy2, L.iz2, &v))
            L.phi[q] = v;
        pm = pc;
        pc = pp;
    }
}

// r = b - A phi on a level (_compute_residual!, src/Multigrid.jl:281-285):
// one thread per cell, a 3-D grid; the arithmetic of aphi.
template <typename R, int CF>
__global__ void __launch_bounds__(RB_X * RB_Y) mg_residual_kernel(Level<R> F, Bc bc, const int* done) {
    pdl_wait();
    __shared__ R stab[CF == CF_CODES ? 256 : 1];
    if (*done) return;
    if (CF == CF_CODES) {
        for (int q = tid(); q < 256; q += nthreads()) stab[q] = F.c.tab[q];
        __syncthreads();
    }
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.z;
    const int nx = F.nx, ny = F.ny, nz = F.nz, pl = nx * ny;
    if (i >= nx || j >= ny) return;
    const int q = i + nx * (j + ny * k);
    const Nbr n = nbr_of(q, i, j, k, nx, ny, nz, pl, bc);
    const R* __restrict__ f = F.phi;
    const R c = f[q];
    R a;
    if (CF == CF_CONST) {
        a = (f[n.xp] - R(2) * c + f[n.xm]) * F.ix2 + (f[n.yp] - R(2) * c + f[n.ym]) * F.iy2 +
            (f[n.zp] - R(2) * c + f[n.zm]) * F.iz2;
    } else {
        const int fx = q + j + ny * k, fy = q + nx * k;
        const R fxm = face_coef<R, CF>(F.c.cx, F.c.kx, stab, fx), fxp = face_coef<R, CF>(F.c.cx, F.c.kx, stab, fx + 1);
        const R fym = face_coef<R, CF>(F.c.cy, F.c.ky, stab, fy), fyp = face_coef<R, CF>(F.c.cy, F.c.ky, stab, fy + nx);
        const R fzm = face_coef<R, CF>(F.c.cz, F.c.kz, stab, q), fzp = face_coef<R, CF>(F.c.cz, F.c.kz, stab, q + pl);
        a = (fxp * (f[n.xp] - c) - fxm * (c - f[n.xm])) * F.ix2 + (fyp * (f[n.yp] - c) - fym * (c - f[n.ym])) * F.iy2 +
            (fzp * (f[n.zp] - c) - fzm * (c - f[n.zm])) * F.iz2;
    }
    F.r[q] = F.b[q] - a;
}

// Coarse b = mean of the eight fine residuals (src/Multigrid.jl:380-406),
// summed in the reference's order; one thread per coarse cell on a 3-D
// grid.  The last block stores the coarse mean that the coarse level
// subtracts before use.
template <typename R>
__global__ void mg_restrict_kernel(Level<R> F, Level<R> Cl, double* part, unsigned* counter, const int* done) {
    pdl_wait();
    if (*done) return;
    const int I = blockIdx.x * blockDim.x + threadIdx.x, J = blockIdx.y * blockDim.y + threadIdx.y, K = blockIdx.z;
    double v[1] = {0.0};
    if (I < Cl.nx && J < Cl.ny) {
        const int sy = F.nx, sz = F.nx * F.ny;
        const R* r = F.r + (2 * I) + sy * (2 * J) + sz * (2 * K);
        R s = r[0];
        s += r[1];
        s += r[sy];
        s += r[sy + 1];
        s += r[sz];
        s += r[sz + 1];
        s += r[sz + sy];
        s += r[sz + sy + 1];
        const R bcv = s * R(0.125);
        Cl.b[Cl.nx * (J + Cl.ny * K) + I] = bcv;
        v[0] = double(bcv);
    }
    double tot[1];
    if (reduce_last<1>(v, part, counter, tot) && tid() == 0) *Cl.bmean = tot[0] / double(Cl.n);
}

// phi_fine += trilinear (3/4, 1/4) interpolation of phi_coarse
// (src/Multigrid.jl:412-455), the eight terms in the reference's order.
template <typename R>
__global__ void mg_prolong_kernel(Level<R> F, Level<R> Cl, Bc bc, const int* done) {
    pdl_wait();
    if (*done) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.z;
    if (i >= F.nx || j >= F.ny) return;
    const int Ih = i >> 1, Jh = j >> 1, Kh = k >> 1;
    const int Ix = (i & 1) ? wp(Ih, Cl.nx, bc.x) : wm(Ih, Cl.nx, bc.x);
    const int Jy = (j & 1) ? wp(Jh, Cl.ny, bc.y) : wm(Jh, Cl.ny, bc.y);
    const int Kz = (k & 1) ? wp(Kh, Cl.nz, bc.z) : wm(Kh, Cl.nz, bc.z);
    const R n_ = R(3) / R(4), f_ = R(1) / R(4);
    const int sy = Cl.nx, sz = Cl.nx * Cl.ny;
    const R* P = Cl.phi;
    R acc = R(0);
    acc += (n_ * n_ * n_) * P[Ih + Jh * sy + Kh * sz];
    acc += (f_ * n_ * n_) * P[Ix + Jh * sy + Kh * sz];
    acc += (n_ * f_ * n_) * P[Ih + Jy * sy + Kh * sz];
    acc += (f_ * f_ * n_) * P[Ix + Jy * sy + Kh * sz];
    acc += (n_ * n_ * f_) * P[Ih + Jh * sy + Kz * sz];
    acc += (f_ * n_ * f_) * P[Ix + Jh * sy + Kz * sz];
    acc += (n_ * f_ * f_) * P[Ih + Jy * sy + Kz * sz];
    acc += (f_ * f_ * f_) * P[Ix + Jy * sy + Kz * sz];
    const int q = F.nx * (j + F.ny * k) + i;
    F.phi[q] += acc;
}

// The coarsest level: phi = 0, b -= mean, then `sweeps` RB-GS sweeps, all in
// one block (_solve_coarsest!, src/Multigrid.jl:681-685).  Threads own
// (x, y) columns (and a share of the column's levels when the plane has
// fewer columns than threads), so the in-plane neighbour offsets are
// computed once per column.  The colour passes update in place, which is
// the reference's halo-copy semantics whenever no periodic axis has an odd
// length; otherwise (inplace = 0) each pass reads buffer A and writes B,
// the other colour copied, so every update sees the values from before the
// pass.  One barrier per pass.  phi, b and the coefficients are staged in
// shared memory when they fit.
// With `mat` (set-up, staged only) block j runs the same sweeps on the unit
// right-hand side e_j and stores the result as column j of the n x n
// row-major matrix of the whole coarsest solve (see mg_coarse_matvec_kernel).
template <typename R>
__global__ void __launch_bounds__(COARSE_THREADS) mg_coarsest_kernel(Level<R> L, R* spare, Bc bc, int sweeps,
                                                                    int staged, int inplace,
                                                                    const double* __restrict__ r0, const double* mr0,
                                                                    const int* done, R* mat) {
    pdl_wait();
    if (*done) return;
    const int unit = mat ? (int)blockIdx.x : -1;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int nx = L.nx, ny = L.ny, nz = L.nz, n = L.n;
    const int ncx = (nx + 1) * ny * nz, ncy = nx * (ny + 1) * nz, ncz = nx * ny * (nz + 1);
    const int nt = blockDim.x, t = threadIdx.x;
    R* A = L.phi;
    R* B = spare;
    R* bb = L.b;
    const R *cx = nullptr, *cy = nullptr, *cz = nullptr;
    const bool var = L.c.var();
    if (staged) {
        R* base = reinterpret_cast<R*>(smem_raw);
        A = base;
        B = base + n;
        bb = base + 2 * n;
        if (var) {
            R* c = base + 3 * n;
            for (int q = t; q < ncx; q += nt) c[q] = L.c.x(q);
            for (int q = t; q < ncy; q += nt) c[ncx + q] = L.c.y(q);
            for (int q = t; q < ncz; q += nt) c[ncx + ncy + q] = L.c.z(q);
            cx = c;
            cy = c + ncx;
            cz = c + ncx + ncy;
        }
    }
    const double m0 = (r0 && unit < 0) ? *mr0 : 0.0;
    const R m = (r0 || unit >= 0) ? R(0) : R(*L.bmean);
    for (int q = t; q < n; q += nt) {
        bb[q] = unit >= 0 ? R(q == unit ? 1 : 0) : (r0 ? R(r0[q] - m0) : L.b[q] - m);
        A[q] = R(0);
    }
    __syncthreads();
    const int ncol = nx * ny;
    int col0, cstep, kq, kparts;
    if (ncol >= nt) {
        col0 = t; cstep = nt; kq = 0; kparts = 1;
    } else {
        kparts = nt / ncol;
        col0 = t % ncol; cstep = ncol; kq = t / ncol;
        if (kq >= kparts) col0 = ncol;          // idle thread
    }
    const R ix2 = L.ix2, iy2 = L.iy2, iz2 = L.iz2;
    const R cdiag = -R(2) * (ix2 + iy2 + iz2);
    const int pl = ncol;
    for (int sw = 0; sw < sweeps; ++sw)
        for (int colour = 0; colour < 2; ++colour) {
            for (int col = col0; col < ncol; col += cstep) {
                const int i = col % nx, j = col / nx;
                const int oxm = wm(i, nx, bc.x) - i, oxp = wp(i, nx, bc.x) - i;
                const int oym = (wm(j, ny, bc.y) - j) * nx, oyp = (wp(j, ny, bc.y) - j) * nx;
                const int cxb = i + (nx + 1) * j, cyb = i + nx * j;
                for (int k = kq; k < nz; k += kparts) {
                    const int q = col + pl * k;
                    if (((i + j + k) & 1) != colour) {
                        if (!inplace) B[q] = A[q];
                        continue;
                    }
                    const int zm = col + pl * wm(k, nz, bc.z), zp = col + pl * wp(k, nz, bc.z);
                    R v = A[q];
                    R off, diag;
                    bool upd = true;
                    if (!var) {
                        diag = cdiag;
                        off = (A[q + oxp] + A[q + oxm]) * ix2 + (A[q + oyp] + A[q + oym]) * iy2 + (A[zp] + A[zm]) * iz2;
                    } else {
                        const int ax = cxb + (nx + 1) * ny * k, ay = cyb + nx * (ny + 1) * k;
                        R fxp, fxm, fyp, fym, fzp, fzm;
                        if (staged) {
                            fxp = cx[ax + 1]; fxm = cx[ax];
                            fyp = cy[ay + nx]; fym = cy[ay];
                            fzp = cz[q + pl]; fzm = cz[q];
                        } else {
                            fxp = L.c.x(ax + 1); fxm = L.c.x(ax);
                            fyp = L.c.y(ay + nx); fym = L.c.y(ay);
                            fzp = L.c.z(q + pl); fzm = L.c.z(q);
                        }
                        diag = -((fxp + fxm) * ix2 + (fyp + fym) * iy2 + (fzp + fzm) * iz2);
                        upd = !(fabs(diag) < Eps<R>::v());
                        off = (fxp * A[q + oxp] + fxm * A[q + oxm]) * ix2 + (fyp * A[q + oyp] + fym * A[q + oym]) * iy2 +
                              (fzp * A[zp] + fzm * A[zm]) * iz2;
                    }
                    if (upd) v = (bb[q] - off) / diag;
                    if (inplace) A[q] = v; else B[q] = v;
                }
            }
            __syncthreads();
            if (!inplace) {
                R* tmp = A;
                A = B;
                B = tmp;
            }
        }
    if (unit >= 0) {
        for (int q = t; q < n; q += nt) mat[(size_t)q * n + unit] = A[q];
    } else if (A != L.phi) {
        for (int q = t; q < n; q += nt) L.phi[q] = A[q];
    }
}

// The coarsest solve as one dense product phi = M (b - mean b), M the n x n
// matrix of the sweeps above (a linear map of the right-hand side, built
// once per coefficient field): the same result up to the order of the sums,
// with the n^2 values read from L2 by all SMs instead of 2 * sweeps
// dependent passes on one.  One warp per row, FP64 accumulation, fixed order.
template <typename R>
__global__ void mg_coarse_matvec_kernel(Level<R> L, const R* __restrict__ mat, const double* __restrict__ r0,
                                        const double* mr0, const int* done) {
    pdl_wait();
    if (*done) return;
    const int n = L.n;
    const int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (row >= n) return;
    const double m0 = r0 ? *mr0 : 0.0;
    const R m = r0 ? R(0) : R(*L.bmean);
    const R* Mr = mat + (size_t)row * n;
    double acc = 0.0;
    for (int j = lane; j < n; j += 32) {
        const R bj = r0 ? R(r0[j] - m0) : L.b[j] - m;
        acc += double(Mr[j]) * double(bj);
    }
    acc = warp_sum(acc);
    if (lane == 0) L.phi[row] = R(acc);
}

// The coarsest level when its columns are short (nz <= COL_NZ), fit one
// block (nx ny <= 1024 threads) and no periodic axis has an odd length: one
// thread per (x, y) column keeps the column's phi and b in registers, so the
// vertical neighbours never leave the thread; phi is mirrored in shared
// memory for the lateral neighbours, which are always of the other colour.
// The same sweeps and arithmetic as mg_coarsest_kernel, in place.
constexpr int COL_NZ = 8;
template <typename R, int MAXT>
__global__ void __launch_bounds__(MAXT) mg_coarsest_col_kernel(Level<R> L, Bc bc, int sweeps,
                                                                        const double* __restrict__ r0,
                                                                        const double* mr0, const int* done) {
    pdl_wait();
    if (*done) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int nx = L.nx, ny = L.ny, nz = L.nz, n = L.n, ncol = nx * ny;
    const int ncx = (nx + 1) * ny * nz, ncy = nx * (ny + 1) * nz, ncz = nx * ny * (nz + 1);
    const int nt = blockDim.x, t = threadIdx.x;
    const bool var = L.c.var();
    R* A = reinterpret_cast<R*>(smem_raw);
    R* bv = A + n;
    R* cx = bv + n;
    R* cy = cx + ncx;
    R* cz = cy + ncy;
    if (var) {
        for (int q = t; q < ncx; q += nt) cx[q] = L.c.x(q);
        for (int q = t; q < ncy; q += nt) cy[q] = L.c.y(q);
        for (int q = t; q < ncz; q += nt) cz[q] = L.c.z(q);
    }
    for (int q = t; q < n; q += nt) A[q] = R(0);
    const bool act = t < ncol;
    const int col = act ? t : 0;
    const int i = col % nx, j = col / nx;
    const double m0 = r0 ? *mr0 : 0.0;
    const R m = r0 ? R(0) : R(*L.bmean);
    for (int q = t; q < n; q += nt) bv[q] = r0 ? R(r0[q] - m0) : L.b[q] - m;
    R ph[COL_NZ];
#pragma unroll
    for (int k = 0; k < COL_NZ; ++k) ph[k] = R(0);
    const int oxm = wm(i, nx, bc.x) - i, oxp = wp(i, nx, bc.x) - i;
    const int oym = (wm(j, ny, bc.y) - j) * nx, oyp = (wp(j, ny, bc.y) - j) * nx;
    const int cxb = i + (nx + 1) * j, cyb = i + nx * j;
    const R ix2 = L.ix2, iy2 = L.iy2, iz2 = L.iz2;
    const R cdiag = -R(2) * (ix2 + iy2 + iz2);
    const bool zper = bc.z == 0;
    __syncthreads();
    for (int sw = 0; sw < sweeps; ++sw)
        for (int colour = 0; colour < 2; ++colour) {
            if (act) {
                R top = ph[0];
#pragma unroll
                for (int k = 1; k < COL_NZ; ++k)
                    if (k == nz - 1) top = ph[k];
#pragma unroll
                for (int k = 0; k < COL_NZ; ++k) {
                    if (k >= nz || ((i + j + k) & 1) != colour) continue;
                    const int q = col + ncol * k;
                    const R vzm = k > 0 ? ph[k > 0 ? k - 1 : 0] : (zper ? top : ph[0]);
                    const R vzp = k < nz - 1 ? ph[k + 1 < COL_NZ ? k + 1 : COL_NZ - 1] : (zper ? ph[0] : ph[k]);
                    R off, diag;
                    bool upd = true;
                    if (!var) {
                        diag = cdiag;
                        off = (A[q + oxp] + A[q + oxm]) * ix2 + (A[q + oyp] + A[q + oym]) * iy2 + (vzp + vzm) * iz2;
                    } else {
                        const int ax = cxb + (nx + 1) * ny * k, ay = cyb + nx * (ny + 1) * k;
                        const R fxp = cx[ax + 1], fxm = cx[ax], fyp = cy[ay + nx], fym = cy[ay];
                        const R fzp = cz[q + ncol], fzm = cz[q];
                        diag = -((fxp + fxm) * ix2 + (fyp + fym) * iy2 + (fzp + fzm) * iz2);
                        upd = !(fabs(diag) < Eps<R>::v());
                        off = (fxp * A[q + oxp] + fxm * A[q + oxm]) * ix2 + (fyp * A[q + oyp] + fym * A[q + oym]) * iy2 +
                              (fzp * vzp + fzm * vzm) * iz2;
                    }
                    if (upd) {
                        const R v = (bv[q] - off) / diag;
                        ph[k] = v;
                        A[q] = v;
                    }
                }
            }
            __syncthreads();
        }
    if (act)
#pragma unroll
        for (int k = 0; k < COL_NZ; ++k)
            if (k < nz) L.phi[col + ncol * k] = ph[k];
}

// level-0 right-hand side of the standalone cycles: b0 = b - mean(b), phi0 = 0
template <typename R>
__global__ void mg_load_kernel(Level<R> L, const double* __restrict__ r0, const double* mr0) {
    GRID_STRIDE(t, L.n) {
        L.b[t] = R(r0[t] - *mr0);
        L.phi[t] = R(0);
    }
}

// relative residual of the standalone cycles (_residual_norm!,
// src/Multigrid.jl:780-785): |r - mean r| / |b| from sum r and sum r^2
template <typename R>
__global__ void mg_resnorm_kernel(Level<R> L, Bc bc, PcgState* S, double* part) {
    if (S->done) return;
    double v[2] = {0.0, 0.0};
    const int nrows = L.ny * L.nz;
    for (int row = blockIdx.x * blockDim.y + threadIdx.y; row < nrows; row += gridDim.x * blockDim.y) {
        const int j = row % L.ny, k = row / L.ny;
        for (int i = threadIdx.x; i < L.nx; i += blockDim.x) {
            Idx d = make_idx(i, j, k, L.nx, L.ny, L.nz, bc);
            double rr = double(L.b[d.q] - aphi<R, R>(L.phi, d, L.c, L.ix2, L.iy2, L.iz2));
            v[0] += rr;
            v[1] += rr * rr;
        }
    }
    double tot[2];
    if (reduce_last<2>(v, part, &S->counter, tot) && tid() == 0) {
        double ss = tot[1];
        if (S->project) ss -= tot[0] * (tot[0] / S->n);
        S->iters += 1;
        S->rel = sqrt(fmax(ss, 0.0)) / S->bnorm;
        S->rnorm = S->rel;
        if (S->rel < S->tol) {
            S->status = MG_CONVERGED;
            S->done = 1;
        }
    }
}

// phi0 -> x (FP64) after the cycles; the mean is removed by shift_kernel
template <typename R>
__global__ void mg_store_kernel(Level<R> L, double* __restrict__ x) {
    GRID_STRIDE(t, L.n) x[t] = double(L.phi[t]);
}

// |b0| of the standalone cycles; a zero rhs ends before the first cycle
template <typename R>
__global__ void mg_bnorm_kernel(Level<R> L, PcgState* S, double* part) {
    double v[1] = {0.0};
    GRID_STRIDE(t, L.n) {
        double bv = double(L.b[t]);
        v[0] += bv * bv;
    }
    double tot[1];
    if (reduce_last<1>(v, part, &S->counter, tot) && tid() == 0) {
        S->bnorm = sqrt(tot[0]);
        S->iters = 0;
        S->rel = 1.0;
        S->curvature = nan("");
        if (S->bnorm == 0.0) {
            S->status = MG_ZERO_RHS;
            S->done = 3;
        } else {
            S->status = MG_MAXIT;
            S->done = 0;
        }
    }
}

#undef GRID_STRIDE

}  // namespace mgk
