// aeo_positive.cuh -- positivity-preserving scalar advection
// (advect_positive!, src/AdvectionSchemes.jl:1100-1160, the limiter
// apply_positivity_limiter! :998-1098).
//
// -div(u phi) with the face fluxes limited so that a forward-Euler update
// with the same dt keeps a non-negative phi non-negative (under the
// first-order CFL condition):
//   F  = vel * face value, WENO-JS5 or WENO-Z5 reconstruction upwinded on the
//        face velocity (_reconstructed_fluxes! :868-892),
//   L  = vel * the upwind cell value (_upwind_fluxes! :899-909),
//   R  = min(1, Q / P) per cell, P = dt * the antidiffusive outflow
//        sum(max(+-(F - L), 0) / h), Q = max(phi - dt div L, 0), 1 where
//        nothing flows out (_b_limit_ratio! :1015-1043),
//   F' = L + c (F - L) with c the donor's R, R wrapped periodically one layer
//        beyond the interior (_wrap_one_layer! :951-958, the default without
//        boundary conditions; at walls the face velocity and flux are zero),
//   tend (+)= -div F' (_b_flux_div! :911-926).
// Three kernels, because each R needs the fluxes of its six faces and each
// limited flux the R of its donor: the face fluxes F (WENO, each face once);
// the ratios; the limited fluxes and their divergence (each face's limited
// flux evaluated by both of its cells, from the same values, so the two see
// the same flux and the update conserves phi).
//
// Arrays: u, v, w, phi, tend in the reference storage layout (halos hx, hy,
// hz >= 3, filled), x fastest; F on the interior faces ((nx+1) ny nz,
// nx (ny+1) nz, nx ny (nz+1)); R on the interior cells.
#pragma once

#include "aeo_common.cuh"

struct PosGeo {
    int nx, ny, nz, hx, hy, hz;
    long long sx, sy, sz;   // storage strides: 1, NX, NX*NY
    double idx, idy, idz;
};

__device__ __forceinline__ long long pos_sidx(const PosGeo& g, int i, int j, int k) {
    return (long long)(i + g.hx) + g.sy * (j + g.hy) + g.sz * (k + g.hz);
}

// the 5-point left-biased reconstructions (src/AdvectionSchemes.jl:240-255,
// :319-333): the three candidate stencils, the indicators a1^2 + (13/3) a2^2
// of their half first and second differences, and the JS or Z weights
template <typename R>
__device__ __forceinline__ R pos_beta(R a1, R a2) {
    return a1 * a1 + (R(13) / R(3)) * (a2 * a2);
}
// the weight divisions: IEEE in FP64; in FP32 the two-instruction
// reciprocal-multiply (within 2 ulp; the denominators are normal numbers)
__device__ __forceinline__ double pos_div(double a, double b) { return a / b; }
__device__ __forceinline__ float pos_div(float a, float b) { return __fdividef(a, b); }

template <typename R, int S>
__device__ __forceinline__ R pos_recon(R v1, R v2, R v3, R v4, R v5) {
    const R sixth = R(1) / R(6), half = R(0.5);
    const R q0 = (R(2) * v1 - R(7) * v2 + R(11) * v3) * sixth;
    const R q1 = (-v2 + R(5) * v3 + R(2) * v4) * sixth;
    const R q2 = (R(2) * v3 + R(5) * v4 - v5) * sixth;
    const R b0 = pos_beta<R>((v1 - R(4) * v2 + R(3) * v3) * half, (v1 - R(2) * v2 + v3) * half);
    const R b1 = pos_beta<R>((v4 - v2) * half, (v2 - R(2) * v3 + v4) * half);
    const R b2 = pos_beta<R>((-R(3) * v3 + R(4) * v4 - v5) * half, (v3 - R(2) * v4 + v5) * half);
    R a0, a1, a2;
    if (S == AEO_ADV_WENO_JS5) {
        const R e = R(1e-6);
        a0 = pos_div(R(0.1), (b0 + e) * (b0 + e));
        a1 = pos_div(R(0.6), (b1 + e) * (b1 + e));
        a2 = pos_div(R(0.3), (b2 + e) * (b2 + e));
    } else {   // p = 2, eps = eps(T)^2
        const R eps = sizeof(R) == 8 ? R(4.930380657631324e-32) : R(1.4210854715202004e-14);
        const R tau = fabs(b0 - b2);
        const R t0 = pos_div(tau, b0 + eps), t1 = pos_div(tau, b1 + eps), t2 = pos_div(tau, b2 + eps);
        a0 = R(0.1) * (R(1) + t0 * t0);
        a1 = R(0.6) * (R(1) + t1 * t1);
        a2 = R(0.3) * (R(1) + t2 * t2);
    }
    return pos_div(a0 * q0 + a1 * q1 + a2 * q2, a0 + a1 + a2);
}

// the face value between cells c and c+1 (c at p, the axis stride s): the
// left-biased stencil for vel >= 0, the mirrored one otherwise
// (src/AdvectionSchemes.jl:623-666)
template <typename R, int S>
__device__ __forceinline__ R pos_face(const R* __restrict__ f, long long p, long long s, R vel) {
    const R m2 = f[p - 2 * s], m1 = f[p - s], c0 = f[p], p1 = f[p + s], p2 = f[p + 2 * s], p3 = f[p + 3 * s];
    const bool up = vel >= R(0);
    return pos_recon<R, S>(up ? m2 : p3, up ? m1 : p2, up ? c0 : p1, up ? p1 : c0, up ? p2 : m1);
}

// F on the interior faces: thread (i, j, k) over (nx+1) x (ny+1) x (nz+1)
// computes the x face i of row (j, k), the y face j of column (i, k) and the
// z face k of column (i, j) where they exist
template <typename R, int S>
__global__ void __launch_bounds__(256) pos_flux_kernel(PosGeo g, const R* __restrict__ u, const R* __restrict__ v,
                                                       const R* __restrict__ w, const R* __restrict__ f,
                                                       R* __restrict__ Fx, R* __restrict__ Fy, R* __restrict__ Fz) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, k = blockIdx.z;
    if (i > g.nx) return;
    const long long p = pos_sidx(g, i, j, k);
    if (j < g.ny && k < g.nz) {
        const R vel = u[p];
        Fx[(long long)(g.nx + 1) * (j + (long long)g.ny * k) + i] = vel * pos_face<R, S>(f, p - 1, 1, vel);
    }
    if (i < g.nx && k < g.nz) {
        const R vel = v[p];
        Fy[(long long)g.nx * (j + (long long)(g.ny + 1) * k) + i] = vel * pos_face<R, S>(f, p - g.sy, g.sy, vel);
    }
    if (i < g.nx && j < g.ny) {
        const R vel = w[p];
        Fz[(long long)g.nx * (j + (long long)g.ny * k) + i] = vel * pos_face<R, S>(f, p - g.sz, g.sz, vel);
    }
}

// the first-order upwind flux of the face between storage points a (low) and b
template <typename R>
__device__ __forceinline__ R pos_lo(const R* __restrict__ vel, const R* __restrict__ f, long long a, long long b) {
    const R v = vel[b];
    return v * (v >= R(0) ? f[a] : f[b]);
}

// the six faces of interior cell (i, j, k): F and L, east/west, north/south, top/bottom
template <typename R>
struct PosFaces {
    R fe, fw, fn, fs, ft, fb, le, lw, ln, ls, lt, lb;
};
template <typename R>
__device__ __forceinline__ PosFaces<R> pos_faces(const PosGeo& g, const R* __restrict__ u, const R* __restrict__ v,
                                                 const R* __restrict__ w, const R* __restrict__ f,
                                                 const R* __restrict__ Fx, const R* __restrict__ Fy,
                                                 const R* __restrict__ Fz, int i, int j, int k, long long p) {
    PosFaces<R> a;
    const long long xr = (long long)(g.nx + 1) * (j + (long long)g.ny * k) + i;
    const long long yr = (long long)g.nx * (j + (long long)(g.ny + 1) * k) + i;
    const long long zr = (long long)g.nx * (j + (long long)g.ny * k) + i;
    a.fw = Fx[xr];
    a.fe = Fx[xr + 1];
    a.fs = Fy[yr];
    a.fn = Fy[yr + g.nx];
    a.fb = Fz[zr];
    a.ft = Fz[zr + (long long)g.nx * g.ny];
    a.lw = pos_lo<R>(u, f, p - 1, p);
    a.le = pos_lo<R>(u, f, p, p + 1);
    a.ls = pos_lo<R>(v, f, p - g.sy, p);
    a.ln = pos_lo<R>(v, f, p, p + g.sy);
    a.lb = pos_lo<R>(w, f, p - g.sz, p);
    a.lt = pos_lo<R>(w, f, p, p + g.sz);
    return a;
}

template <typename R>
__global__ void __launch_bounds__(256) pos_ratio_kernel(PosGeo g, const R* __restrict__ u, const R* __restrict__ v,
                                                        const R* __restrict__ w, const R* __restrict__ f,
                                                        const R* __restrict__ Fx, const R* __restrict__ Fy,
                                                        const R* __restrict__ Fz, const double* __restrict__ dtp,
                                                        R* __restrict__ Rr) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, k = blockIdx.z;
    if (i >= g.nx) return;
    const long long p = pos_sidx(g, i, j, k);
    const PosFaces<R> a = pos_faces<R>(g, u, v, w, f, Fx, Fy, Fz, i, j, k, p);
    const R dt = R(*dtp), z = R(0), idx = R(g.idx), idy = R(g.idy), idz = R(g.idz);
    const R axe = a.fe - a.le, axw = a.fw - a.lw, ayn = a.fn - a.ln, ays = a.fs - a.ls, azt = a.ft - a.lt,
            azb = a.fb - a.lb;
    const R Pm = dt * ((fmax(axe, z) + fmax(-axw, z)) * idx + (fmax(ayn, z) + fmax(-ays, z)) * idy +
                       (fmax(azt, z) + fmax(-azb, z)) * idz);
    const R div_lo = (a.le - a.lw) * idx + (a.ln - a.ls) * idy + (a.lt - a.lb) * idz;
    const R Q = fmax(f[p] - dt * div_lo, z);
    Rr[(long long)g.nx * (j + (long long)g.ny * k) + i] = Pm > z ? fmin(R(1), Q / Pm) : R(1);
}

template <typename R>
__device__ __forceinline__ R pos_ratio_at(const PosGeo& g, const R* __restrict__ Rr, int i, int j, int k) {
    i = i < 0 ? i + g.nx : (i >= g.nx ? i - g.nx : i);
    j = j < 0 ? j + g.ny : (j >= g.ny ? j - g.ny : j);
    k = k < 0 ? k + g.nz : (k >= g.nz ? k - g.nz : k);
    return Rr[(long long)g.nx * (j + (long long)g.ny * k) + i];
}

// the limited flux of a face: lo + c (F - lo), c the ratio of the donor
// (the low cell where the antidiffusive flux is >= 0)
template <typename R>
__device__ __forceinline__ R pos_limited(R F, R lo, R r_low, R r_high) {
    const R a = F - lo;
    const R c = a >= R(0) ? r_low : r_high;
    return lo + c * a;
}

template <typename R>
__global__ void __launch_bounds__(256) pos_apply_kernel(PosGeo g, const R* __restrict__ u, const R* __restrict__ v,
                                                        const R* __restrict__ w, const R* __restrict__ f,
                                                        const R* __restrict__ Fx, const R* __restrict__ Fy,
                                                        const R* __restrict__ Fz, const R* __restrict__ Rr,
                                                        R* __restrict__ tend, int accumulate) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, k = blockIdx.z;
    if (i >= g.nx) return;
    const long long p = pos_sidx(g, i, j, k);
    const PosFaces<R> a = pos_faces<R>(g, u, v, w, f, Fx, Fy, Fz, i, j, k, p);
    const R rc = Rr[(long long)g.nx * (j + (long long)g.ny * k) + i];
    const R fe = pos_limited<R>(a.fe, a.le, rc, pos_ratio_at<R>(g, Rr, i + 1, j, k));
    const R fw = pos_limited<R>(a.fw, a.lw, pos_ratio_at<R>(g, Rr, i - 1, j, k), rc);
    const R fn = pos_limited<R>(a.fn, a.ln, rc, pos_ratio_at<R>(g, Rr, i, j + 1, k));
    const R fs = pos_limited<R>(a.fs, a.ls, pos_ratio_at<R>(g, Rr, i, j - 1, k), rc);
    const R ft = pos_limited<R>(a.ft, a.lt, rc, pos_ratio_at<R>(g, Rr, i, j, k + 1));
    const R fb = pos_limited<R>(a.fb, a.lb, pos_ratio_at<R>(g, Rr, i, j, k - 1), rc);
    const R d = (fe - fw) * R(g.idx) + (fn - fs) * R(g.idy) + (ft - fb) * R(g.idz);
    tend[p] = accumulate ? tend[p] - d : -d;
}
