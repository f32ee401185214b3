// aeo_tke.cuh -- the once-per-step commit of the Deardorff (1980) / Moeng
// (1984) prognostic-TKE closure (TKEClosure, advance_sgs!,
// src/PrognosticSGS.jl:978-1145) on the Boussinesq core's uniform grid.
//
// The step's substages read nu_t and kappa_t of the committed e in the
// sweeps' coefficient pass (tke_point).  After the step the commit runs:
//   tke_coef_kernel   K = 2 nu_t of e^n and the new N^2 (interior);
//   halo fill of K and e;
//   the flux-limited WENO-Z5 transport of e (the positivity kernels of
//   aeo_positive.cuh, accumulate = false) into tend;
//   tke_update_kernel every cell's new e (diffusion div(K grad e), the shear
//   production nu_t D with D the discrete dual of the momentum operator, the
//   buoyancy production and the sinks) into tend, its own entry only;
//   tke_copy_kernel   e = tend on the interior, then e's halos.
// FP64 arithmetic in the commit; e is stored in the working precision.
#pragma once

#include "aeo_common.cuh"

struct TkeArgs {
    double ck, ce0, ce1, cl, delta, bg;   // c_k, c_eps0, c_eps1, c_l, (dx dy dz)^(1/3), g / theta0
    double pb1, pb2;                      // (g/theta0) F / 2 of the bottom / top surface heat flux
    int exact;                            // the exact dissipation step
};

template <typename R>
struct TkePad {   // a padded field around the thread's cell (0-based interior indices)
    const R* __restrict__ p;
    Geo g;
    __device__ __forceinline__ double operator()(int i, int j, int k) const { return (double)__ldg(p + pidx(g, i, j, k)); }
};

// tke_length_scale (src/PrognosticSGS.jl:93-110): l and s = sqrt(e) / l
__device__ __forceinline__ void tke_length(const TkeArgs& t, double e, double N2, double* l, double* s) {
    const double sq = sqrt(fmax(e, 0.0)), lmax = t.delta;
    const bool stable = N2 > 0;
    const double N = sqrt(fmax(N2, 0.0));
    *l = stable ? fmin(lmax, t.cl * sq / N) : lmax;
    *s = stable ? fmax(sq / lmax, N / t.cl) : sq / lmax;
}

template <typename R>
__device__ __forceinline__ double tke_n2(const Geo& g, const TkeArgs& t, const TkePad<R>& th, int i, int j, int k) {
    const double below = 0.5 * (th(i, j, k - 1) + th(i, j, k)), above = 0.5 * (th(i, j, k) + th(i, j, k + 1));
    return t.bg * (above - below) * (1 / g.dz);
}

// K = 2 nu_t of e^n and the state's N^2 on the interior (_coefficients! then _double!)
template <typename R>
__global__ void __launch_bounds__(256) tke_coef_kernel(Geo g, TkeArgs t, const R* __restrict__ e,
                                                       const R* __restrict__ th, R* __restrict__ k2) {
    const TkePad<R> T{th, g};
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < g.nin; q += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(q % g.nx);
        const long long r = q / g.nx;
        const int j = (int)(r % g.ny), k = (int)(r / g.ny);
        const long long p = pidx(g, i, j, k);
        const double ev = (double)e[p];
        double l, s;
        tke_length(t, ev, tke_n2<R>(g, t, T, i, j, k), &l, &s);
        k2[p] = R(2 * (t.ck * l * sqrt(fmax(ev, 0.0))));
    }
}

// The share of D destined for cell (I, J, K) (0-based; a halo cell when the
// fold asks for it) from the velocity points around it (_dual_raw,
// src/PrognosticSGS.jl:589-632, flux shares :541-560): every flux nu dq / h
// of the momentum operator gives -u_p (+-flux) / h to the cells of its nu;
// points outside the interior give nothing.
template <typename R>
__device__ double tke_dual_raw(const Geo& g, const TkePad<R>& u, const TkePad<R>& v, const TkePad<R>& w, int I, int J,
                               int K) {
    const double ix2 = g.idx * g.idx, iy2 = g.idy * g.idy, iz2 = g.idz * g.idz;
    auto in = [&](int i, int j, int k) { return i >= 0 && i < g.nx && j >= 0 && j < g.ny && k >= 0 && k < g.nz; };
    // the shares of point p = (i, j, k) of field f: its flux toward +d (sign -1)
    // or from -d (sign +1), 0.25 for a cross flux
    auto sh = [&](const TkePad<R>& f, int i, int j, int k, int di, int dj, int dk, double ih2, bool plus, bool cross) {
        if (!in(i, j, k)) return 0.0;
        const double c = f(i, j, k);
        const double x = plus ? -c * (f(i + di, j + dj, k + dk) - c) * ih2 : c * (c - f(i - di, j - dj, k - dk)) * ih2;
        return cross ? 0.25 * x : x;
    };
    // u
    double d = sh(u, I, J, K, 1, 0, 0, ix2, true, false) + sh(u, I + 1, J, K, 1, 0, 0, ix2, false, false);
    d += (sh(u, I + 1, J, K, 0, 1, 0, iy2, true, true) + sh(u, I, J, K, 0, 1, 0, iy2, true, true)) +
         (sh(u, I + 1, J - 1, K, 0, 1, 0, iy2, true, true) + sh(u, I, J - 1, K, 0, 1, 0, iy2, true, true));
    d += (sh(u, I + 1, J + 1, K, 0, 1, 0, iy2, false, true) + sh(u, I, J + 1, K, 0, 1, 0, iy2, false, true)) +
         (sh(u, I + 1, J, K, 0, 1, 0, iy2, false, true) + sh(u, I, J, K, 0, 1, 0, iy2, false, true));
    d += (sh(u, I + 1, J, K, 0, 0, 1, iz2, true, true) + sh(u, I, J, K, 0, 0, 1, iz2, true, true)) +
         (sh(u, I + 1, J, K - 1, 0, 0, 1, iz2, true, true) + sh(u, I, J, K - 1, 0, 0, 1, iz2, true, true));
    d += (sh(u, I + 1, J, K + 1, 0, 0, 1, iz2, false, true) + sh(u, I, J, K + 1, 0, 0, 1, iz2, false, true)) +
         (sh(u, I + 1, J, K, 0, 0, 1, iz2, false, true) + sh(u, I, J, K, 0, 0, 1, iz2, false, true));
    // v
    d += sh(v, I, J, K, 0, 1, 0, iy2, true, false) + sh(v, I, J + 1, K, 0, 1, 0, iy2, false, false);
    d += (sh(v, I, J + 1, K, 1, 0, 0, ix2, true, true) + sh(v, I - 1, J + 1, K, 1, 0, 0, ix2, true, true)) +
         (sh(v, I, J, K, 1, 0, 0, ix2, true, true) + sh(v, I - 1, J, K, 1, 0, 0, ix2, true, true));
    d += (sh(v, I + 1, J + 1, K, 1, 0, 0, ix2, false, true) + sh(v, I, J + 1, K, 1, 0, 0, ix2, false, true)) +
         (sh(v, I + 1, J, K, 1, 0, 0, ix2, false, true) + sh(v, I, J, K, 1, 0, 0, ix2, false, true));
    d += (sh(v, I, J + 1, K, 0, 0, 1, iz2, true, true) + sh(v, I, J, K, 0, 0, 1, iz2, true, true)) +
         (sh(v, I, J + 1, K - 1, 0, 0, 1, iz2, true, true) + sh(v, I, J, K - 1, 0, 0, 1, iz2, true, true));
    d += (sh(v, I, J + 1, K + 1, 0, 0, 1, iz2, false, true) + sh(v, I, J, K + 1, 0, 0, 1, iz2, false, true)) +
         (sh(v, I, J + 1, K, 0, 0, 1, iz2, false, true) + sh(v, I, J, K, 0, 0, 1, iz2, false, true));
    // w
    d += sh(w, I, J, K, 0, 0, 1, iz2, true, false) + sh(w, I, J, K + 1, 0, 0, 1, iz2, false, false);
    d += (sh(w, I, J, K + 1, 1, 0, 0, ix2, true, true) + sh(w, I - 1, J, K + 1, 1, 0, 0, ix2, true, true)) +
         (sh(w, I, J, K, 1, 0, 0, ix2, true, true) + sh(w, I - 1, J, K, 1, 0, 0, ix2, true, true));
    d += (sh(w, I + 1, J, K + 1, 1, 0, 0, ix2, false, true) + sh(w, I, J, K + 1, 1, 0, 0, ix2, false, true)) +
         (sh(w, I + 1, J, K, 1, 0, 0, ix2, false, true) + sh(w, I, J, K, 1, 0, 0, ix2, false, true));
    d += (sh(w, I, J, K + 1, 0, 1, 0, iy2, true, true) + sh(w, I, J - 1, K + 1, 0, 1, 0, iy2, true, true)) +
         (sh(w, I, J, K, 0, 1, 0, iy2, true, true) + sh(w, I, J - 1, K, 0, 1, 0, iy2, true, true));
    d += (sh(w, I, J + 1, K + 1, 0, 1, 0, iy2, false, true) + sh(w, I, J, K + 1, 0, 1, 0, iy2, false, true)) +
         (sh(w, I, J + 1, K, 0, 1, 0, iy2, false, true) + sh(w, I, J, K, 0, 1, 0, iy2, false, true));
    return d;
}

// _fold_src (:639-640): source n (1 the cell, 2 the low halo layer -1, 3 the
// high one N) of index I when that layer is a copy of lo / hi; -2 = none
__device__ __forceinline__ int tke_fold_src(int I, int N, int lo, int hi, int n) {
    return n == 1 ? I : (n == 2 ? (lo == I ? -1 : -2) : (hi == I ? N : -2));
}

// The new e of every interior cell into tend (its own entry: the advection
// it holds is read first) (_tke_update_body, :1077-1145, with D of
// _dual_strain_body! :642-665, the diffusion _b_eddy_scalar!,
// src/FiniteVolume.jl:1280-1300, and the surface buoyancy of
// _surface_buoyancy :408-426).
template <typename R>
__global__ void __launch_bounds__(128) tke_update_kernel(Geo g, TkeArgs t, const R* __restrict__ e,
                                                         const R* __restrict__ k2, const R* __restrict__ th,
                                                         const R* __restrict__ u, const R* __restrict__ v,
                                                         const R* __restrict__ w, const double* __restrict__ dtp,
                                                         R* __restrict__ tend) {
    const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (q >= g.nin) return;
    const int i = (int)(q % g.nx);
    const long long r = q / g.nx;
    const int j = (int)(r % g.ny), k = (int)(r / g.ny);
    const TkePad<R> E{e, g}, K2{k2, g}, T{th, g}, U{u, g}, V{v, g}, W{w, g};
    const double dt = *dtp;
    // the diffusion of e with K = 2 nu_t (face means)
    const double nE = 0.5 * (K2(i, j, k) + K2(i + 1, j, k)), nW = 0.5 * (K2(i - 1, j, k) + K2(i, j, k));
    const double nN = 0.5 * (K2(i, j, k) + K2(i, j + 1, k)), nS = 0.5 * (K2(i, j - 1, k) + K2(i, j, k));
    const double nT = 0.5 * (K2(i, j, k) + K2(i, j, k + 1)), nB = 0.5 * (K2(i, j, k - 1) + K2(i, j, k));
    const double ec = E(i, j, k);
    const double fxE = nE * (E(i + 1, j, k) - ec) * g.idx, fxW = nW * (ec - E(i - 1, j, k)) * g.idx;
    const double fyN = nN * (E(i, j + 1, k) - ec) * g.idy, fyS = nS * (ec - E(i, j - 1, k)) * g.idy;
    const double fzT = nT * (E(i, j, k + 1) - ec) * g.idz, fzB = nB * (ec - E(i, j, k - 1)) * g.idz;
    const long long p = pidx(g, i, j, k);
    const double tr = (double)tend[p] + 1.0 * ((fxE - fxW) * g.idx + (fyN - fyS) * g.idy + (fzT - fzB) * g.idz);
    // D: the shares of every source the halo fold gives this cell (periodic x, y;
    // z periodic or mirrored at walls)
    const bool pz = g.bc_z == 0;
    const int loz = pz ? g.nz - 1 : 0, hiz = pz ? 0 : g.nz - 1;
    double D = 0.0;
    for (int nz = 1; nz <= 3; ++nz) {
        const int sz = tke_fold_src(k, g.nz, loz, hiz, nz);
        if (sz == -2) continue;
        for (int ny = 1; ny <= 3; ++ny) {
            const int sy = tke_fold_src(j, g.ny, g.ny - 1, 0, ny);
            if (sy == -2) continue;
            for (int nx = 1; nx <= 3; ++nx) {
                const int sx = tke_fold_src(i, g.nx, g.nx - 1, 0, nx);
                if (sx == -2) continue;
                D += tke_dual_raw<R>(g, U, V, W, sx, sy, sz);
            }
        }
    }
    // the update
    const double N2 = tke_n2<R>(g, t, T, i, j, k);
    double l, s;
    tke_length(t, ec, N2, &l, &s);
    const double ce = (t.ce0 + t.ce1 * l / t.delta) * 1.0;
    const double nu = K2(i, j, k) / 2;
    const double Ps = nu * D + 0.0;
    const double kv = (1 + 2 * l / t.delta) * nu;
    const double Psf = (k == 0 ? t.pb1 : 0.0) + (k == g.nz - 1 ? t.pb2 : 0.0);
    const double src = Ps + (N2 < 0 ? -kv * N2 : 0.0) + fmax(Psf, 0.0);
    const double rb = ((N2 > 0) && (s > 0) ? (1 + 2 * l / t.delta) * t.ck * N2 / s : 0.0) +
                      (Psf < 0 ? -Psf / fmax(ec, 2.2250738585072014e-308) : 0.0);
    double es = ec + dt * (tr + src);
    if (es < 0) es = 0.0;
    double en = es / (1 + dt * (ce * s + rb));
    if (t.exact && l > 0 && es > 0) {
        const double a = 1 / (1 / sqrt(es) + ce * dt / (2 * l));
        en = (a * a) / (1 + dt * rb);
    }
    tend[p] = R(en);
}

// e = tend on the interior
template <typename R>
__global__ void __launch_bounds__(256) tke_copy_kernel(Geo g, const R* __restrict__ src, R* __restrict__ e) {
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < g.nin; q += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(q % g.nx);
        const long long r = q / g.nx;
        const int j = (int)(r % g.ny), k = (int)(r / g.ny);
        const long long p = pidx(g, i, j, k);
        e[p] = src[p];
    }
}
