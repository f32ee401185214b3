// aeo_adapt.cuh -- CFL diagnostics, the adaptive time-step pick and the
// post-step guard, all on the device so an adaptive step is one graph.
//
// Reference: cfl_diagnostics / adaptive_dt (src/TimeIntegration.jl:127-454),
// the per-cell advective rate _adv_rate_at (:178-185), the Brunt-Vaisala
// limit _brunt_vaisala (:209-226, buoyancy_frequency_squared
// src/TurbulenceStability.jl:129-133) and the fused step guard _guard_at /
// step_guard (src/TimeIntegration.jl:663-721).
#pragma once

#include "aeo_sweep.cuh"
#include "aeo_dynamic.cuh"

// Scalars of the step that live in device memory (read by the stage kernels).
struct StepScalars {
    double dt;        // the dt of the step being taken
    double dt_prev;   // the last accepted dt (0: none)
    double one;       // 1.0: the dt of a stand-alone projection
    int limiter;      // 0 advective, 1 diffusive, 2 buoyancy, 3 Coriolis, 4 sgs, 5 growth, 6 dt_min, 7 dt_max
    int pad;
    double rate, nut_max, N;   // the pick's diagnostics
    double pos_dt;             // the dt of the positivity-limited advection (aeo_advect_positive)
};

struct CflParams {
    double c_adv, c_diff, c_buoy, c_cor, dt_min, dt_max, growth;
    double nu, pr_t, fcor, gacc, theta0, dz_min;
    double th_off;   // the stored offset of theta (plane means are of theta - th_off)
    int sgs, buoy, anel;
};

// Per level: max advective rate, max nut (SGS), sum of theta, max kappa_t
// (the AMD closure's own; 0 otherwise).
template <typename R, bool UNI, bool SGS>
__global__ void __launch_bounds__(256) cfl_levels_kernel(Geo g, const R* __restrict__ u, const R* __restrict__ v,
                                                         const R* __restrict__ w, const R* __restrict__ th, R c_s,
                                                         R pr_t, const double* __restrict__ cs2, double dd2,
                                                         double* __restrict__ part, const R* __restrict__ cs2f = nullptr) {
    __shared__ double rmax[256], nmax[256], tsum[256], kmax[256];
    const int k = blockIdx.x;
    const double iz = UNI ? g.idz : lvl(g.idzc, k);
    double r = 0.0, nm = 0.0, ts = 0.0, km = 0.0;
    bool nanr = false;
    for (int e = threadIdx.x; e < g.nx * g.ny; e += blockDim.x) {
        const int i = e % g.nx, j = e / g.nx;
        const long long q = pidx(g, i, j, k);
        double au = fmax(fabs((double)u[q]), fabs((double)u[q + 1]));
        double av = fmax(fabs((double)v[q]), fabs((double)v[q + g.sy]));
        double aw = fmax(fabs((double)w[q]), fabs((double)w[q + g.sz]));
        double rate = au * g.idx + av * g.idy + aw * iz;
        nanr = nanr || isnan(rate);
        r = fmax(r, rate);
        if (SGS) {
            Nb<R> U{u + q, g.sy, g.sz}, V{v + q, g.sy, g.sz}, W{w + q, g.sy, g.sz};
            if (g.sgs_model == 4) {   // dynamic Smagorinsky: cs2(k) Delta^2 |S|
                nm = fmax(nm, (double)(R(dyn_cs2_cell(g, cs2, cs2f, i, j, k) * dd2) *
                                       strain_at<R, UNI>(Met<R, UNI>(g), g, k, U, V, W, (R*)nullptr)));
            } else if (g.sgs_model == 3) {
                Nb<R> T{th + q, g.sy, g.sz};
                const Met<R, UNI> m(g);
                const NuKappa<R> nk = amd_point<R, UNI>(m, g, k, c_s, m.lv(LV_BGC, k), pr_t, U, V, W, T);
                nm = fmax(nm, (double)nk.nu);
                km = fmax(km, (double)nk.ka);
            } else if (g.sgs_model == 7) {   // the TKE closure's nu_t and kappa_t
                const NuKappa<R> nk = tke_point<R>(g, i, j, k, th[q - g.sz], th[q], th[q + g.sz]);
                nm = fmax(nm, (double)nk.nu);
                km = fmax(km, (double)nk.ka);
            } else {
                nm = fmax(nm, (double)smag_point<R, UNI>(Met<R, UNI>(g), g, k, c_s, U, V, W));
            }
        }
        ts += (double)th[q];
    }
    rmax[threadIdx.x] = nanr ? NAN : r;
    nmax[threadIdx.x] = nm;
    tsum[threadIdx.x] = ts;
    kmax[threadIdx.x] = km;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            double a = rmax[threadIdx.x], b = rmax[threadIdx.x + s];
            rmax[threadIdx.x] = (isnan(a) || isnan(b)) ? NAN : fmax(a, b);
            nmax[threadIdx.x] = fmax(nmax[threadIdx.x], nmax[threadIdx.x + s]);
            tsum[threadIdx.x] += tsum[threadIdx.x + s];
            kmax[threadIdx.x] = fmax(kmax[threadIdx.x], kmax[threadIdx.x + s]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        part[4 * k + 0] = rmax[0];
        part[4 * k + 1] = nmax[0];
        part[4 * k + 2] = tsum[0] / ((double)g.nx * g.ny);
        part[4 * k + 3] = kmax[0];
    }
}

// One thread: fold the levels and pick dt (adaptive_dt, src/TimeIntegration.jl:436-454).
__global__ void dt_pick_kernel(Geo g, CflParams c, const double* __restrict__ part, StepScalars* s) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const double INF = 1.0 / 0.0;
    double rate = 0.0, nutm = 0.0, ktm = 0.0, n2max = 0.0, prev = 0.0;
    bool nanr = false;
    for (int k = 0; k < g.nz; ++k) {
        double r = part[4 * k];
        nanr = nanr || isnan(r);
        rate = fmax(rate, r);
        nutm = fmax(nutm, part[4 * k + 1]);
        ktm = fmax(ktm, part[4 * k + 3]);
        double mean = part[4 * k + 2] + c.th_off;
        if (k > 0 && c.buoy) {
            double dzf = g.uniform ? g.dz : 1.0 / lvl(g.idzf, k);
            double n2 = c.anel ? c.gacc * (log(mean) - log(prev)) / dzf
                               : (c.gacc / c.theta0) * (mean - prev) * (1 / dzf);
            n2max = fmax(n2max, n2);
        }
        prev = mean;
    }
    if (nanr) rate = NAN;
    double dt_adv = isnan(rate) ? NAN : (rate > 0 ? c.c_adv / rate : INF);
    double dx2 = 1 / (g.dx * g.dx), dy2 = 1 / (g.dy * g.dy), dz2 = 1 / (c.dz_min * c.dz_min);
    double harm = 1.0 / (dx2 + dy2 + dz2);
    double nu_total = c.nu + nutm;
    double dt_diff = nu_total > 0 ? c.c_diff * harm / nu_total : INF;
    // kappa_t: nut / Pr_t, or the AMD closure's own (max(nu_t, kappa_t) binds, src/TimeIntegration.jl:322-335)
    double kt = c.sgs ? ((g.sgs_model == 3 || g.sgs_model == 7) ? ktm : nutm / c.pr_t) : 0.0;
    double ksgs = fmax(nutm, kt);
    double dt_sgs = ksgs > 0 ? c.c_diff * harm / ksgs : INF;
    double N = sqrt(fmax(n2max, 0.0));
    double dt_buoy = N > 0 ? c.c_buoy / N : INF;
    double f = fabs(c.fcor);
    double dt_cor = f > 0 ? c.c_cor / f : INF;
    double dt = dt_adv;
    int lim = 0;
    if (dt_diff < dt) { dt = dt_diff; lim = 1; }
    if (dt_buoy < dt) { dt = dt_buoy; lim = 2; }
    if (dt_cor < dt) { dt = dt_cor; lim = 3; }
    if (dt_sgs < dt) { dt = dt_sgs; lim = 4; }
    if (isnan(dt)) {
        dt = c.dt_min;
        lim = 6;
    } else {
        double dtp = s->dt_prev;
        if (dtp > 0 && c.growth * dtp < dt) { dt = c.growth * dtp; lim = 5; }
        if (dt < c.dt_min) lim = 6;
        if (dt > c.dt_max) lim = 7;
        dt = fmin(fmax(dt, c.dt_min), c.dt_max);
    }
    s->dt = dt;
    s->limiter = lim;
    s->rate = rate;
    s->nut_max = nutm;
    s->N = N;
}

// The post-step guard per level: any non-finite prognostic value, max |div u|
// (plain, or W-normalised for the sound-proof core), max speed.
template <typename R, bool ANEL, bool UNI>
__global__ void __launch_bounds__(256) guard_levels_kernel(Geo g, const R* __restrict__ u, const R* __restrict__ v,
                                                           const R* __restrict__ w, const R* __restrict__ th,
                                                           const R* __restrict__ p, double* __restrict__ part) {
    __shared__ double dmax[256], smax[256];
    __shared__ int nf;
    if (threadIdx.x == 0) nf = 0;
    __syncthreads();
    const int k = blockIdx.x;
    const double idz = UNI ? g.idz : lvl(g.idzc, k);
    double dm = 0.0, sm = 0.0;
    bool bad = false;
    for (int e = threadIdx.x; e < g.nx * g.ny; e += blockDim.x) {
        const int i = e % g.nx, j = e / g.nx;
        const long long q = pidx(g, i, j, k);
        const double uu = u[q], vv = v[q], ww = w[q];
        const double fin = uu * 0 + vv * 0 + ww * 0 + (double)th[q] * 0 + (double)p[iidx(g, i, j, k)] * 0;
        bad = bad || !(fin == 0.0);
        double du = ((double)u[q + 1] - uu) * g.idx, dv = ((double)v[q + g.sy] - vv) * g.idy;
        double d;
        if (ANEL) {
            double wc = lvl(g.wc, k), wfb = lvl(g.wf, k), wft = lvl(g.wf, k + 1);
            d = (wc * (du + dv) + (wft * (double)w[q + g.sz] - wfb * ww) * idz) / wc;
        } else {
            d = du + dv + ((double)w[q + g.sz] - ww) * idz;
        }
        dm = fmax(dm, fabs(d));
        sm = fmax(sm, fmax(fabs(uu), fmax(fabs(vv), fabs(ww))));
    }
    if (bad) atomicOr(&nf, 1);
    dmax[threadIdx.x] = dm;
    smax[threadIdx.x] = sm;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            dmax[threadIdx.x] = fmax(dmax[threadIdx.x], dmax[threadIdx.x + s]);
            smax[threadIdx.x] = fmax(smax[threadIdx.x], smax[threadIdx.x + s]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        part[3 * k + 0] = nf ? 1.0 : 0.0;
        part[3 * k + 1] = dmax[0];
        part[3 * k + 2] = smax[0];
    }
}

__global__ void set_scalar_kernel(double* p, double v) {
    if (threadIdx.x == 0 && blockIdx.x == 0) *p = v;
}
