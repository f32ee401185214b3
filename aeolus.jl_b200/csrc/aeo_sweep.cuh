// aeo_sweep.cuh -- the fused tendency + predictor sweep of one RK3 substage.
//
// One launch computes, per interior cell, the tendencies of u, v, w and theta
// (advection, molecular diffusion, Smagorinsky SGS, buoyancy, Coriolis, wall
// fluxes, sponge) and writes the predictor u* = u + dt*t (interior-only
// arrays) and the updated, stage-combined theta (padded array).  It restates
// the reference's substage passes, src/Simulations.jl:548-620 (Boussinesq)
// and src/Anelastic.jl:1809-1849 (sound-proof), whose point bodies are
//   centred momentum   src/FiniteVolume.jl:730-797 (_mom_u/v/w_at)
//   centred scalar     src/FiniteVolume.jl:1682-1693 (_adv_centered_at)
//   W-weighted forms   src/Anelastic.jl:1193-1306 (_wmom_u/v/w, _wscal)
//   WENO-JS5 / WENO-Z5 src/AdvectionSchemes.jl:240-255, :319-333, :623-699,
//                      :1203-1256 (_b_recon!, _b_mrecon_u/v/w!)
//   Laplacian          src/FiniteVolume.jl:271-280 (_lap_at)
//   Smagorinsky        src/FiniteVolume.jl:936-944, src/Operators.jl:451-496
//   eddy viscosity     src/FiniteVolume.jl:969-1042, :1280-1300, :1473-1492
//   buoyancy           src/FiniteVolume.jl:838-858, src/Anelastic.jl:1343-1350
//   wall fluxes        src/FiniteVolume.jl:417-440
//   sponge             src/FiniteVolume.jl:578-702
//   predictor / stage  src/Simulations.jl:690-694, :1182-1198
#pragma once

#include "aeo_common.cuh"

template <typename R>
struct SweepArgs {
    Geo g;
    const R* u;
    const R* v;
    const R* w;
    const R* th;
    const R* nut;   // padded eddy viscosity (SGS only)
    const R* th0;   // padded step-start theta (stages 2, 3)
    R* us;          // interior predictor velocities
    R* vs;
    R* ws;
    R* th_out;      // padded
    const double* dtp;  // the step's dt in device memory
    R ca, cb;
    int stage;
    R nu, gacc, theta0, fcor, inv_prt, pr_t, flux_bot, flux_top, sp_alpha, sp_zstart, sp_inv;
    R bref;         // theta0 in stored units (theta is held as theta - offset)
    R c_s;
    const double* cs2;  // the dynamic Smagorinsky coefficient per level
    const R* cs2f;      // ... or per cell (averaging = :local; padded, halos filled; else nullptr)
    double dyn_d2;      // ... and its Delta^2 = (dx dy dz)^(2/3)
    int kofs;       // the AMD closure: its kappa_t sits kofs elements past nut_t (0: kappa_t = nut_t / Pr_t)
};

// padded-array accessor around the thread's point
template <typename R>
struct Nb {
    const R* __restrict__ p;
    long long sy, sz;
    __device__ __forceinline__ R operator()(int di, int dj, int dk) const {
        return __ldg(p + di + (long long)dj * sy + (long long)dk * sz);
    }
    __device__ __forceinline__ Nb shifted(int o) const { return Nb{p + o, sy, sz}; }
};

// ---- WENO reconstructions (src/AdvectionSchemes.jl:105-120, :240-255, :319-333)
template <typename R>
__device__ __forceinline__ R beta3(R a1, R a2) { return a1 * a1 + R(13.0 / 3.0) * (a2 * a2); }

// a / b for the nonlinear weights: FP32 uses the two-instruction division
// (2 ulp; the denominators b_i + eps and (b_i + eps)^2 lie in the normal
// range), FP64 the IEEE one
template <typename R>
__device__ __forceinline__ R wdiv(R a, R b) {
    if constexpr (sizeof(R) == 4) return __fdividef(a, b);
    else return a / b;
}

template <typename R, int ADV>
__device__ __forceinline__ R weno5_left(R v1, R v2, R v3, R v4, R v5) {
    const R s6 = R(1.0 / 6.0);
    R q0 = (R(2) * v1 - R(7) * v2 + R(11) * v3) * s6;
    R q1 = (-v2 + R(5) * v3 + R(2) * v4) * s6;
    R q2 = (R(2) * v3 + R(5) * v4 - v5) * s6;
    R d2a = (v1 - R(2) * v2 + v3) * R(0.5);
    R d2b = (v2 - R(2) * v3 + v4) * R(0.5);
    R d2c = (v3 - R(2) * v4 + v5) * R(0.5);
    R b0 = beta3<R>((v1 - R(4) * v2 + R(3) * v3) * R(0.5), d2a);
    R b1 = beta3<R>((v4 - v2) * R(0.5), d2b);
    R b2 = beta3<R>((R(-3) * v3 + R(4) * v4 - v5) * R(0.5), d2c);
    R a0, a1, a2;
    if (ADV == 2) {  // WENO-Z5, p = 2, eps = eps(T)^2
        const R eps = sizeof(R) == 8 ? R(4.930380657631324e-32) : R(1.4210854715202004e-14);
        R tau = fabs(b0 - b2);
        R t0 = wdiv(tau, b0 + eps), t1 = wdiv(tau, b1 + eps), t2 = wdiv(tau, b2 + eps);
        a0 = R(0.1) * (R(1) + t0 * t0);
        a1 = R(0.6) * (R(1) + t1 * t1);
        a2 = R(0.3) * (R(1) + t2 * t2);
    } else {         // WENO-JS5, eps = 1e-6
        const R e = R(1e-6);
        a0 = wdiv(R(0.1), (b0 + e) * (b0 + e));
        a1 = wdiv(R(0.6), (b1 + e) * (b1 + e));
        a2 = wdiv(R(0.3), (b2 + e) * (b2 + e));
    }
    return (a0 * q0 + a1 * q1 + a2 * q2) / (a0 + a1 + a2);
}

// Upwinded face values between cells c and c+1 along x, y or z
// (src/AdvectionSchemes.jl:623-666, mirror-symmetric selection): the
// left-biased stencil c-2..c+2 for a non-negative face velocity, else the
// mirrored right-biased c+3..c-1.  The six values are loaded once and the
// stencil is selected by the sign, so a warp whose faces see both signs runs
// one reconstruction, not two.
template <typename R, int ADV>
__device__ __forceinline__ R weno_upwind(bool pos, R f0, R f1, R f2, R f3, R f4, R f5) {
    return weno5_left<R, ADV>(pos ? f0 : f5, pos ? f1 : f4, pos ? f2 : f3, pos ? f3 : f2, pos ? f4 : f1);
}
template <typename R, int ADV, class A>
__device__ __forceinline__ R face_x(const A& F, int c, int dj, int dk, R vel) {
    return weno_upwind<R, ADV>(vel >= R(0), F(c - 2, dj, dk), F(c - 1, dj, dk), F(c, dj, dk), F(c + 1, dj, dk),
                               F(c + 2, dj, dk), F(c + 3, dj, dk));
}
template <typename R, int ADV, class A>
__device__ __forceinline__ R face_y(const A& F, int di, int c, int dk, R vel) {
    return weno_upwind<R, ADV>(vel >= R(0), F(di, c - 2, dk), F(di, c - 1, dk), F(di, c, dk), F(di, c + 1, dk),
                               F(di, c + 2, dk), F(di, c + 3, dk));
}
template <typename R, int ADV, class A>
__device__ __forceinline__ R face_z(const A& F, int di, int dj, int c, R vel) {
    return weno_upwind<R, ADV>(vel >= R(0), F(di, dj, c - 2), F(di, dj, c - 1), F(di, dj, c), F(di, dj, c + 1),
                               F(di, dj, c + 2), F(di, dj, c + 3));
}

// The z fluxes of the WENO forms at the top face of a level are the bottom
// fluxes of the level above (same velocities, same stencil values): a
// thread marching up a column carries them instead of recomputing them.
template <typename VT>
struct ZCarry {
    VT f[4];     // w-weighted top-face fluxes of u, v, w, theta
    bool valid;  // f holds the bottom fluxes of this level
};

// The WENO advective fluxes of field f (0 u, 1 v, 2 w, 3 theta) through the
// west x-face, the south y-face and the top z-face of the point the
// accessors are centred on (src/AdvectionSchemes.jl:1203-1256): the
// advecting velocity interpolated to the face times the upwinded face value.
// F is the accessor of field f itself.
template <typename R, int ADV, class AU, class AF>
__device__ __forceinline__ R weno_xflux(int f, const AU& U, const AF& F) {
    R vel;
    if (f == 0) vel = (U(-1, 0, 0) + U(0, 0, 0)) / R(2);
    else if (f == 1) vel = (U(0, -1, 0) + U(0, 0, 0)) / R(2);
    else if (f == 2) vel = (U(0, 0, -1) + U(0, 0, 0)) / R(2);
    else vel = U(0, 0, 0);
    return vel * face_x<R, ADV>(F, -1, 0, 0, vel);
}
template <typename R, int ADV, class AV, class AF>
__device__ __forceinline__ R weno_yflux(int f, const AV& V, const AF& F) {
    R vel;
    if (f == 0) vel = (V(-1, 0, 0) + V(0, 0, 0)) / R(2);
    else if (f == 1) vel = (V(0, -1, 0) + V(0, 0, 0)) / R(2);
    else if (f == 2) vel = (V(0, 0, -1) + V(0, 0, 0)) / R(2);
    else vel = V(0, 0, 0);
    return vel * face_y<R, ADV>(F, 0, -1, 0, vel);
}
// S = 0: the top z-face; S = -1: the bottom one (the top face one level down)
template <typename R, int ADV, int S, class AW, class AF>
__device__ __forceinline__ R weno_zflux(int f, const AW& W, const AF& F) {
    R vel;
    if (f == 0) vel = (W(-1, 0, 1 + S) + W(0, 0, 1 + S)) / R(2);
    else if (f == 1) vel = (W(0, -1, 1 + S) + W(0, 0, 1 + S)) / R(2);
    else if (f == 2) vel = (W(0, 0, S) + W(0, 0, 1 + S)) / R(2);
    else vel = W(0, 0, 1 + S);
    return vel * face_z<R, ADV>(F, 0, 0, S, vel);
}

// ---- the tendency at one point ------------------------------------------------
// U, V, W, T, N are accessors (di, dj, dk) -> value around the point at level
// k; the same arithmetic serves the direct form (global memory) and the
// tiled form (shared-memory planes).  VT is the value type: R, or a pair of
// FP32 lanes (F2) for two x-adjacent cells of the paired sweep (the
// centred forms only).
template <typename R, int ADV, bool SGS, bool ANEL, bool UNI, bool EXT = false, bool AMD = false, class AU, class AV,
          class AW, class AT, class AN, typename VT>
__device__ __forceinline__ void sweep_point(const Met<R, UNI>& m, const SweepArgs<R>& a, const Geo& g, int k,
                                            const AU& U, const AV& V, const AW& W, const AT& T, const AN& N, VT& tu,
                                            VT& tv, VT& tw, VT& tt, ZCarry<VT>* zc = nullptr) {
    const VT idx = VT(g.idx), idy = VT(g.idy), idx2 = VT(g.idx2), idy2 = VT(g.idy2);
    const VT h = VT(0.5);

    if constexpr (ANEL) {
        // W-weighted centred forms (src/Anelastic.jl:1193-1306)
        VT iwc = m.iwc(k), wfb = m.wf(k), wft = m.wf(k + 1);
        {
            VT uce = h * (U(0, 0, 0) + U(1, 0, 0)), ucw = h * (U(-1, 0, 0) + U(0, 0, 0));
            VT d_uu_dx = (uce * uce - ucw * ucw) * idx;
            VT vun = h * (V(-1, 1, 0) + V(0, 1, 0)), uvn = h * (U(0, 0, 0) + U(0, 1, 0));
            VT vus = h * (V(-1, 0, 0) + V(0, 0, 0)), uvs = h * (U(0, -1, 0) + U(0, 0, 0));
            VT d_vu_dy = (vun * uvn - vus * uvs) * idy;
            VT wut = h * (W(-1, 0, 1) + W(0, 0, 1)), uwt = h * (U(0, 0, 0) + U(0, 0, 1));
            VT wub = h * (W(-1, 0, 0) + W(0, 0, 0)), uwb = h * (U(0, 0, -1) + U(0, 0, 0));
            VT d_wu_dz = (wft * wut * uwt - wfb * wub * uwb) * m.idz(k) * iwc;
            tu = VT(0) - (d_uu_dx + d_vu_dy + d_wu_dz);
        }
        {
            VT uve = h * (U(1, -1, 0) + U(1, 0, 0)), vue = h * (V(0, 0, 0) + V(1, 0, 0));
            VT uvw = h * (U(0, -1, 0) + U(0, 0, 0)), vuw = h * (V(-1, 0, 0) + V(0, 0, 0));
            VT d_uv_dx = (uve * vue - uvw * vuw) * idx;
            VT vcn = h * (V(0, 0, 0) + V(0, 1, 0)), vcs = h * (V(0, -1, 0) + V(0, 0, 0));
            VT d_vv_dy = (vcn * vcn - vcs * vcs) * idy;
            VT wvt = h * (W(0, -1, 1) + W(0, 0, 1)), vwt = h * (V(0, 0, 0) + V(0, 0, 1));
            VT wvb = h * (W(0, -1, 0) + W(0, 0, 0)), vwb = h * (V(0, 0, -1) + V(0, 0, 0));
            VT d_wv_dz = (wft * wvt * vwt - wfb * wvb * vwb) * m.idz(k) * iwc;
            tv = VT(0) - (d_uv_dx + d_vv_dy + d_wv_dz);
        }
        {
            VT iwf = m.iwf(k), wcb = m.wc(k - 1), wct = m.wc(k);
            VT uwe = m.zflux(k, U(1, 0, -1), U(1, 0, 0)), wue = h * (W(0, 0, 0) + W(1, 0, 0));
            VT uww = m.zflux(k, U(0, 0, -1), U(0, 0, 0)), wuw = h * (W(-1, 0, 0) + W(0, 0, 0));
            VT d_uw_dx = (uwe * wue - uww * wuw) * idx;
            VT vwn = m.zflux(k, V(0, 1, -1), V(0, 1, 0)), wvn = h * (W(0, 0, 0) + W(0, 1, 0));
            VT vws = m.zflux(k, V(0, 0, -1), V(0, 0, 0)), wvs = h * (W(0, -1, 0) + W(0, 0, 0));
            VT d_vw_dy = (vwn * wvn - vws * wvs) * idy;
            VT wtop = h * (W(0, 0, 0) + W(0, 0, 1)), wbot = h * (W(0, 0, -1) + W(0, 0, 0));
            VT d_ww_dz = (wct * wtop * wtop - wcb * wbot * wbot) * m.idzf(k) * iwf;
            tw = VT(0) - (d_uw_dx + d_vw_dy + d_ww_dz);
        }
        {
            VT ue = U(1, 0, 0) * h * (T(0, 0, 0) + T(1, 0, 0)), uw = U(0, 0, 0) * h * (T(-1, 0, 0) + T(0, 0, 0));
            VT vn = V(0, 1, 0) * h * (T(0, 0, 0) + T(0, 1, 0)), vs = V(0, 0, 0) * h * (T(0, -1, 0) + T(0, 0, 0));
            VT wt = wft * W(0, 0, 1) * h * (T(0, 0, 0) + T(0, 0, 1)), wb = wfb * W(0, 0, 0) * h * (T(0, 0, -1) + T(0, 0, 0));
            tt = VT(0) - ((ue - uw) * idx + (vn - vs) * idy + (wt - wb) * m.idz(k) * iwc);
        }
    } else if constexpr (ADV == 0) {
        // centred flux form (src/FiniteVolume.jl:730-797, :1682-1693)
        {
            VT uce = h * (U(0, 0, 0) + U(1, 0, 0)), ucw = h * (U(-1, 0, 0) + U(0, 0, 0));
            VT d_uu_dx = (uce * uce - ucw * ucw) * idx;
            VT vun = h * (V(-1, 1, 0) + V(0, 1, 0)), uvn = h * (U(0, 0, 0) + U(0, 1, 0));
            VT vus = h * (V(-1, 0, 0) + V(0, 0, 0)), uvs = h * (U(0, -1, 0) + U(0, 0, 0));
            VT d_vu_dy = (vun * uvn - vus * uvs) * idy;
            VT wut = h * (W(-1, 0, 1) + W(0, 0, 1)), uwt = h * (U(0, 0, 0) + U(0, 0, 1));
            VT wub = h * (W(-1, 0, 0) + W(0, 0, 0)), uwb = h * (U(0, 0, -1) + U(0, 0, 0));
            VT d_wu_dz = (wut * uwt - wub * uwb) * m.idz(k);
            tu = VT(0) - (d_uu_dx + d_vu_dy + d_wu_dz);
        }
        {
            VT uve = h * (U(1, -1, 0) + U(1, 0, 0)), vue = h * (V(0, 0, 0) + V(1, 0, 0));
            VT uvw = h * (U(0, -1, 0) + U(0, 0, 0)), vuw = h * (V(-1, 0, 0) + V(0, 0, 0));
            VT d_uv_dx = (uve * vue - uvw * vuw) * idx;
            VT vcn = h * (V(0, 0, 0) + V(0, 1, 0)), vcs = h * (V(0, -1, 0) + V(0, 0, 0));
            VT d_vv_dy = (vcn * vcn - vcs * vcs) * idy;
            VT wvt = h * (W(0, -1, 1) + W(0, 0, 1)), vwt = h * (V(0, 0, 0) + V(0, 0, 1));
            VT wvb = h * (W(0, -1, 0) + W(0, 0, 0)), vwb = h * (V(0, 0, -1) + V(0, 0, 0));
            VT d_wv_dz = (wvt * vwt - wvb * vwb) * m.idz(k);
            tv = VT(0) - (d_uv_dx + d_vv_dy + d_wv_dz);
        }
        {
            VT uwe = m.zflux(k, U(1, 0, -1), U(1, 0, 0)), wue = h * (W(0, 0, 0) + W(1, 0, 0));
            VT uww = m.zflux(k, U(0, 0, -1), U(0, 0, 0)), wuw = h * (W(-1, 0, 0) + W(0, 0, 0));
            VT d_uw_dx = (uwe * wue - uww * wuw) * idx;
            VT vwn = m.zflux(k, V(0, 1, -1), V(0, 1, 0)), wvn = h * (W(0, 0, 0) + W(0, 1, 0));
            VT vws = m.zflux(k, V(0, 0, -1), V(0, 0, 0)), wvs = h * (W(0, -1, 0) + W(0, 0, 0));
            VT d_vw_dy = (vwn * wvn - vws * wvs) * idy;
            VT wct = h * (W(0, 0, 0) + W(0, 0, 1)), wcb = h * (W(0, 0, -1) + W(0, 0, 0));
            VT d_ww_dz = (wct * wct - wcb * wcb) * m.idzf(k);
            tw = VT(0) - (d_uw_dx + d_vw_dy + d_ww_dz);
        }
        {
            VT ue = U(1, 0, 0) * h * (T(0, 0, 0) + T(1, 0, 0)), uw = U(0, 0, 0) * h * (T(-1, 0, 0) + T(0, 0, 0));
            VT vn = V(0, 1, 0) * h * (T(0, 0, 0) + T(0, 1, 0)), vs = V(0, 0, 0) * h * (T(0, -1, 0) + T(0, 0, 0));
            VT wt = W(0, 0, 1) * h * (T(0, 0, 0) + T(0, 0, 1)), wb = W(0, 0, 0) * h * (T(0, 0, -1) + T(0, 0, 0));
            tt = VT(0) - ((ue - uw) * idx + (vn - vs) * idy + (wt - wb) * m.idz(k));
        }
    } else if constexpr (!EXT) {
        // WENO flux forms on a uniform grid (src/AdvectionSchemes.jl:685-699, :1203-1256);
        // EXT: the caller computed them (face fluxes shared between cells) into tu..tt
        const VT idz = VT(g.idz);
        {
            VT Ue = (U(0, 0, 0) + U(1, 0, 0)) / VT(2), Uw = (U(-1, 0, 0) + U(0, 0, 0)) / VT(2);
            VT dx = (Ue * face_x<VT, ADV>(U, 0, 0, 0, Ue) - Uw * face_x<VT, ADV>(U, -1, 0, 0, Uw)) * idx;
            VT Vn = (V(-1, 1, 0) + V(0, 1, 0)) / VT(2), Vs = (V(-1, 0, 0) + V(0, 0, 0)) / VT(2);
            VT dy = (Vn * face_y<VT, ADV>(U, 0, 0, 0, Vn) - Vs * face_y<VT, ADV>(U, 0, -1, 0, Vs)) * idy;
            VT Wt = (W(-1, 0, 1) + W(0, 0, 1)) / VT(2), Wb = (W(-1, 0, 0) + W(0, 0, 0)) / VT(2);
            const VT ft = Wt * face_z<VT, ADV>(U, 0, 0, 0, Wt);
            const VT fb = (zc && zc->valid) ? zc->f[0] : VT(Wb * face_z<VT, ADV>(U, 0, 0, -1, Wb));
            if (zc) zc->f[0] = ft;
            VT dz = (ft - fb) * idz;
            tu = VT(0) - (dx + dy + dz);
        }
        {
            VT Ue = (U(1, -1, 0) + U(1, 0, 0)) / VT(2), Uw = (U(0, -1, 0) + U(0, 0, 0)) / VT(2);
            VT dx = (Ue * face_x<VT, ADV>(V, 0, 0, 0, Ue) - Uw * face_x<VT, ADV>(V, -1, 0, 0, Uw)) * idx;
            VT Vn = (V(0, 0, 0) + V(0, 1, 0)) / VT(2), Vs = (V(0, -1, 0) + V(0, 0, 0)) / VT(2);
            VT dy = (Vn * face_y<VT, ADV>(V, 0, 0, 0, Vn) - Vs * face_y<VT, ADV>(V, 0, -1, 0, Vs)) * idy;
            VT Wt = (W(0, -1, 1) + W(0, 0, 1)) / VT(2), Wb = (W(0, -1, 0) + W(0, 0, 0)) / VT(2);
            const VT ft = Wt * face_z<VT, ADV>(V, 0, 0, 0, Wt);
            const VT fb = (zc && zc->valid) ? zc->f[1] : VT(Wb * face_z<VT, ADV>(V, 0, 0, -1, Wb));
            if (zc) zc->f[1] = ft;
            VT dz = (ft - fb) * idz;
            tv = VT(0) - (dx + dy + dz);
        }
        {
            VT Ue = (U(1, 0, -1) + U(1, 0, 0)) / VT(2), Uw = (U(0, 0, -1) + U(0, 0, 0)) / VT(2);
            VT dx = (Ue * face_x<VT, ADV>(W, 0, 0, 0, Ue) - Uw * face_x<VT, ADV>(W, -1, 0, 0, Uw)) * idx;
            VT Vn = (V(0, 1, -1) + V(0, 1, 0)) / VT(2), Vs = (V(0, 0, -1) + V(0, 0, 0)) / VT(2);
            VT dy = (Vn * face_y<VT, ADV>(W, 0, 0, 0, Vn) - Vs * face_y<VT, ADV>(W, 0, -1, 0, Vs)) * idy;
            VT Wt = (W(0, 0, 0) + W(0, 0, 1)) / VT(2), Wb = (W(0, 0, -1) + W(0, 0, 0)) / VT(2);
            const VT ft = Wt * face_z<VT, ADV>(W, 0, 0, 0, Wt);
            const VT fb = (zc && zc->valid) ? zc->f[2] : VT(Wb * face_z<VT, ADV>(W, 0, 0, -1, Wb));
            if (zc) zc->f[2] = ft;
            VT dz = (ft - fb) * idz;
            tw = VT(0) - (dx + dy + dz);
        }
        {
            VT uw = U(0, 0, 0), ue = U(1, 0, 0);
            VT Fx = (ue * face_x<VT, ADV>(T, 0, 0, 0, ue) - uw * face_x<VT, ADV>(T, -1, 0, 0, uw)) * idx;
            VT vs = V(0, 0, 0), vn = V(0, 1, 0);
            VT Fy = (vn * face_y<VT, ADV>(T, 0, 0, 0, vn) - vs * face_y<VT, ADV>(T, 0, -1, 0, vs)) * idy;
            VT wb = W(0, 0, 0), wt = W(0, 0, 1);
            const VT ft = wt * face_z<VT, ADV>(T, 0, 0, 0, wt);
            const VT fb = (zc && zc->valid) ? zc->f[3] : VT(wb * face_z<VT, ADV>(T, 0, 0, -1, wb));
            if (zc) zc->f[3] = ft;
            VT Fz = (ft - fb) * idz;
            tt = VT(0) - (Fx + Fy + Fz);
        }
    }

    // molecular viscosity / diffusion
    if (a.nu != R(0)) {
        VT c;
        c = U(0, 0, 0);
        tu = tu + a.nu * ((U(1, 0, 0) - VT(2) * c + U(-1, 0, 0)) * idx2 + (U(0, 1, 0) - VT(2) * c + U(0, -1, 0)) * idy2 +
                          m.lapz(LOC_FX, k, U(0, 0, -1), c, U(0, 0, 1)));
        c = V(0, 0, 0);
        tv = tv + a.nu * ((V(1, 0, 0) - VT(2) * c + V(-1, 0, 0)) * idx2 + (V(0, 1, 0) - VT(2) * c + V(0, -1, 0)) * idy2 +
                          m.lapz(LOC_FY, k, V(0, 0, -1), c, V(0, 0, 1)));
        c = W(0, 0, 0);
        tw = tw + a.nu * ((W(1, 0, 0) - VT(2) * c + W(-1, 0, 0)) * idx2 + (W(0, 1, 0) - VT(2) * c + W(0, -1, 0)) * idy2 +
                          m.lapz(LOC_FZ, k, W(0, 0, -1), c, W(0, 0, 1)));
        c = T(0, 0, 0);
        tt = tt + a.nu * ((T(1, 0, 0) - VT(2) * c + T(-1, 0, 0)) * idx2 + (T(0, 1, 0) - VT(2) * c + T(0, -1, 0)) * idy2 +
                          m.lapz(LOC_C, k, T(0, 0, -1), c, T(0, 0, 1)));
    }

    // Smagorinsky SGS fluxes (eddy viscosity from the nut array, halos filled)
    if (SGS) {
        const VT q4 = VT(0.25);
        {
            VT fxE = N(0, 0, 0) * (U(1, 0, 0) - U(0, 0, 0)) * idx;
            VT fxW = N(-1, 0, 0) * (U(0, 0, 0) - U(-1, 0, 0)) * idx;
            VT eN = q4 * (N(-1, 0, 0) + N(0, 0, 0) + N(-1, 1, 0) + N(0, 1, 0));
            VT eS = q4 * (N(-1, -1, 0) + N(0, -1, 0) + N(-1, 0, 0) + N(0, 0, 0));
            VT fyN = eN * (U(0, 1, 0) - U(0, 0, 0)) * idy;
            VT fyS = eS * (U(0, 0, 0) - U(0, -1, 0)) * idy;
            VT eT = q4 * (N(-1, 0, 0) + N(0, 0, 0) + N(-1, 0, 1) + N(0, 0, 1));
            VT eB = q4 * (N(-1, 0, -1) + N(0, 0, -1) + N(-1, 0, 0) + N(0, 0, 0));
            VT fzT = eT * (U(0, 0, 1) - U(0, 0, 0)) * m.idzf(k + 1);
            VT fzB = eB * (U(0, 0, 0) - U(0, 0, -1)) * m.idzf(k);
            VT vert = ANEL ? (m.wf(k + 1) * fzT - m.wf(k) * fzB) * m.idz(k) * m.iwc(k)
                          : (fzT - fzB) * m.idz(k);
            tu += (fxE - fxW) * idx + (fyN - fyS) * idy + vert;
        }
        {
            VT fyN = N(0, 0, 0) * (V(0, 1, 0) - V(0, 0, 0)) * idy;
            VT fyS = N(0, -1, 0) * (V(0, 0, 0) - V(0, -1, 0)) * idy;
            VT eE = q4 * (N(0, -1, 0) + N(1, -1, 0) + N(0, 0, 0) + N(1, 0, 0));
            VT eW = q4 * (N(-1, -1, 0) + N(0, -1, 0) + N(-1, 0, 0) + N(0, 0, 0));
            VT fxE = eE * (V(1, 0, 0) - V(0, 0, 0)) * idx;
            VT fxW = eW * (V(0, 0, 0) - V(-1, 0, 0)) * idx;
            VT eT = q4 * (N(0, -1, 0) + N(0, 0, 0) + N(0, -1, 1) + N(0, 0, 1));
            VT eB = q4 * (N(0, -1, -1) + N(0, 0, -1) + N(0, -1, 0) + N(0, 0, 0));
            VT fzT = eT * (V(0, 0, 1) - V(0, 0, 0)) * m.idzf(k + 1);
            VT fzB = eB * (V(0, 0, 0) - V(0, 0, -1)) * m.idzf(k);
            VT vert = ANEL ? (m.wf(k + 1) * fzT - m.wf(k) * fzB) * m.idz(k) * m.iwc(k)
                          : (fzT - fzB) * m.idz(k);
            tv += (fxE - fxW) * idx + (fyN - fyS) * idy + vert;
        }
        {
            VT fzT = N(0, 0, 0) * (W(0, 0, 1) - W(0, 0, 0)) * m.idz(k);
            VT fzB = N(0, 0, -1) * (W(0, 0, 0) - W(0, 0, -1)) * m.idz(k - 1);
            VT eE = q4 * (N(0, 0, -1) + N(1, 0, -1) + N(0, 0, 0) + N(1, 0, 0));
            VT eW = q4 * (N(-1, 0, -1) + N(0, 0, -1) + N(-1, 0, 0) + N(0, 0, 0));
            VT fxE = eE * (W(1, 0, 0) - W(0, 0, 0)) * idx;
            VT fxW = eW * (W(0, 0, 0) - W(-1, 0, 0)) * idx;
            VT eN = q4 * (N(0, 0, -1) + N(0, 1, -1) + N(0, 0, 0) + N(0, 1, 0));
            VT eS = q4 * (N(0, -1, -1) + N(0, 0, -1) + N(0, -1, 0) + N(0, 0, 0));
            VT fyN = eN * (W(0, 1, 0) - W(0, 0, 0)) * idy;
            VT fyS = eS * (W(0, 0, 0) - W(0, -1, 0)) * idy;
            VT vert = ANEL ? (m.wc(k) * fzT - m.wc(k - 1) * fzB) * m.idzf(k) * m.iwf(k)
                          : (fzT - fzB) * m.idzf(k);
            tw += (fxE - fxW) * idx + (fyN - fyS) * idy + vert;
        }
        if (!ANEL) {
            // K = nut (scaled by 1/Pr_t), or the AMD closure's own kappa_t (inv_prt = 1)
            const AN K = AMD ? N.shifted(a.kofs) : N;
            VT nE = h * (K(0, 0, 0) + K(1, 0, 0)), nW = h * (K(-1, 0, 0) + K(0, 0, 0));
            VT nN = h * (K(0, 0, 0) + K(0, 1, 0)), nS = h * (K(0, -1, 0) + K(0, 0, 0));
            VT nT = h * (K(0, 0, 0) + K(0, 0, 1)), nB = h * (K(0, 0, -1) + K(0, 0, 0));
            VT fxE = nE * (T(1, 0, 0) - T(0, 0, 0)) * idx, fxW = nW * (T(0, 0, 0) - T(-1, 0, 0)) * idx;
            VT fyN = nN * (T(0, 1, 0) - T(0, 0, 0)) * idy, fyS = nS * (T(0, 0, 0) - T(0, -1, 0)) * idy;
            VT fzT = nT * (T(0, 0, 1) - T(0, 0, 0)) * m.idzf(k + 1), fzB = nB * (T(0, 0, 0) - T(0, 0, -1)) * m.idzf(k);
            tt += a.inv_prt * ((fxE - fxW) * idx + (fyN - fyS) * idy + (fzT - fzB) * m.idz(k));
        } else {
            // kappa = nut / Pr_t, the W-weighted form (1/Pr_t applied once per face), or
            // the AMD closure's own kappa_t (inv_prt = 1)
            const AN K = AMD ? N.shifted(a.kofs) : N;
            const VT hk = h * a.inv_prt;
            const VT N0 = K(0, 0, 0);
            VT fxE = hk * (N0 + K(1, 0, 0)) * (T(1, 0, 0) - T(0, 0, 0)) * idx;
            VT fxW = hk * (K(-1, 0, 0) + N0) * (T(0, 0, 0) - T(-1, 0, 0)) * idx;
            VT fyN = hk * (N0 + K(0, 1, 0)) * (T(0, 1, 0) - T(0, 0, 0)) * idy;
            VT fyS = hk * (K(0, -1, 0) + N0) * (T(0, 0, 0) - T(0, -1, 0)) * idy;
            VT fzT = hk * (N0 + K(0, 0, 1)) * (T(0, 0, 1) - T(0, 0, 0)) * m.idzf(k + 1);
            VT fzB = hk * (K(0, 0, -1) + N0) * (T(0, 0, 0) - T(0, 0, -1)) * m.idzf(k);
            VT vert = (m.wf(k + 1) * fzT - m.wf(k) * fzB) * m.idz(k) * m.iwc(k);
            tt += (fxE - fxW) * idx + (fyN - fyS) * idy + vert;
        }
    }

    // buoyancy on the z faces
    if (ANEL) {
        if (a.gacc != R(0)) {
            VT tb = m.thf(k);
            VT coef = m.gthf(k);   // g / theta_f
            tw += coef * (m.zface(k, T(0, 0, -1), T(0, 0, 0)) - tb);
        }
    } else if (a.theta0 != R(0)) {
        tw += (a.gacc / a.theta0) * (m.zface(k, T(0, 0, -1), T(0, 0, 0)) - a.bref);
    }
    // Coriolis
    if (a.fcor != R(0)) {
        VT v_at_u = VT(0.25) * (V(-1, 0, 0) + V(0, 0, 0) + V(-1, 1, 0) + V(0, 1, 0));
        tu += a.fcor * v_at_u;
        VT u_at_v = VT(0.25) * (U(0, -1, 0) + U(1, -1, 0) + U(0, 0, 0) + U(1, 0, 0));
        tv -= a.fcor * u_at_v;
    }
    // prescribed wall fluxes of theta
    if (k == 0) tt += a.flux_bot * m.idz(0);
    if (k == g.nz - 1) tt -= a.flux_top * m.idz(g.nz - 1);
    // Rayleigh sponge toward rest: the per-level rates alpha sin^2(pi/2 (z - z_s)/(z_top - z_s))
    // above z_s, zero below (src/FiniteVolume.jl:578-702)
    if (a.sp_alpha != R(0)) {
        const VT rc = m.spc(k), rf = m.spf(k);
        tu -= rc * U(0, 0, 0);
        tv -= rc * V(0, 0, 0);
        tw -= rf * W(0, 0, 0);
    }
}

// ---- direct form: one thread per cell, neighbours from global memory --------------
template <typename R, int ADV, bool SGS, bool ANEL, bool UNI>
__global__ void __launch_bounds__(256) sweep_kernel(SweepArgs<R> a) {
    const Geo& g = a.g;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int j = blockIdx.y * blockDim.y + threadIdx.y;
    int k = blockIdx.z * blockDim.z + threadIdx.z;
    if (i >= g.nx || j >= g.ny || k >= g.nz) return;
    const long long q = pidx(g, i, j, k);
    const long long sy = g.sy, sz = g.sz;
    Nb<R> U{a.u + q, sy, sz}, V{a.v + q, sy, sz}, W{a.w + q, sy, sz}, T{a.th + q, sy, sz};
    Nb<R> N{SGS ? a.nut + q : a.u + q, sy, sz};
    R tu, tv, tw, tt;
    sweep_point<R, ADV, SGS, ANEL, UNI>(Met<R, UNI>(g), a, g, k, U, V, W, T, N, tu, tv, tw, tt);
    // predictor and the theta update (with the RK3 stage combination)
    const long long qi = iidx(g, i, j, k);
    const R dt = R(__ldg(a.dtp));
    a.us[qi] = U(0, 0, 0) + dt * tu;
    a.vs[qi] = V(0, 0, 0) + dt * tv;
    a.ws[qi] = (g.bc_z == 1 && k == 0) ? R(0) : W(0, 0, 0) + dt * tw;
    R tn = T(0, 0, 0) + dt * tt;
    if (a.stage) tn = rk_combine(a.ca, a.cb, a.th0[q], tn);  // th0 may alias th_out (stage 3): plain load
    a.th_out[q] = tn;
}

template <typename R>
__device__ __forceinline__ R sqrt_ratio_or_zero(R b, R a, R c) {
    return a > R(0) ? c * sqrt(b / a) : R(0);
}

// The sigma-model operator D = s3 (s1 - s2)(s2 - s3) / s1^2 of the velocity
// gradient g (rows g_a = d u_a / d x_b), clipped at zero (sigma_operator,
// src/operators/sigma_closure.jl:130-196): the eigenvalues of g^T g in closed
// form -- the trigonometric solution in the deviator, then, where the smaller
// gap is under 1 % of the spread, the simple eigenvalue deflated through the
// largest cross product of two rows of G - lambda I and the close pair
// recomputed from the 2 x 2 compression (_sym3_eigvals :48-97) -- and s3 from
// the determinant (exactly zero for a gradient of rank <= 2).  Out of line:
// the closed form is long and only the sigma closure calls it.
template <typename R>
__device__ __noinline__ R sigma_operator(R g11, R g12, R g13, R g21, R g22, R g23, R g31, R g32, R g33) {
    const R G11 = g11 * g11 + g21 * g21 + g31 * g31, G22 = g12 * g12 + g22 * g22 + g32 * g32;
    const R G33 = g13 * g13 + g23 * g23 + g33 * g33;
    const R G12 = g11 * g12 + g21 * g22 + g31 * g32, G13 = g11 * g13 + g21 * g23 + g31 * g33;
    const R G23 = g12 * g13 + g22 * g23 + g32 * g33;
    const R m = (G11 + G22 + G33) / R(3);
    const R a = G11 - m, b = G22 - m, c = G33 - m;
    const R off2 = G12 * G12 + G13 * G13 + G23 * G23;
    const R al1 = (a * a + b * b + c * c + R(2) * off2) / R(6);
    R l1 = m, l2 = m;
    if (al1 > R(0)) {
        const R detd = a * (b * c - G23 * G23) - G12 * (G12 * c - G23 * G13) + G13 * (G12 * G23 - b * G13);
        const R al2 = detd / R(2);
        const R r = fmin(fmax(al2 / (al1 * sqrt(al1)), R(-1)), R(1));
        R sp, cp;
        sincos(acos(r) / R(3), &sp, &cp);
        const R s = R(2) * sqrt(al1);
        l1 = m + s * cp;
        const R l3 = m - s * (cp + sqrt(R(3)) * sp) / R(2);
        l2 = R(3) * m - l1 - l3;
        if (!(fmin(l1 - l2, l2 - l3) >= R(0.01) * (l1 - l3))) {
            const bool top = (l1 - l2) >= (l2 - l3);
            const R iso = top ? l1 : l3;
            const R r1x = G11 - iso, r1y = G12, r1z = G13;
            const R r2x = G12, r2y = G22 - iso, r2z = G23;
            const R r3x = G13, r3y = G23, r3z = G33 - iso;
            // cross products of the rows; the largest is the simple eigenvector
            R vx = r1y * r2z - r1z * r2y, vy = r1z * r2x - r1x * r2z, vz = r1x * r2y - r1y * r2x;
            R nv = vx * vx + vy * vy + vz * vz;
            {
                const R cx = r1y * r3z - r1z * r3y, cy = r1z * r3x - r1x * r3z, cz = r1x * r3y - r1y * r3x;
                const R n = cx * cx + cy * cy + cz * cz;
                if (n > nv) { vx = cx; vy = cy; vz = cz; nv = n; }
            }
            {
                const R cx = r2y * r3z - r2z * r3y, cy = r2z * r3x - r2x * r3z, cz = r2x * r3y - r2y * r3x;
                const R n = cx * cx + cy * cy + cz * cz;
                if (n > nv) { vx = cx; vy = cy; vz = cz; nv = n; }
            }
            if (nv > R(0)) {
                const R inv = sqrt(nv);
                vx = vx / inv; vy = vy / inv; vz = vz / inv;
                const R ax = fabs(vx), ay = fabs(vy), az = fabs(vz);
                const R tx = (ax <= ay && ax <= az) ? R(1) : R(0);
                const R ty = (ax <= ay && ax <= az) ? R(0) : (ay <= az ? R(1) : R(0));
                const R tz = (ax <= ay && ax <= az) ? R(0) : (ay <= az ? R(0) : R(1));
                R e1x = vy * tz - vz * ty, e1y = vz * tx - vx * tz, e1z = vx * ty - vy * tx;
                const R ne = sqrt(e1x * e1x + e1y * e1y + e1z * e1z);
                e1x = e1x / ne; e1y = e1y / ne; e1z = e1z / ne;
                const R e2x = vy * e1z - vz * e1y, e2y = vz * e1x - vx * e1z, e2z = vx * e1y - vy * e1x;
                const R Gvx = G11 * vx + G12 * vy + G13 * vz, Gvy = G12 * vx + G22 * vy + G23 * vz,
                        Gvz = G13 * vx + G23 * vy + G33 * vz;
                const R G1x = G11 * e1x + G12 * e1y + G13 * e1z, G1y = G12 * e1x + G22 * e1y + G23 * e1z,
                        G1z = G13 * e1x + G23 * e1y + G33 * e1z;
                const R G2x = G11 * e2x + G12 * e2y + G13 * e2z, G2y = G12 * e2x + G22 * e2y + G23 * e2z,
                        G2z = G13 * e2x + G23 * e2y + G33 * e2z;
                const R liso = vx * Gvx + vy * Gvy + vz * Gvz;
                const R pp = e1x * G1x + e1y * G1y + e1z * G1z;
                const R qq = e1x * G2x + e1y * G2y + e1z * G2z;
                const R rr = e2x * G2x + e2y * G2y + e2z * G2z;
                const R h = sqrt((pp - rr) * (pp - rr) + R(4) * qq * qq) / R(2);
                const R mp = (pp + rr) / R(2) + h, mm = (pp + rr) / R(2) - h;
                if (top) { l1 = fmax(liso, mp); l2 = mp; }
                else { l1 = mp; l2 = mm; }
            }
        }
    }
    const R s1 = sqrt(fmax(l1, R(0)));
    if (!(s1 > R(0))) return R(0);
    const R s2 = sqrt(fmax(l2, R(0)));
    const R detg = g11 * (g22 * g33 - g23 * g32) - g12 * (g21 * g33 - g23 * g31) + g13 * (g21 * g32 - g22 * g31);
    const R pr = s1 * s2;
    const R s3 = pr > R(0) ? fabs(detg) / pr : R(0);
    const R d12 = fmax(l1 - l2, R(0)) / (s1 + s2);
    return fmax(s3 * d12 * (s2 - s3) / (s1 * s1), R(0));
}


// Smagorinsky nut = (C_s Delta_k)^2 |S| at a cell centre (src/FiniteVolume.jl:936-944,
// strain src/Operators.jl:451-496), accessors around the point at level k; or,
// with g.sgs_model = 1, Vreman's nut = c sqrt(B_beta / alpha:alpha) from the
// same gradient tensor, B_beta in the Cauchy-Binet form over the rows a_m =
// d_m u (_vreman_point / _vreman_body!, src/operators/sgs_amd_vreman.jl:93-100,
// :293-298; uniform grids).
template <typename R, bool UNI, class AU, class AV, class AW>
__device__ __forceinline__ auto smag_point(const Met<R, UNI>& m, const Geo& g, int k, R c_s, const AU& U, const AV& V,
                                           const AW& W) {
    using VT = decltype(U(0, 0, 0));   // R, or a pair of FP32 lanes
    const R idx = R(g.idx), idy = R(g.idy), idz = m.idz(k), ido = m.idz_off(k);
    const R cf = c_s * m.filter(k);
    const R coef = cf * cf;
    VT du_dx = (U(1, 0, 0) - U(0, 0, 0)) * idx;
    VT dv_dy = (V(0, 1, 0) - V(0, 0, 0)) * idy;
    VT dw_dz = (W(0, 0, 1) - W(0, 0, 0)) * idz;
    VT du_dy = ((U(0, 1, 0) + U(1, 1, 0)) - (U(0, -1, 0) + U(1, -1, 0))) * (R(0.25) * idy);
    VT dv_dx = ((V(1, 0, 0) + V(1, 1, 0)) - (V(-1, 0, 0) + V(-1, 1, 0))) * (R(0.25) * idx);
    VT du_dz = ((U(0, 0, 1) + U(1, 0, 1)) - (U(0, 0, -1) + U(1, 0, -1))) * (R(0.25) * ido);
    VT dw_dx = ((W(1, 0, 0) + W(1, 0, 1)) - (W(-1, 0, 0) + W(-1, 0, 1))) * (R(0.25) * idx);
    VT dv_dz = ((V(0, 0, 1) + V(0, 1, 1)) - (V(0, 0, -1) + V(0, 1, -1))) * (R(0.25) * ido);
    VT dw_dy = ((W(0, 1, 0) + W(0, 1, 1)) - (W(0, -1, 0) + W(0, -1, 1))) * (R(0.25) * idy);
    if (g.sgs_model == 2)   // sigma model: (C_sigma Delta)^2 D_sigma (compute_sigma_nut!, sigma_closure.jl:208-222)
        return VT(VT(coef) * sigma_operator(VT(du_dx), VT(du_dy), VT(du_dz), VT(dv_dx), VT(dv_dy), VT(dv_dz),
                                            VT(dw_dx), VT(dw_dy), VT(dw_dz)));
    if (g.sgs_model == 1) {
        const R d2x = R(g.dx * g.dx), d2y = R(g.dy * g.dy), d2z = R(g.dz * g.dz);
        // |a_m x a_n|^2 of the rows a1 = d_x u, a2 = d_y u, a3 = d_z u
        VT c12a = dv_dx * dw_dy - dw_dx * dv_dy, c12b = dw_dx * du_dy - du_dx * dw_dy, c12c = du_dx * dv_dy - dv_dx * du_dy;
        VT c13a = dv_dx * dw_dz - dw_dx * dv_dz, c13b = dw_dx * du_dz - du_dx * dw_dz, c13c = du_dx * dv_dz - dv_dx * du_dz;
        VT c23a = dv_dy * dw_dz - dw_dy * dv_dz, c23b = dw_dy * du_dz - du_dy * dw_dz, c23c = du_dy * dv_dz - dv_dy * du_dz;
        VT x12 = c12a * c12a + c12b * c12b + c12c * c12c;
        VT x13 = c13a * c13a + c13b * c13b + c13c * c13c;
        VT x23 = c23a * c23a + c23b * c23b + c23c * c23c;
        VT Bb = VT(d2x * d2y) * x12 + VT(d2x * d2z) * x13 + VT(d2y * d2z) * x23;
        VT aa = du_dx * du_dx + du_dy * du_dy + du_dz * du_dz + dv_dx * dv_dx + dv_dy * dv_dy + dv_dz * dv_dz +
                dw_dx * dw_dx + dw_dy * dw_dy + dw_dz * dw_dz;
        return sqrt_ratio_or_zero(Bb, aa, R(g.sgs_cv));
    }
    VT S12 = R(0.5) * (du_dy + dv_dx), S13 = R(0.5) * (du_dz + dw_dx), S23 = R(0.5) * (dv_dz + dw_dy);
    VT S2 = R(2) * (du_dx * du_dx + dv_dy * dv_dy + dw_dz * dw_dz) + R(4) * (S12 * S12 + S13 * S13 + S23 * S23);
    return VT(coef * sqrt(S2));
}

// The anisotropic minimum-dissipation closure at one point (_amd_point,
// _amd_scalar_point and _amd_body!, src/operators/sgs_amd_vreman.jl:54-90,
// :204-212; Rozema et al. 2015, Abkar & Moin 2017), from g_ab = du_a/dx_b, the
// centred theta gradient t, the squared spacings d2, bg = g / theta0 and the
// Poincare constant C:
//   nu_t = C max(0, -(d_k du_i)(d_k du_j) S_ij + bg (d_k dw)(d_k dtheta) min(1, 1/Ri)) / du:du,
//   kappa_t = C max(0, -(d_k du_i)(d_k dtheta) dtheta_i) / |grad theta|^2,
// with (d_k da)(d_k db) = sum_k d2_k da_k db_k, Ri = |bg| |grad theta| / du:du,
// nu_t = 0 where du:du = 0 and kappa_t = nu_t / Pr_t where grad theta = 0.
template <class T>
struct NuKappa {
    T nu, ka;
};

// The Deardorff (1980) / Moeng (1984) coefficients of the TKE closure at
// cell (i, j, k) (TKEClosure: _coefficients_body!, tke_length_scale,
// tke_eddy_coefficients, src/PrognosticSGS.jl:93-110, :135-139, :432-454):
// N^2 = (g/theta0) (theta_face_above - theta_face_below) / dz with the faces
// the two-cell means (buoyancy_frequency_squared!,
// src/operators/stratification.jl:124-135), l = min(Delta, c_l sqrt(e) / N)
// where N^2 > 0 (else Delta), nu_t = c_k l sqrt(e), kappa_t = (1 + 2 l /
// Delta) nu_t; e of the committed step (the padded field g.tke).
template <typename R>
__device__ __forceinline__ NuKappa<R> tke_point(const Geo& g, int i, int j, int k, R tlo, R tc, R thi) {
    const R e = __ldg(static_cast<const R*>(g.tke) + pidx(g, i, j, k));
    const R N2 = R(g.tke_bg) * ((R(0.5) * (tc + thi)) - (R(0.5) * (tlo + tc))) * R(g.idz);
    const R D = R(g.tke_delta);
    const R sq = sqrt(fmax(e, R(0)));
    const R l = N2 > R(0) ? fmin(D, R(g.tke_cl) * sq / sqrt(N2)) : D;
    const R nu = R(g.tke_ck) * l * sq;
    return NuKappa<R>{nu, (R(1) + R(2) * l / D) * nu};
}

template <typename R>
__device__ __noinline__ NuKappa<R> amd_lane(R ux, R uy, R uz, R vx, R vy, R vz, R wx, R wy, R wz, R tx, R ty, R tz,
                                            R d2x, R d2y, R d2z, R bg, R C, R pr_t) {
    auto sdot = [&](R a1, R a2, R a3, R b1, R b2, R b3) { return d2x * a1 * b1 + d2y * a2 * b2 + d2z * a3 * b3; };
    const R S12 = R(0.5) * (uy + vx), S13 = R(0.5) * (uz + wx), S23 = R(0.5) * (vz + wy);
    const R P = sdot(ux, uy, uz, ux, uy, uz) * ux + sdot(vx, vy, vz, vx, vy, vz) * vy +
                sdot(wx, wy, wz, wx, wy, wz) * wz +
                R(2) * (sdot(ux, uy, uz, vx, vy, vz) * S12 + sdot(ux, uy, uz, wx, wy, wz) * S13 +
                        sdot(vx, vy, vz, wx, wy, wz) * S23);
    const R B = bg * sdot(wx, wy, wz, tx, ty, tz);
    const R D = ux * ux + uy * uy + uz * uz + vx * vx + vy * vy + vz * vz + wx * wx + wy * wy + wz * wz;
    const R kd = tx * tx + ty * ty + tz * tz;
    const R N2 = fabs(bg) * sqrt(kd);
    const R Bw = D >= N2 ? B : B * (D / N2);
    const R Q = sdot(ux, uy, uz, tx, ty, tz) * tx + sdot(vx, vy, vz, tx, ty, tz) * ty + sdot(wx, wy, wz, tx, ty, tz) * tz;
    const R nn = -P + Bw;
    NuKappa<R> o;
    o.nu = D > R(0) ? C * fmax(R(0), nn) / D : R(0);
    o.ka = kd > R(0) ? C * fmax(R(0), -Q) / kd : o.nu / pr_t;
    return o;
}

// the velocity gradient of smag_point and the theta gradient (centred over two
// cells, _scalar_gradient_at, src/operators/sgs_amd_vreman.jl:18-25) around
// the point at level k; uniform grids
template <typename R, bool UNI, class AU, class AV, class AW, class AT>
__device__ __forceinline__ auto amd_point(const Met<R, UNI>& m, const Geo& g, int k, R C, R bg, R pr_t, const AU& U,
                                          const AV& V, const AW& W, const AT& T) {
    using VT = decltype(U(0, 0, 0));
    const R idx = R(g.idx), idy = R(g.idy), idz = m.idz(k), ido = m.idz_off(k);
    VT du_dx = (U(1, 0, 0) - U(0, 0, 0)) * idx;
    VT dv_dy = (V(0, 1, 0) - V(0, 0, 0)) * idy;
    VT dw_dz = (W(0, 0, 1) - W(0, 0, 0)) * idz;
    VT du_dy = ((U(0, 1, 0) + U(1, 1, 0)) - (U(0, -1, 0) + U(1, -1, 0))) * (R(0.25) * idy);
    VT dv_dx = ((V(1, 0, 0) + V(1, 1, 0)) - (V(-1, 0, 0) + V(-1, 1, 0))) * (R(0.25) * idx);
    VT du_dz = ((U(0, 0, 1) + U(1, 0, 1)) - (U(0, 0, -1) + U(1, 0, -1))) * (R(0.25) * ido);
    VT dw_dx = ((W(1, 0, 0) + W(1, 0, 1)) - (W(-1, 0, 0) + W(-1, 0, 1))) * (R(0.25) * idx);
    VT dv_dz = ((V(0, 0, 1) + V(0, 1, 1)) - (V(0, 0, -1) + V(0, 1, -1))) * (R(0.25) * ido);
    VT dw_dy = ((W(0, 1, 0) + W(0, 1, 1)) - (W(0, -1, 0) + W(0, -1, 1))) * (R(0.25) * idy);
    VT tx = (T(1, 0, 0) - T(-1, 0, 0)) * (R(0.5) * idx);
    VT ty = (T(0, 1, 0) - T(0, -1, 0)) * (R(0.5) * idy);
    VT tz = (T(0, 0, 1) - T(0, 0, -1)) * (R(0.5) * idz);
    return amd_lane(VT(du_dx), VT(du_dy), VT(du_dz), VT(dv_dx), VT(dv_dy), VT(dv_dz), VT(dw_dx), VT(dw_dy), VT(dw_dz),
                    VT(tx), VT(ty), VT(tz), VT(R(g.dx * g.dx)), VT(R(g.dy * g.dy)), VT(R(g.dz * g.dz)), VT(bg), VT(C),
                    VT(pr_t));
}

// |S| = sqrt(2 S:S) from the velocity-gradient stencil of smag_point
// (_strain_at, src/Operators.jl:488-496), with the six strain components
template <typename R, bool UNI, class AU, class AV, class AW>
__device__ __forceinline__ auto strain_at(const Met<R, UNI>& m, const Geo& g, int k, const AU& U, const AV& V,
                                          const AW& W, decltype(U(0, 0, 0))* S6) {
    using VT = decltype(U(0, 0, 0));
    const R idx = R(g.idx), idy = R(g.idy), idz = m.idz(k), ido = m.idz_off(k);
    VT du_dx = (U(1, 0, 0) - U(0, 0, 0)) * idx;
    VT dv_dy = (V(0, 1, 0) - V(0, 0, 0)) * idy;
    VT dw_dz = (W(0, 0, 1) - W(0, 0, 0)) * idz;
    VT du_dy = ((U(0, 1, 0) + U(1, 1, 0)) - (U(0, -1, 0) + U(1, -1, 0))) * (R(0.25) * idy);
    VT dv_dx = ((V(1, 0, 0) + V(1, 1, 0)) - (V(-1, 0, 0) + V(-1, 1, 0))) * (R(0.25) * idx);
    VT du_dz = ((U(0, 0, 1) + U(1, 0, 1)) - (U(0, 0, -1) + U(1, 0, -1))) * (R(0.25) * ido);
    VT dw_dx = ((W(1, 0, 0) + W(1, 0, 1)) - (W(-1, 0, 0) + W(-1, 0, 1))) * (R(0.25) * idx);
    VT dv_dz = ((V(0, 0, 1) + V(0, 1, 1)) - (V(0, 0, -1) + V(0, 1, -1))) * (R(0.25) * ido);
    VT dw_dy = ((W(0, 1, 0) + W(0, 1, 1)) - (W(0, -1, 0) + W(0, -1, 1))) * (R(0.25) * idy);
    VT S12 = R(0.5) * (du_dy + dv_dx), S13 = R(0.5) * (du_dz + dw_dx), S23 = R(0.5) * (dv_dz + dw_dy);
    VT S2 = R(2) * (du_dx * du_dx + dv_dy * dv_dy + dw_dz * dw_dz) + R(4) * (S12 * S12 + S13 * S13 + S23 * S23);
    if (S6) {
        S6[0] = du_dx; S6[1] = dv_dy; S6[2] = dw_dz;
        S6[3] = S12; S6[4] = S13; S6[5] = S23;
    }
    return VT(sqrt(S2));
}

// The direct form: nut into a padded array (halos filled by a separate launch).
template <typename R, bool UNI>
__global__ void __launch_bounds__(256) smagorinsky_kernel(Geo g, const R* __restrict__ u, const R* __restrict__ v,
                                                          const R* __restrict__ w, const R* __restrict__ th,
                                                          R* __restrict__ nut, R c_s, R pr_t,
                                                          const double* __restrict__ cs2, double dd2,
                                                          const R* __restrict__ cs2f = nullptr) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int j = blockIdx.y * blockDim.y + threadIdx.y;
    int k = blockIdx.z * blockDim.z + threadIdx.z;
    if (i >= g.nx || j >= g.ny || k >= g.nz) return;
    const long long q = pidx(g, i, j, k);
    Nb<R> U{u + q, g.sy, g.sz}, V{v + q, g.sy, g.sz}, W{w + q, g.sy, g.sz};
    if (g.sgs_model == 4) {
        nut[q] = R(dyn_cs2_cell(g, cs2, cs2f, i, j, k) * dd2) * strain_at<R, UNI>(Met<R, UNI>(g), g, k, U, V, W, (R*)nullptr);
    } else if (g.sgs_model == 3) {
        Nb<R> T{th + q, g.sy, g.sz};
        const Met<R, UNI> m(g);
        nut[q] = amd_point<R, UNI>(m, g, k, c_s, m.lv(LV_BGC, k), pr_t, U, V, W, T).nu;
    } else if (g.sgs_model == 7) {
        nut[q] = tke_point<R>(g, i, j, k, th[q - g.sz], th[q], th[q + g.sz]).nu;
    } else {
        nut[q] = smag_point<R, UNI>(Met<R, UNI>(g), g, k, c_s, U, V, W);
    }
}
