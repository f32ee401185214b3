// aeo_common.cuh -- layouts, metrics and small helpers shared by the kernels.
//
// Device layout.  The stencil inputs (the stage states u, v, w, theta and the
// eddy viscosity) live in PADDED arrays: interior (nx, ny, nz) plus a halo of
// AEO_H = 3 cells in y and z and an x offset of AEO_HX = 8 cells, so that
// each interior row starts on a 32-byte sector for fp32 and fp64.  Index
//   q(i, j, k) = (i + AEO_HX) + px * ((j + AEO_H) + py * (k + AEO_H)),
//   px = nx + 2*AEO_HX, py = ny + 2*AEO_H,
// with (i, j, k) interior coordinates that may step into the halo.  Halos hold
// the values the reference's fill_halos! puts there
// (src/boundary_conditions/halo_kernels.jl:100-140, x then y then z).
// Everything else (predictor velocities, the potential, pressure, the
// Poisson source) is interior-only, q = i + nx*(j + ny*k); kernels that read
// its neighbours apply the boundary maps themselves.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#define AEO_HX 8
#define AEO_H 3
#define AEO_LH 4   // offset of level k in the per-level metric vectors

enum { LOC_C = 0, LOC_FX = 1, LOC_FY = 2, LOC_FZ = 3 };

template <typename R>
struct cplx {
    R x, y;
};

template <typename R>
__device__ __forceinline__ cplx<R> cmk(R a, R b) {
    cplx<R> c;
    c.x = a;
    c.y = b;
    return c;
}
template <typename R>
__device__ __forceinline__ cplx<R> cadd(cplx<R> a, cplx<R> b) { return cmk<R>(a.x + b.x, a.y + b.y); }
template <typename R>
__device__ __forceinline__ cplx<R> csub(cplx<R> a, cplx<R> b) { return cmk<R>(a.x - b.x, a.y - b.y); }
template <typename R>
__device__ __forceinline__ cplx<R> cmul(cplx<R> a, cplx<R> b) {
    return cmk<R>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename R>
__device__ __forceinline__ cplx<R> cconj(cplx<R> a) { return cmk<R>(a.x, -a.y); }

// The RK3 stage combination c(x, s) = ca*s + cb*x (_Lin2r,
// src/Simulations.jl:1194-1198).  FP64 evaluates it as written, as the
// reference does.  FP32 evaluates x + ca*(s - x), whose two weights sum to
// one exactly: with ca = fl(1/3) and cb = fl(2/3) the written form's weights
// sum to 1 + 3.0e-8, which scales every field by that factor once per step
// (a kinetic-energy drift of 6e-8 per step, the size of a whole step's
// physical decay in a weakly dissipative flow).
template <typename R>
__device__ __forceinline__ R rk_combine(R ca, R cb, R s, R x) {
    if constexpr (sizeof(R) == 4) return fmaf(ca, s - x, x);
    else return ca * s + cb * x;
}

// Geometry of one domain, passed by value to every kernel.
struct Geo {
    int nx, ny, nz;
    int px, py;            // padded row / plane extents
    long long sy, sz;      // padded strides of j and k
    long long nin;         // nx*ny*nz
    int bc_z;              // 0 periodic, 1 wall
    int ox, oy;            // open x / y faces (aeo_set_open): fields without planes take the mirror there
    int uniform;           // 1: uniform z metrics
    double dx, dy, dz;
    double idx, idy, idx2, idy2, idz, idz2, delta_u;
    // per-level vectors, entry (k + AEO_LH) for level k (interior 0-based)
    const double* idzc;
    const double* idzf;
    const double* idz_off;
    const double* wlo;
    const double* whi;
    const double* alo;
    const double* ahi;
    const double* delta;
    const double* zc;
    const double* zf;
    // sound-proof weights (NULL for the Boussinesq core), same indexing
    const double* wc;
    const double* wf;
    const double* thf;
    // the per-level factors in the working precision (rows LV_*, entry k + AEO_LH)
    const void* lvr;
    int lvn;   // row stride
    // the SGS closure when c_s > 0: 0 Smagorinsky, 1 Vreman (coefficient 2.5 c_s^2)
    int sgs_model;
    double sgs_cv;
    // the TKE closure (sgs_model 7): its e (padded, working precision, halos
    // filled), c_k, c_l, Delta = (dx dy dz)^(1/3), g / theta0 (0 without
    // buoyancy)
    const void* tke;
    double tke_ck, tke_cl, tke_delta, tke_bg;
};

// The cell whose value a closure field takes at (i, j) on open faces: the
// zero-gradient mirror of the reference's halo fill
// (src/boundary_conditions/open_boundary.jl:54-58) across an open x or y face.
__device__ __forceinline__ int open_src(int open, int i, int n) {
    if (!open) return i;
    return i < 0 ? -1 - i : (i >= n ? 2 * n - 1 - i : i);
}

__device__ __forceinline__ long long pidx(const Geo& g, int i, int j, int k) {
    return (long long)(i + AEO_HX) + (long long)(j + AEO_H) * g.sy + (long long)(k + AEO_H) * g.sz;
}
__device__ __forceinline__ long long iidx(const Geo& g, int i, int j, int k) {
    return (long long)i + (long long)g.nx * ((long long)j + (long long)g.ny * (long long)k);
}
__device__ __forceinline__ double lvl(const double* a, int k) { return __ldg(a + k + AEO_LH); }

__device__ __forceinline__ int wrapi(int i, int n) {
    i %= n;
    return i < 0 ? i + n : i;
}

// The composite boundary map of the reference's halo fill for a point that
// may lie outside the interior: periodic wrap in x and y; in z periodic wrap,
// or for an ImpermeableWall the mirror (cell-centred and horizontal-face
// fields) or the odd extension about the zero wall faces (w).  Returns the
// multiplier: 1, -1 or 0 (the wall face itself).
__device__ __forceinline__ int zmap(const Geo& g, int k, int loc, int* kk) {
    if (g.bc_z == 0) {
        *kk = wrapi(k, g.nz);
        return 1;
    }
    if (loc != LOC_FZ) {
        if (k < 0) k = -k - 1;
        else if (k >= g.nz) k = 2 * g.nz - 1 - k;
        *kk = k;
        return 1;
    }
    if (k == 0 || k == g.nz) {
        *kk = 0;
        return 0;
    }
    if (k < 0) {
        *kk = -k;
        return -1;
    }
    if (k > g.nz) {
        *kk = 2 * g.nz - k;
        return -1;
    }
    *kk = k;
    return 1;
}

template <typename R>
__device__ __forceinline__ R ld_mapped_interior(const Geo& g, const R* __restrict__ a, int i, int j, int k, int loc) {
    int kk;
    int s = zmap(g, k, loc, &kk);
    if (s == 0) return R(0);
    R v = __ldg(a + iidx(g, wrapi(i, g.nx), wrapi(j, g.ny), kk));
    return s > 0 ? v : -v;
}

// ---- metric accessors (src/FiniteVolume.jl:146-186) -----------------------
// Per-level factors in the working precision: row f holds the factor of level
// k at entry k + AEO_LH.  The engine builds the rows once from its FP64
// metric vectors (the reciprocals and g/theta_f rounded exactly as the
// division in R would round them; the sponge rates from the profile), so a
// kernel reads each factor with one load instead of an FP64 load, a
// conversion and, for the reciprocals, a division per point.
enum {
    LV_IDZC = 0, LV_IDZF, LV_IDZOFF, LV_WLO, LV_WHI, LV_ALO, LV_AHI, LV_DELTA,
    LV_WC, LV_WF, LV_IWC, LV_IWF, LV_THF, LV_GTHF, LV_SPC, LV_SPF,
    LV_BGC,   // the AMD closure's buoyancy parameter of the level: g/theta0, or g/theta_bar(z_k) (sound-proof core)
    LV_N
};

template <typename R, bool UNI>
struct Met {
    const Geo& g;
    const R* t;        // row f, level k at t[f * stride + k + off]
    int stride, off;
    __device__ __forceinline__ explicit Met(const Geo& gg)
        : g(gg), t(static_cast<const R*>(gg.lvr)), stride(gg.lvn), off(AEO_LH) {}
    __device__ __forceinline__ Met(const Geo& gg, const R* tab, int s, int o) : g(gg), t(tab), stride(s), off(o) {}
    __device__ __forceinline__ R lv(int f, int k) const { return t[f * stride + k + off]; }
    __device__ __forceinline__ R idz(int k) const { return UNI ? R(g.idz) : lv(LV_IDZC, k); }
    __device__ __forceinline__ R idzf(int k) const { return UNI ? R(g.idz) : lv(LV_IDZF, k); }
    __device__ __forceinline__ R idz_off(int k) const { return UNI ? R(g.idz) : lv(LV_IDZOFF, k); }
    // the mixing helpers take the value type of the caller: R, or a pair of
    // FP32 lanes (the factors broadcast)
    template <typename V>
    __device__ __forceinline__ V zface(int k, V lo, V hi) const {
        if constexpr (UNI) return V(R(0.5)) * (lo + hi);
        else return V(lv(LV_WLO, k)) * lo + V(lv(LV_WHI, k)) * hi;
    }
    template <typename V>
    __device__ __forceinline__ V zflux(int k, V lo, V hi) const {
        if constexpr (UNI) return V(R(0.5)) * (lo + hi);
        else return V(lv(LV_ALO, k)) * lo + V(lv(LV_AHI, k)) * hi;
    }
    template <typename V>
    __device__ __forceinline__ V lapz(int loc, int k, V fm, V c, V fp) const {
        if constexpr (UNI) {
            return (fp - V(R(2)) * c + fm) * V(R(g.idz2));
        } else {
            if (loc == LOC_FZ) return ((fp - c) * V(lv(LV_IDZC, k)) - (c - fm) * V(lv(LV_IDZC, k - 1))) * V(lv(LV_IDZF, k));
            return ((fp - c) * V(lv(LV_IDZF, k + 1)) - (c - fm) * V(lv(LV_IDZF, k))) * V(lv(LV_IDZC, k));
        }
    }
    __device__ __forceinline__ R filter(int k) const { return UNI ? R(g.delta_u) : lv(LV_DELTA, k); }
    // sound-proof weights
    __device__ __forceinline__ R wc(int k) const { return lv(LV_WC, k); }
    __device__ __forceinline__ R wf(int k) const { return lv(LV_WF, k); }
    __device__ __forceinline__ R iwc(int k) const { return lv(LV_IWC, k); }
    __device__ __forceinline__ R iwf(int k) const { return lv(LV_IWF, k); }
    __device__ __forceinline__ R thf(int k) const { return lv(LV_THF, k); }
    __device__ __forceinline__ R gthf(int k) const { return lv(LV_GTHF, k); }
    // Rayleigh sponge rates at the centre and the bottom face of level k
    __device__ __forceinline__ R spc(int k) const { return lv(LV_SPC, k); }
    __device__ __forceinline__ R spf(int k) const { return lv(LV_SPF, k); }
};

// N = 16 / sizeof(R) consecutive values as one 16-byte access (the caller
// guarantees 16-byte alignment: an x-offset that is a multiple of N in an
// array whose rows hold a multiple of N values).
template <typename R>
struct Vec16 {
    static constexpr int N = 16 / (int)sizeof(R);
};
__device__ __forceinline__ void vld(const float* p, float (&v)[4]) {
    const float4 t = *reinterpret_cast<const float4*>(p);
    v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
}
__device__ __forceinline__ void vld(const double* p, double (&v)[2]) {
    const double2 t = *reinterpret_cast<const double2*>(p);
    v[0] = t.x; v[1] = t.y;
}
__device__ __forceinline__ void vst(float* p, const float (&v)[4]) {
    *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
}
__device__ __forceinline__ void vst(double* p, const double (&v)[2]) {
    *reinterpret_cast<double2*>(p) = make_double2(v[0], v[1]);
}

#define AEO_CHECK_LAUNCH() ((void)0)
