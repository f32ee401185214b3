// aeo_ghost.cu -- ghost-cell wall reconstruction on cut-cell surfaces and the
// cut-cell wall model (include/aeolus_b200_ghost.h).
//
// The stencils (build_ghost_stencils, src/CutCell.jl:996-1172) come from the
// host; the per-step work is a gather over each stencil's eight donors:
//   reconstruct_wall_velocity! / reconstruct_wall_scalar!  src/CutCell.jl:1187-1266
//   wall_shear_stress (resolved)                           src/CutCell.jl:1268-1336
//   wall_shear_stress(..., law), wall_slip_velocity        src/wall_models/cutcell.jl:1-120
//   friction_velocity of SpaldingLaw, RoughLogLaw, MOSTWallLaw
//                                                          src/wall_models/laws.jl:72-284
// One thread per stencil.  A ghost target is never a donor (donors are fluid
// samples, targets are not), so the reconstruction has no race.
#include <cuda_runtime.h>
#include <float.h>
#include <math.h>

#include <algorithm>
#include <string>
#include <vector>

#include "../../include/aeolus_b200_ghost.h"

namespace {

std::string g_ghost_error;

// e^x - sum_{n<m} x^n/n! (m = 3 or 4) without the cancellation of the direct
// form at small x: the Taylor tail for |x| < 1/2 (_exp_tail,
// src/wall_models/laws.jl:108-121)
__device__ double exp_tail(double x, int m) {
    if (fabs(x) < 0.5) {
        double term = 1.0;
        for (int n = 1; n <= m; ++n) term *= x / n;   // x^m / m!
        double s = term;
        int n = m;
        while (fabs(term) > DBL_EPSILON * fabs(s) / 4 && n < m + 60) {
            ++n;
            term *= x / n;
            s += term;
        }
        return s;
    }
    const double s = expm1(x) - x - x * x / 2;
    return m == 3 ? s : s - x * x * x / 6;
}

// Spalding's y+ of u+ and its derivative (spalding_yplus, _spalding_dyplus)
__device__ double spalding_yplus(double kap, double B, double up) {
    return up + exp(-kap * B) * exp_tail(kap * up, 4);
}
__device__ double spalding_dyplus(double kap, double B, double up) {
    return 1.0 + kap * exp(-kap * B) * exp_tail(kap * up, 3);
}

// u_tau of Spalding's law: u+ y+(u+) = U h / nu by the safeguarded Newton of
// _increasing_root (a step leaving the bracket or a non-finite value bisects)
__device__ double spalding_utau(double kap, double B, double U, double h, double nu) {
    const double a = fabs(U);
    if (!(a > 0)) return 0.0;
    const double Re = a * h / nu;
    double lo = 0.0, hi = sqrt(Re);
    double x = hi;
    if (Re > 1) {
        x = 10.0;
        for (int it = 0; it < 3; ++it) x = fmax(log(Re / x) / kap + B, 1.0);
        x = fmin(x, hi);
    }
    for (int it = 0; it < 200; ++it) {
        const double y = spalding_yplus(kap, B, x);
        const double f = x * y - Re, gp = y + x * spalding_dyplus(kap, B, x);
        if (!isfinite(f) || f > 0) hi = x;
        else if (f < 0) lo = x;
        else break;
        double xn = (isfinite(f) && gp > 0) ? x - f / gp : (lo + hi) / 2;
        if (!(lo < xn && xn < hi)) xn = (lo + hi) / 2;
        if (fabs(xn - x) <= 2 * DBL_EPSILON * fabs(xn)) { x = xn; break; }
        x = xn;
    }
    return a / x;
}

// psi_m of the Businger-Dyer-Beljaars-Holtslag functions (src/SurfaceExchange.jl:189-225)
__device__ double psi_m_bdbh(double zeta) {
    if (zeta < 0) {
        const double x = pow(1.0 - 16.0 * zeta, 0.25);
        return 2 * log((1 + x) / 2) + log((1 + x * x) / 2) - 2 * atan(x) + M_PI / 2;
    }
    const double a = 1.0, b = 2.0 / 3.0, c = 5.0, d = 0.35;
    return -(a * zeta + b * (zeta - c / d) * exp(-d * zeta) + b * c / d);
}

// u_tau of the wall law `law` for the speed U at height h
__device__ double law_utau(int law, const double* p, double U, double h, double nu) {
    if (law == 1) return spalding_utau(p[0], p[1], U, h, nu);
    if (law == 2) return p[0] * fabs(U) / log(h / p[1]);
    // Monin-Obukhov: kappa max(U, U_min) / (ln(h/z0m) - psi_m(h/L) + psi_m(z0m/L))
    const double Ue = fmax(sqrt(U * U), p[3]);
    const double zeta = h / p[2];   // _Phi_m(sf, zeta, h, z0m), src/SurfaceExchange.jl:440
    const double phim = log(h / p[1]) - psi_m_bdbh(zeta) + psi_m_bdbh(zeta * p[1] / h);
    return p[0] * Ue / phim;
}

template <typename R>
__global__ void ghost_reconstruct_kernel(long long n, const long long* __restrict__ tgt,
                                         const long long* __restrict__ dnr, const double* __restrict__ w,
                                         const double* __restrict__ dn, const double* __restrict__ pr,
                                         const unsigned char* __restrict__ flags, R* f, int mode, double val,
                                         double kinv) {
    const long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n || (flags[s] & 3) != 3) return;
    double img = 0.0;
    for (int m = 0; m < 8; ++m) {
        const long long d = dnr[8 * s + m];
        if (d < 0) continue;
        img += w[8 * s + m] * (double)f[d];
    }
    const double out = mode == 0 ? val + (dn[s] / pr[s]) * (img - val) : img + (dn[s] - pr[s]) * (val * kinv);
    f[tgt[s]] = R(out);
}

// the aperture-weighted mean of a cell's two faces along one axis (_center_velocity)
__device__ double center(const double* __restrict__ f, const double* __restrict__ a, long long d, long long step,
                         bool has_next) {
    const double a1 = a[d], a2 = has_next ? a[d + step] : 0.0;
    const double s = a1 + a2;
    return s > 0 ? (a1 * f[d] + a2 * (has_next ? f[d + step] : 0.0)) / s : 0.0;
}

__global__ void ghost_wall_stress_kernel(long long n, int n1, int n2, int n3, const long long* __restrict__ dnr,
                                         const double* __restrict__ w, const double* __restrict__ pr,
                                         const double* __restrict__ nrm, const unsigned char* __restrict__ flags,
                                         const double* __restrict__ u, const double* __restrict__ v,
                                         const double* __restrict__ wv, const double* __restrict__ ax,
                                         const double* __restrict__ ay, const double* __restrict__ az, int law,
                                         const double* __restrict__ prm, double nu, double nu_eff,
                                         double* __restrict__ tau, double* __restrict__ slip) {
    const long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const bool valid = (flags[s] & 2) != 0;
    double p[5];
    for (int q = 0; q < 5; ++q) p[q] = prm[q];
    if (!valid) {
        tau[s] = 0.0;
        if (slip) slip[3 * s] = slip[3 * s + 1] = slip[3 * s + 2] = 0.0;
        return;
    }
    const long long pl = (long long)n1 * n2;
    double ui = 0.0, vi = 0.0, wi = 0.0;
    for (int m = 0; m < 8; ++m) {
        const long long d = dnr[8 * s + m];
        if (d < 0) continue;
        const int i = (int)(d % n1), j = (int)((d / n1) % n2), k = (int)(d / pl);
        const double wt = w[8 * s + m];
        ui += wt * center(u, ax, d, 1, i < n1 - 1);
        vi += wt * center(v, ay, d, n1, j < n2 - 1);
        wi += wt * center(wv, az, d, pl, k < n3 - 1);
    }
    const double nx = nrm[3 * s], ny = nrm[3 * s + 1], nz = nrm[3 * s + 2];
    const double un = ui * nx + vi * ny + wi * nz;
    const double h = pr[s];
    if (law == 0) {
        const double t2 = ui * ui + vi * vi + wi * wi - un * un;
        tau[s] = nu * sqrt(fmax(t2, 0.0)) / h;
        if (slip) slip[3 * s] = slip[3 * s + 1] = slip[3 * s + 2] = 0.0;
        return;
    }
    const double t0 = ui - un * nx, t1 = vi - un * ny, t2 = wi - un * nz;
    const double ut = sqrt(t0 * t0 + t1 * t1 + t2 * t2);
    const double ut_law = law_utau(law, p, ut, h, nu);
    const double ts = ut_law * ut_law;
    tau[s] = ts;
    if (slip) {
        double r = 0.0;
        if (ut != 0.0) r = (ut - ts * h / nu_eff) / ut;
        slip[3 * s] = r * t0;
        slip[3 * s + 1] = r * t1;
        slip[3 * s + 2] = r * t2;
    }
}

}  // namespace

struct aeo_ghost {
    int dev = 0;
    int n1 = 0, n2 = 0, n3 = 0;
    long long n = 0;
    long long* tgt = nullptr;
    long long* dnr = nullptr;
    double *w = nullptr, *dn = nullptr, *pr = nullptr, *nrm = nullptr, *prm = nullptr;
    unsigned char* flags = nullptr;
    double min_probe = INFINITY;   // over the valid stencils
    std::string err;
};

#define GCK(call)                                                                       \
    do {                                                                                \
        cudaError_t e_ = (call);                                                        \
        if (e_ != cudaSuccess) {                                                        \
            h->err = std::string(#call) + ": " + cudaGetErrorString(e_);                \
            return AEO_ERR_CUDA;                                                        \
        }                                                                               \
    } while (0)

namespace {

template <typename T>
aeo_status upload(aeo_ghost* h, T** dst, const T* src, size_t count) {
    GCK(cudaMalloc(dst, std::max<size_t>(count, 1) * sizeof(T)));
    if (count) GCK(cudaMemcpy(*dst, src, count * sizeof(T), cudaMemcpyHostToDevice));
    return AEO_OK;
}

void release(aeo_ghost* h) {
    cudaFree(h->tgt); cudaFree(h->dnr); cudaFree(h->w); cudaFree(h->dn); cudaFree(h->pr); cudaFree(h->nrm);
    cudaFree(h->flags); cudaFree(h->prm);
}

// the law's parameters checked on the host (the reference throws there)
aeo_status check_law(aeo_ghost* h, int law, const double* p, double nu, double nu_eff) {
    if (law < 0 || law > 3) { h->err = "unknown wall law"; return AEO_ERR_ARGUMENT; }
    if (law == 0 && !(nu >= 0)) { h->err = "the resolved wall stress needs nu >= 0"; return AEO_ERR_ARGUMENT; }
    if (law == 1 && !(nu > 0)) { h->err = "SpaldingLaw: the kinematic viscosity nu is required"; return AEO_ERR_ARGUMENT; }
    if (law >= 1 && !(nu_eff > 0)) { h->err = "wall_slip_velocity: nu_eff (or nu) is required"; return AEO_ERR_ARGUMENT; }
    if (law >= 1 && !p) { h->err = "the wall law needs its parameters"; return AEO_ERR_ARGUMENT; }
    if ((law == 2 || law == 3) && !(h->min_probe > p[1])) {
        h->err = "the rough-wall laws need every probe height above z0";
        return AEO_ERR_ARGUMENT;
    }
    return AEO_OK;
}

}  // namespace

extern "C" {

aeo_status aeo_ghost_create(int32_t nx_s, int32_t ny_s, int32_t nz_s, int64_t n, const int64_t* target,
                            const int64_t* donors, const double* weights, const double* dn, const double* probe,
                            const double* normal, const uint8_t* flags, int32_t device, aeo_ghost** out) {
    if (!out || nx_s < 1 || ny_s < 1 || nz_s < 1 || n < 0 ||
        (n > 0 && (!target || !donors || !weights || !dn || !probe || !normal || !flags))) {
        g_ghost_error = "aeo_ghost_create: bad arguments";
        return AEO_ERR_ARGUMENT;
    }
    const long long total = (long long)nx_s * ny_s * nz_s;
    for (int64_t s = 0; s < n; ++s) {
        if (target[s] < 0 || target[s] >= total) { g_ghost_error = "aeo_ghost_create: target out of range"; return AEO_ERR_ARGUMENT; }
        for (int m = 0; m < 8; ++m)
            if (donors[8 * s + m] < -1 || donors[8 * s + m] >= total) {
                g_ghost_error = "aeo_ghost_create: donor out of range";
                return AEO_ERR_ARGUMENT;
            }
        if (!(probe[s] > 0)) { g_ghost_error = "aeo_ghost_create: probe distances must be positive"; return AEO_ERR_ARGUMENT; }
    }
    aeo_ghost* h = new aeo_ghost;
    h->dev = device; h->n1 = nx_s; h->n2 = ny_s; h->n3 = nz_s; h->n = n;
    for (int64_t s = 0; s < n; ++s)
        if (flags[s] & 2) h->min_probe = std::min(h->min_probe, probe[s]);
    aeo_status st = AEO_OK;
    if (cudaSetDevice(device) != cudaSuccess) { g_ghost_error = "aeo_ghost_create: cudaSetDevice failed"; delete h; return AEO_ERR_CUDA; }
    static_assert(sizeof(long long) == sizeof(int64_t), "flat indices are 64-bit");
    if (!st) st = upload(h, &h->tgt, reinterpret_cast<const long long*>(target), (size_t)n);
    if (!st) st = upload(h, &h->dnr, reinterpret_cast<const long long*>(donors), 8 * (size_t)n);
    if (!st) st = upload(h, &h->w, weights, 8 * (size_t)n);
    if (!st) st = upload(h, &h->dn, dn, (size_t)n);
    if (!st) st = upload(h, &h->pr, probe, (size_t)n);
    if (!st) st = upload(h, &h->nrm, normal, 3 * (size_t)n);
    if (!st) st = upload(h, &h->flags, reinterpret_cast<const unsigned char*>(flags), (size_t)n);
    const double zero[5] = {0, 0, 0, 0, 0};
    if (!st) st = upload(h, &h->prm, zero, 5);
    if (st) {
        g_ghost_error = h->err;
        release(h);
        delete h;
        return st;
    }
    *out = h;
    return AEO_OK;
}

aeo_status aeo_ghost_destroy(aeo_ghost* h) {
    if (!h) return AEO_OK;
    cudaSetDevice(h->dev);
    release(h);
    delete h;
    return AEO_OK;
}

aeo_status aeo_ghost_reconstruct(aeo_ghost* h, void* field, int32_t fp32, int32_t mode, double value, double kappa,
                                 void* stream) {
    if (!h) return AEO_ERR_ARGUMENT;
    if (!field || (mode != 0 && mode != 1) || (mode == 1 && !(kappa != 0.0))) {
        h->err = "aeo_ghost_reconstruct: a field, mode 0 (Dirichlet) or 1 (Neumann, kappa != 0)";
        return AEO_ERR_ARGUMENT;
    }
    GCK(cudaSetDevice(h->dev));
    if (h->n == 0) return AEO_OK;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    const unsigned nb = (unsigned)((h->n + 255) / 256);
    const double kinv = mode == 1 ? 1.0 / kappa : 0.0;
    if (fp32)
        ghost_reconstruct_kernel<float><<<nb, 256, 0, st>>>(h->n, h->tgt, h->dnr, h->w, h->dn, h->pr, h->flags,
                                                             static_cast<float*>(field), mode, value, kinv);
    else
        ghost_reconstruct_kernel<double><<<nb, 256, 0, st>>>(h->n, h->tgt, h->dnr, h->w, h->dn, h->pr, h->flags,
                                                              static_cast<double*>(field), mode, value, kinv);
    GCK(cudaGetLastError());
    return AEO_OK;
}

aeo_status aeo_ghost_reconstruct_host(aeo_ghost* h, double* field, int32_t mode, double value, double kappa) {
    if (!h) return AEO_ERR_ARGUMENT;
    if (!field) { h->err = "aeo_ghost_reconstruct_host: NULL field"; return AEO_ERR_ARGUMENT; }
    GCK(cudaSetDevice(h->dev));
    const size_t bytes = (size_t)h->n1 * h->n2 * h->n3 * sizeof(double);
    double* d = nullptr;
    GCK(cudaMalloc(&d, bytes));
    aeo_status st = AEO_OK;
    if (cudaMemcpy(d, field, bytes, cudaMemcpyHostToDevice) != cudaSuccess) { h->err = "copy in"; st = AEO_ERR_CUDA; }
    if (!st) st = aeo_ghost_reconstruct(h, d, 0, mode, value, kappa, nullptr);
    if (!st && cudaMemcpy(field, d, bytes, cudaMemcpyDeviceToHost) != cudaSuccess) { h->err = "copy out"; st = AEO_ERR_CUDA; }
    cudaFree(d);
    return st;
}

aeo_status aeo_ghost_wall_stress(aeo_ghost* h, const double* u, const double* v, const double* w, const double* ax,
                                 const double* ay, const double* az, int32_t law, const double* params, double nu,
                                 double nu_eff, double* tau, double* slip, void* stream) {
    if (!h) return AEO_ERR_ARGUMENT;
    if (!u || !v || !w || !ax || !ay || !az || !tau) { h->err = "aeo_ghost_wall_stress: NULL array"; return AEO_ERR_ARGUMENT; }
    // the parameters are read on the host for the checks, then copied to the device
    double p[5] = {0, 0, 0, 0, 0};
    if (params) for (int q = 0; q < 5; ++q) p[q] = params[q];
    if (aeo_status e = check_law(h, law, params ? p : nullptr, nu, nu_eff)) return e;
    GCK(cudaSetDevice(h->dev));
    if (h->n == 0) return AEO_OK;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    GCK(cudaMemcpyAsync(h->prm, p, sizeof(p), cudaMemcpyHostToDevice, st));
    const unsigned nb = (unsigned)((h->n + 255) / 256);
    ghost_wall_stress_kernel<<<nb, 256, 0, st>>>(h->n, h->n1, h->n2, h->n3, h->dnr, h->w, h->pr, h->nrm, h->flags, u,
                                                v, w, ax, ay, az, law, h->prm, nu, nu_eff, tau, slip);
    GCK(cudaGetLastError());
    GCK(cudaStreamSynchronize(st));   // the parameter copy is from the stack
    return AEO_OK;
}

aeo_status aeo_ghost_wall_stress_host(aeo_ghost* h, const double* u, const double* v, const double* w,
                                      const double* ax, const double* ay, const double* az, int32_t law,
                                      const double* params, double nu, double nu_eff, double* tau, double* slip) {
    if (!h) return AEO_ERR_ARGUMENT;
    if (!u || !v || !w || !ax || !ay || !az || !tau) { h->err = "aeo_ghost_wall_stress_host: NULL array"; return AEO_ERR_ARGUMENT; }
    GCK(cudaSetDevice(h->dev));
    const size_t cells = (size_t)h->n1 * h->n2 * h->n3;
    const double* src[6] = {u, v, w, ax, ay, az};
    double* d[6] = {};
    double *dt = nullptr, *ds = nullptr;
    aeo_status st = AEO_OK;
    for (int a = 0; a < 6 && !st; ++a) {
        if (cudaMalloc(&d[a], cells * sizeof(double)) != cudaSuccess ||
            cudaMemcpy(d[a], src[a], cells * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess) {
            h->err = "aeo_ghost_wall_stress_host: copy in";
            st = AEO_ERR_CUDA;
        }
    }
    const size_t n = (size_t)std::max<long long>(h->n, 1);
    if (!st && (cudaMalloc(&dt, n * sizeof(double)) != cudaSuccess ||
                (slip && cudaMalloc(&ds, 3 * n * sizeof(double)) != cudaSuccess))) {
        h->err = "aeo_ghost_wall_stress_host: cudaMalloc";
        st = AEO_ERR_CUDA;
    }
    if (!st) st = aeo_ghost_wall_stress(h, d[0], d[1], d[2], d[3], d[4], d[5], law, params, nu, nu_eff, dt, ds, nullptr);
    if (!st && h->n > 0) {
        if (cudaMemcpy(tau, dt, (size_t)h->n * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess ||
            (slip && cudaMemcpy(slip, ds, 3 * (size_t)h->n * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)) {
            h->err = "aeo_ghost_wall_stress_host: copy out";
            st = AEO_ERR_CUDA;
        }
    }
    for (auto* p : d) cudaFree(p);
    cudaFree(dt);
    cudaFree(ds);
    return st;
}

const char* aeo_ghost_last_error(const aeo_ghost* h) { return h ? h->err.c_str() : g_ghost_error.c_str(); }

}  // extern "C"
