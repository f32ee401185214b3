// aeolus_b200.cu -- libaeolus_b200.so: the C-ABI of include/aeolus_b200.h and
// the per-domain orchestration of the projected SSP-RK3 step on one B200.
//
// One substage (src/Simulations.jl:531-650; src/Anelastic.jl:1791-1876):
//   sweep           tendencies (in-tile Smagorinsky) + predictor u* + theta
//   div, src_fftx   divergence of u* (into phi's storage), r2c transform along x
//   ffty            forward transform along y
//   fftz_solve      periodic z: forward, 1/lambda, inverse   | thomas: walls in z
//   ffty            inverse along y
//   ifftx           c2r along x -> phi
//   correct         u = c(u* - grad phi, u^n), p = phi/dt
//   halo            halos of u, v, w, theta for the next substage
//
// State lives in four padded sets.  A step reads set `cur` (u^n), writes the
// stages into sets 2 and 3 and the result into set cur^1, so u^n stays
// untouched until the step is accepted: the snapshot/retry of the adaptive
// step costs nothing.  dt lives in device memory (StepScalars), written by the
// host for fixed steps or by the on-device CFL pick for adaptive ones, so
// each step is one CUDA graph (one per parity of `cur`, with or without the
// pick) that is captured once and replayed.
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/aeolus_b200.h"
#include "aeo_adapt.cuh"
#include "aeo_mg_internal.h"
#include "aeo_common.cuh"
#include "aeo_cutcell.cuh"
#include "aeo_positive.cuh"
#include "aeo_fft.cuh"
#include "aeo_init.cuh"
#include "aeo_misc.cuh"
#include "aeo_sweep.cuh"
#include "aeo_tke.cuh"
#include "aeo_sweep_pair.cuh"
#include "aeo_sweep_wpair.cuh"

// A transform kernel at a compile-time length 2^LG (128, 256 or 512 points:
// the lines fill the CTA's 2048 points) or its general form (LG = 0).
#define AEO_FFT_LEN(L, CALL)                                  \
    switch (L) {                                              \
        case 7: { constexpr int LG = 7; CALL; } break;        \
        case 8: { constexpr int LG = 8; CALL; } break;        \
        case 9: { constexpr int LG = 9; CALL; } break;        \
        default: { constexpr int LG = 0; CALL; } break;       \
    }
static inline int ilog2i(int n) { int l = 0; while ((1 << (l + 1)) <= n) ++l; return l; }
#include "aeo_sweep_tile.cuh"

static std::string g_create_error;

// The message aeo_last_error(NULL) returns (also set by handle-free entry points).
void aeo_set_global_error(const std::string& m) { g_create_error = m; }

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

static bool is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }
static int next_pow2(int n) {
    int p = 1;
    while (p < n) p <<= 1;
    return p;
}

struct CoreBase {
    aeo_config cfg{};
    std::string err;
    cudaStream_t st = nullptr;
    Geo g{};
    int launches = 0;
    virtual ~CoreBase() {}
    // kernels of one RK3 step (solver = PCG: with the last solve's iteration count)
    virtual int step_launches() { return launches; }
    void fail(const std::string& m) { err = m; }
    virtual aeo_status init(const double* zf, const double* wc, const double* wf, const double* thf) = 0;
    virtual aeo_status set_field(int id, const double* host) = 0;
    virtual aeo_status get_field(int id, double* host) = 0;
    virtual aeo_status set_field_f32(int id, const float* host) = 0;
    virtual aeo_status get_field_f32(int id, float* host) = 0;
    virtual aeo_status step_rk3(double dt, int n, bool sync) = 0;
    virtual aeo_status step_euler(double dt, int n) = 0;
    virtual aeo_status step_adaptive(const aeo_cfl* c, int n, double* dt_prev, aeo_adaptive_stats* stats) = 0;
    virtual aeo_status cfl(const aeo_cfl* c, double dt_prev, aeo_adaptive_stats* stats) = 0;
    virtual aeo_status pressure_solve(const double* src, double* phi) = 0;
    virtual aeo_status advect_positive(const void* u, const void* v, const void* w, const void* phi, void* tend,
                                       double dt, int scheme, int accumulate, bool host) = 0;
    virtual aeo_status kinetic_energy(double* out) = 0;
    virtual aeo_status max_divergence(double* out) = 0;
    virtual aeo_status fill_uniform(int id, uint64_t seed, uint32_t stream, double amp, int mode) = 0;
    virtual aeo_status project() = 0;
    virtual aeo_status profile_step(double dt, double* ms, int ncls) = 0;
    virtual aeo_status init_isotropic(double u_rms, double k_peak, uint64_t seed, double kmax, int proj,
                                      double target_rms) = 0;
    virtual aeo_status set_pcg(const double* ax, const double* ay, const double* az, double tol, int maxit) = 0;
    virtual aeo_status pcg_stats(aeo_mg_stats* o) = 0;
    virtual aeo_status pcg_set_learned(aeo_unet* net, double stagnation) = 0;
    virtual aeo_status pcg_harvest(int cap, double* b, double* x, double* rh, double* xh, int* count) = 0;
    virtual aeo_status set_open(int ox, int oy, const double* xp, const double* yp, const int* modes) = 0;
    virtual aeo_status set_open_outflow(const int* rad, int corr, const double* xd, const double* yd, const double* xw,
                                        const double* yw) = 0;
    virtual aeo_status open_ledger(double* out) = 0;
    virtual aeo_status get_open_planes(double* xp, double* yp) = 0;
    virtual aeo_status open_state(double* hx, double* hy, double* sc, bool set) = 0;
    virtual aeo_status set_open_planes(const double* xp, const double* yp) = 0;
    virtual aeo_status set_ibm(const uint8_t* mask, double tau) = 0;
    virtual aeo_status set_sgs_buoyancy(const double* bg) = 0;
    virtual aeo_status set_lagrangian(double c0, double theta, double memory_time) = 0;
    virtual aeo_status get_sgs_state(double* out) = 0;
    virtual aeo_status set_sgs_state(const double* in) = 0;
    virtual aeo_status set_tke(double c_eps0, double c_eps1, double c_l, int exact) = 0;
};

struct aeo_sim {
    CoreBase* core;
};

template <typename R>
struct Core : CoreBase {
    std::vector<void*> allocs;
    double* levels = nullptr;  // metric vectors
    R* levels_r = nullptr;     // per-level factors in the working precision (rows LV_*)
    double *kx2 = nullptr, *ky2 = nullptr, *kz2 = nullptr;
    double* colc = nullptr;    // column coefficients
    ColumnCoef cc{};
    R* P[4][4] = {};           // padded state sets (u, v, w, theta)
    // theta is held as theta - th_off: the reference value (theta0, or the
    // anelastic theta_f at the surface) in FP32, so the stored numbers are the
    // few-kelvin deviations and keep FP32's relative precision; 0 in FP64
    double th_off = 0.0;
    TileMaps tmaps[4];         // TMA maps of the padded sets
    bool pair = false;         // FP32 centred: the paired sweep (64-cell tiles, 72-wide plane boxes)
    int cur = 0;               // the set holding the state (0 or 1)
    R* Q[3] = {};              // predictor (interior)
    R* nut = nullptr;          // padded, diagnostics only
    R* phi = nullptr;          // interior
    R* pres = nullptr;         // interior
    cplx<R>* S = nullptr;      // spectrum
    double* cps = nullptr;     // the column solve's c' scratch (spectrum layout)
    cplx<R>* tw = nullptr;
    int NT = 0;
    // solver = AEO_SOLVER_PCG: the MG-PCG handle (a^2 faces), its device rhs and
    // solution, and the face apertures (aeo_cutcell.cuh)
    bool pcg = false;
    aeo_mg* mg = nullptr;
    double *mg_b = nullptr, *mg_x = nullptr;
    R *apx = nullptr, *apy = nullptr, *apz = nullptr;
    double pcg_tol = 1e-8;
    bool pcg_learned = false;
    std::vector<double> h_ap[3];   // the apertures the PCG operator was built from
    // open lateral faces (aeo_set_open): plane buffers and boundary-face values
    bool open_x = false, open_y = false;
    bool ob_rad = false;           // a radiating (:convective) open face
    OpenSet<R> ob{};
    int pcg_maxit = 200;
    double* d_stage = nullptr; // host-layout staging (device)
    long long host_n = 0;
    double* d_part = nullptr;  // per-level partials (4 per level)
    int* d_flag = nullptr;
    StepScalars* d_sc = nullptr;
    int rows_x = 1, tpx_y = 1, tpx_z = 1;
    int kchunk = 32;
    int wchunk = 32;         // levels a CTA of the paired WENO sweep marches
    int fin_per_sm = 4;      // resident CTAs of the finite check an SM
    int nsm = 148;           // SMs of the device (the persistent sweep's grid)
    // interior column metrics and weights on the host (the PCG operator's coefficients):
    // dz_c per level, dz_f per face, W_c, W_f (1 on the Boussinesq core)
    std::vector<double> h_dzc, h_dzf, h_wc, h_wf;
    double dz_min = 0.0;
    cudaGraphExec_t gexec[2][2] = {};   // [with CFL pick][parity of cur]
    // n steps as one launch: a WHILE node over pairs of steps [parity of cur],
    // its body captured on st_loop, the pair count in d_steps
    cudaGraphExec_t gmulti[2] = {};
    cudaStream_t st_loop = nullptr;
    int* d_steps = nullptr;
    CflParams cflp{};
    bool cflp_set = false;
    bool uni = true, sgs = false, anel = false;
    bool amd() const { return sgs && cfg.sgs_model == AEO_SGS_AMD; }
    bool dyn() const { return sgs && (cfg.sgs_model == AEO_SGS_DYNAMIC || cfg.sgs_model == AEO_SGS_DYNAMIC_LOCAL); }
    bool dyn_local() const { return sgs && cfg.sgs_model == AEO_SGS_DYNAMIC_LOCAL; }
    bool lag() const { return sgs && cfg.sgs_model == AEO_SGS_LAGRANGIAN; }
    bool tke() const { return sgs && cfg.sgs_model == AEO_SGS_TKE; }
    // the closures whose kappa_t is their own (the sweeps' kappa_t planes)
    bool own_kappa() const { return amd() || tke(); }
    // the sweeps' dynamic coefficient (per level, or per cell in cs2f)
    bool dyncl() const { return dyn() || lag(); }
    // the dynamic Smagorinsky workspace: the ten pass-1 fields, the per-block
    // partials of LM and MM, the per-level coefficient
    DynWs<R> dws{};
    double* d_cs2 = nullptr;
    R* d_cs2f = nullptr;       // the per-cell coefficient of the :local averaging (padded)
    double* d_dynpart = nullptr;
    int dyn_nb = 0;
    double dyn_d2 = 0.0;   // Delta^2 = (dx dy dz)^(2/3)
    // the kernels of the dynamic coefficient of the state in `in` (3 launches)
    aeo_status enqueue_dynamic(R* const* in) {
        const long long ns = (long long)dws.sx * dws.sy * (g.nz + 2);
        germano_pass1_kernel<R><<<(unsigned)std::min<long long>((ns + 255) / 256, 148LL * 16), 256, 0, st>>>(
            g, in[0], in[1], in[2], dws);
        CKL();
        if (dyn_local()) {
            germano_pass2_kernel<R, true><<<dim3((unsigned)dyn_nb, (unsigned)g.nz), 256, 0, st>>>(
                g, dws, R(1.0 / 27), R(dyn_d2), R(9.0), d_dynpart, d_cs2f, cfg.c_s * cfg.c_s);
            CKL();
            R* f[1] = {d_cs2f};
            int l[1] = {LOC_C};
            return halo(f, l, 1);
        }
        germano_pass2_kernel<R><<<dim3((unsigned)dyn_nb, (unsigned)g.nz), 256, 0, st>>>(
            g, dws, R(1.0 / 27), R(dyn_d2), R(9.0), d_dynpart);
        CKL();
        germano_level_kernel<<<(g.nz + 127) / 128, 128, 0, st>>>(g.nz, dyn_nb, d_dynpart, cfg.c_s * cfg.c_s, d_cs2);
        CKL();
        return AEO_OK;
    }
    int dyn_launches() const { return dyn() ? 3 : 0; }
    // the Lagrangian closure: its memories (two sets, LagArgs), the committed
    // set and initialised flag on the device (and a copy of them taken before
    // an adaptive step, put back when the step is retried), C0, theta, the
    // fixed memory time (0: MLC96's T)
    LagArgs<R> lagA{};
    int* d_lag_state = nullptr;
    double lag_c0 = 0.16, lag_theta = 1.5, lag_mt = 0.0;
    int lag_launches() const { return lag() ? 4 : 0; }   // per step
    // advance_sgs! of the state in `in` (halos filled): passes 1 and 2 with
    // the memory update, the coefficient's halos, the flip
    aeo_status enqueue_lag_commit(R* const* in) {
        const long long ns = (long long)dws.sx * dws.sy * (g.nz + 2);
        germano_pass1_kernel<R><<<(unsigned)std::min<long long>((ns + 255) / 256, 148LL * 16), 256, 0, st>>>(
            g, in[0], in[1], in[2], dws);
        CKL();
        germano_pass2_kernel<R, 2><<<dim3((unsigned)dyn_nb, (unsigned)g.nz), 256, 0, st>>>(
            g, dws, R(1.0 / 27), R(dyn_d2), R(9.0), d_dynpart, d_cs2f, cfg.c_s * cfg.c_s, lagA);
        CKL();
        R* f[1] = {d_cs2f};
        int l[1] = {LOC_C};
        if (aeo_status e = halo(f, l, 1)) return e;
        lag_flip_kernel<<<1, 1, 0, st>>>(d_lag_state);
        CKL();
        return AEO_OK;
    }
    // the coefficient of the committed memory (set-up, new parameters, a restored state)
    aeo_status lag_refresh() {
        lagA.c02 = lag_c0 * lag_c0;
        lagA.theta_delta = lag_theta * std::cbrt(g.dx * g.dy * g.dz);
        lagA.memory_time = lag_mt;
        lag_coefficient_kernel<R><<<(unsigned)std::min<long long>((g.nin + 255) / 256, 148LL * 16), 256, 0, st>>>(
            g, lagA, d_cs2f);
        CKL();
        R* f[1] = {d_cs2f};
        int l[1] = {LOC_C};
        if (aeo_status e = halo(f, l, 1)) return e;
        CK(cudaStreamSynchronize(st));
        return AEO_OK;
    }
    aeo_status set_lagrangian(double c0, double theta, double memory_time) override {
        if (!lag()) { fail("set_lagrangian: the domain's closure is not the Lagrangian dynamic one"); return AEO_ERR_STATE; }
        if (!(c0 > 0) || !(theta > 0) || !std::isfinite(c0) || !std::isfinite(theta) || !(memory_time >= 0) ||
            !std::isfinite(memory_time)) {
            fail("set_lagrangian: c0 > 0, theta > 0 and memory_time >= 0 (0: MLC96's T) required");
            return AEO_ERR_ARGUMENT;
        }
        CK(cudaStreamSynchronize(st));
        drop_graphs();   // the parameters are captured by value
        lag_c0 = c0; lag_theta = theta; lag_mt = memory_time;
        return lag_refresh();
    }
    // sgs_state / restore_sgs_state! (src/operators/lagrangian_sgs.jl:372-381)
    aeo_status sgs_state(double* out, bool get) {
        if (!lag()) { fail("sgs_state: the domain's closure keeps no memory"); return AEO_ERR_STATE; }
        if (!out) { fail("sgs_state: NULL array"); return AEO_ERR_ARGUMENT; }
        CK(cudaStreamSynchronize(st));
        int hs[2];
        CK(cudaMemcpy(hs, d_lag_state, sizeof(hs), cudaMemcpyDeviceToHost));
        std::vector<R> tmp((size_t)g.nin);
        for (int f = 0; f < 5; ++f) {
            double* o = out + (size_t)f * g.nin;
            if (get) {
                CK(cudaMemcpy(tmp.data(), lagA.mem[hs[0]][f], tmp.size() * sizeof(R), cudaMemcpyDeviceToHost));
                for (size_t q = 0; q < tmp.size(); ++q) o[q] = (double)tmp[q];
            } else {
                for (size_t q = 0; q < tmp.size(); ++q) tmp[q] = R(o[q]);
                CK(cudaMemcpy(lagA.mem[hs[0]][f], tmp.data(), tmp.size() * sizeof(R), cudaMemcpyHostToDevice));
            }
        }
        if (get) {
            out[5 * (size_t)g.nin] = hs[1] ? 1.0 : 0.0;
            return AEO_OK;
        }
        hs[1] = out[5 * (size_t)g.nin] != 0.0;
        CK(cudaMemcpy(d_lag_state, hs, sizeof(hs), cudaMemcpyHostToDevice));
        return lag_refresh();
    }
    aeo_status get_sgs_state(double* out) override {
        return tke() ? tke_state(out, true) : sgs_state(out, true);
    }
    aeo_status set_sgs_state(const double* in) override {
        return tke() ? tke_state(const_cast<double*>(in), false) : sgs_state(const_cast<double*>(in), false);
    }

    // the TKE closure: e (padded, halos filled), K = 2 nu_t and the transport
    // tendency of the commit (padded), the copy of e an adaptive step can
    // return to, the coefficients
    R *d_tke = nullptr, *d_tk2 = nullptr, *d_tkt = nullptr, *d_tke_keep = nullptr;
    TkeArgs tkeA{};
    int tke_launches() const { return tke() ? 8 : 0; }   // per step
    aeo_status set_tke(double c_eps0, double c_eps1, double c_l, int exact) override {
        if (!tke()) { fail("set_tke: the domain's closure is not the TKE closure"); return AEO_ERR_STATE; }
        if (!(c_eps0 >= 0) || !(c_eps1 >= 0) || !(c_l > 0) || !std::isfinite(c_eps0) || !std::isfinite(c_eps1) ||
            !std::isfinite(c_l)) {
            fail("set_tke: c_eps0 >= 0, c_eps1 >= 0 and c_l > 0 required");
            return AEO_ERR_ARGUMENT;
        }
        CK(cudaStreamSynchronize(st));
        drop_graphs();   // the coefficients are captured by value
        tkeA.ce0 = c_eps0; tkeA.ce1 = c_eps1; tkeA.cl = c_l; tkeA.exact = exact != 0;
        g.tke_cl = c_l;
        return AEO_OK;
    }
    // advance_sgs! of the TKE closure for the state in `in` (halos filled)
    aeo_status enqueue_tke_commit(R* const* in) {
        const unsigned nb = (unsigned)std::min<long long>((g.nin + 255) / 256, 148LL * 16);
        tke_coef_kernel<R><<<nb, 256, 0, st>>>(g, tkeA, d_tke, in[3], d_tk2);
        CKL();
        R* f[2] = {d_tk2, d_tke};
        int l[2] = {LOC_C, LOC_C};
        if (aeo_status e = halo(f, l, 2)) return e;
        PosGeo pg{};
        pg.nx = g.nx; pg.ny = g.ny; pg.nz = g.nz;
        pg.hx = AEO_HX; pg.hy = AEO_H; pg.hz = AEO_H;
        pg.sx = 1; pg.sy = g.sy; pg.sz = g.sz;
        pg.idx = g.idx; pg.idy = g.idy; pg.idz = g.idz;
        const dim3 gf((unsigned)((g.nx + 1 + 127) / 128), (unsigned)(g.ny + 1), (unsigned)(g.nz + 1));
        pos_flux_kernel<R, AEO_ADV_WENO_Z5><<<gf, 128, 0, st>>>(pg, in[0], in[1], in[2], d_tke, pos_fx, pos_fy, pos_fz);
        CKL();
        const dim3 gc((unsigned)((g.nx + 127) / 128), (unsigned)g.ny, (unsigned)g.nz);
        pos_ratio_kernel<R><<<gc, 128, 0, st>>>(pg, in[0], in[1], in[2], d_tke, pos_fx, pos_fy, pos_fz, &d_sc->dt, pos_r);
        CKL();
        pos_apply_kernel<R><<<gc, 128, 0, st>>>(pg, in[0], in[1], in[2], d_tke, pos_fx, pos_fy, pos_fz, pos_r, d_tkt, 0);
        CKL();
        tke_update_kernel<R><<<(unsigned)((g.nin + 127) / 128), 128, 0, st>>>(g, tkeA, d_tke, d_tk2, in[3], in[0], in[1],
                                                                              in[2], &d_sc->dt, d_tkt);
        CKL();
        tke_copy_kernel<R><<<nb, 256, 0, st>>>(g, d_tkt, d_tke);
        CKL();
        R* fe[1] = {d_tke};
        int le[1] = {LOC_C};
        return halo(fe, le, 1);
    }
    // the TKE closure's sgs_state / restore_sgs_state! (src/PrognosticSGS.jl:1174-1197): e on the interior
    aeo_status tke_state(double* io, bool get) {
        if (!io) { fail("sgs_state: NULL array"); return AEO_ERR_ARGUMENT; }
        CK(cudaStreamSynchronize(st));
        if (get) return get_padded(d_tke, io);
        for (long long q = 0; q < g.nin; ++q)
            if (!(io[q] >= 0) || !std::isfinite(io[q])) { fail("set_sgs_state: e must be finite and >= 0"); return AEO_ERR_ARGUMENT; }
        if (aeo_status e = put_padded(d_tke, io)) return e;
        R* f[1] = {d_tke};
        int l[1] = {LOC_C};
        if (aeo_status e = halo(f, l, 1)) return e;
        CK(cudaStreamSynchronize(st));
        return AEO_OK;
    }
    // an interior array (x fastest, FP64 on the host) to / from a padded device field
    aeo_status put_padded(R* dst, const double* h) {
        std::vector<R> tmp((size_t)g.nin);
        for (size_t q = 0; q < tmp.size(); ++q) tmp[q] = R(h[q]);
        CK(cudaMemcpyAsync(d_stage, tmp.data(), tmp.size() * sizeof(R), cudaMemcpyHostToDevice, st));
        dim3 gb((g.nx + 127) / 128, g.ny, g.nz);
        interior_to_padded_kernel<R><<<gb, 128, 0, st>>>(g, reinterpret_cast<const R*>(d_stage), dst, R(1));
        CKL();
        CK(cudaStreamSynchronize(st));
        return AEO_OK;
    }
    aeo_status get_padded(const R* src, double* h) {
        dim3 gb((g.nx + 127) / 128, g.ny, g.nz);
        padded_to_interior_kernel<R><<<gb, 128, 0, st>>>(g, src, reinterpret_cast<R*>(d_stage));
        CKL();
        std::vector<R> tmp((size_t)g.nin);
        CK(cudaMemcpyAsync(tmp.data(), d_stage, tmp.size() * sizeof(R), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        for (size_t q = 0; q < tmp.size(); ++q) h[q] = (double)tmp[q];
        return AEO_OK;
    }
    // g / theta0 of the AMD closure's buoyancy term (0 without buoyancy)
    R amd_bg() const { return R(amd() && cfg.theta0 != 0.0 ? cfg.g / cfg.theta0 : 0.0); }
    // the AMD closure on the sound-proof core takes its per-level buoyancy
    // parameter g/theta_bar(z_k) from aeo_set_sgs_buoyancy before the first step
    bool bg_levels_set = false;
    aeo_status sgs_ready() {
        if (amd() && anel && !bg_levels_set) {
            fail("the AMD closure on the sound-proof core needs its per-level buoyancy parameter g/theta_bar "
                 "(aeo_set_sgs_buoyancy) before a step");
            return AEO_ERR_STATE;
        }
        return AEO_OK;
    }
    aeo_status set_sgs_buoyancy(const double* bgv) override {
        if (!bgv) { fail("set_sgs_buoyancy: NULL levels"); return AEO_ERR_ARGUMENT; }
        for (int k = 0; k < g.nz; ++k)
            if (!std::isfinite(bgv[k])) { fail("set_sgs_buoyancy: non-finite level value"); return AEO_ERR_ARGUMENT; }
        // the row of the working-precision table, halo entries from the nearest level
        std::vector<R> row((size_t)g.lvn);
        for (int e = 0; e < g.lvn; ++e) row[e] = R(bgv[std::min(std::max(e - AEO_LH, 0), g.nz - 1)]);
        CK(cudaStreamSynchronize(st));
        CK(cudaMemcpy(levels_r + (size_t)LV_BGC * g.lvn, row.data(), row.size() * sizeof(R), cudaMemcpyHostToDevice));
        bg_levels_set = true;
        return AEO_OK;
    }
    // per-kernel-class timing of one un-graphed step (aeo_profile_step)
    bool profiling = false;
    std::vector<std::pair<int, cudaEvent_t>> marks;
    void mark(int cls) {
        if (!profiling) return;
        cudaEvent_t e;
        cudaEventCreate(&e);
        cudaEventRecord(e, st);
        marks.push_back({cls, e});
    }

    ~Core() override {
        if (st) cudaStreamSynchronize(st);   // solves of the MG-PCG handle may be in flight on st
        drop_graphs();
        if (mg) aeo_mg_destroy(mg);
        for (void* p : allocs) cudaFree(p);
        if (st_loop) cudaStreamDestroy(st_loop);
        if (st) cudaStreamDestroy(st);
    }

    void drop_graphs() {
        for (auto& a : gexec)
            for (auto& e : a)
                if (e) { cudaGraphExecDestroy(e); e = nullptr; }
        for (auto& e : gmulti)
            if (e) { cudaGraphExecDestroy(e); e = nullptr; }
    }

    template <typename T>
    aeo_status alloc(T** p, size_t count) {
        void* q = nullptr;
        cudaError_t e = cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(T));
        if (e != cudaSuccess) {
            fail(std::string("cudaMalloc: ") + cudaGetErrorString(e));
            return AEO_ERR_CUDA;
        }
        CK(cudaMemsetAsync(q, 0, std::max<size_t>(count, 1) * sizeof(T), st));
        allocs.push_back(q);
        *p = reinterpret_cast<T*>(q);
        return AEO_OK;
    }

    long long padded_count() const { return (long long)g.sz * (g.nz + 2 * AEO_H); }

    aeo_status init(const double* zfi, const double* wc, const double* wf, const double* thf) override {
        const aeo_config& c = cfg;
        CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        CK(cudaStreamCreateWithFlags(&st_loop, cudaStreamNonBlocking));
        uni = !c.stretched;
        sgs = c.c_s != 0.0;
        anel = c.core == AEO_CORE_ANELASTIC;
        g.sgs_model = (c.sgs_model == AEO_SGS_DYNAMIC_LOCAL || c.sgs_model == AEO_SGS_LAGRANGIAN) ? AEO_SGS_DYNAMIC
                                                                                                  : c.sgs_model;   // devices: cs2f set
        g.sgs_cv = 2.5 * c.c_s * c.c_s;
        if (sizeof(R) == sizeof(float)) th_off = anel ? (thf ? thf[c.hz] : 0.0) : c.theta0;
        g.nx = c.nx; g.ny = c.ny; g.nz = c.nz;
        g.px = c.nx + 2 * AEO_HX;
        g.py = c.ny + 2 * AEO_H;
        g.sy = g.px;
        g.sz = (long long)g.px * g.py;
        g.nin = (long long)c.nx * c.ny * c.nz;
        g.bc_z = c.bc_z;
        g.uniform = uni;
        g.dx = c.lx / c.nx; g.dy = c.ly / c.ny; g.dz = c.lz / c.nz;
        g.idx = 1 / g.dx; g.idy = 1 / g.dy; g.idx2 = 1 / (g.dx * g.dx); g.idy2 = 1 / (g.dy * g.dy);
        g.idz = 1 / g.dz; g.idz2 = 1 / (g.dz * g.dz);
        g.delta_u = std::pow(g.dx * g.dy * g.dz, 1.0 / 3);
        // ---- vertical metrics over the storage levels (src/StretchedGrids.jl:345-400, :570-590)
        const int Hz = c.hz, Nz = c.nz, NZ = Nz + 2 * Hz;
        std::vector<double> zf(NZ + 1), zc(NZ), dzc(NZ), dzf(NZ + 1);
        if (uni) {
            for (int k = 0; k <= NZ; ++k) zf[k] = c.z0 + (double)(k - Hz) * g.dz;
            for (int k = 0; k < NZ; ++k) zc[k] = c.z0 + ((double)(k - Hz) + 0.5) * g.dz;
            for (int k = 0; k < NZ; ++k) dzc[k] = g.dz;
            for (int k = 0; k <= NZ; ++k) dzf[k] = g.dz;
        } else {
            for (int k = 0; k <= Nz; ++k) zf[Hz + k] = zfi[k];
            for (int k = Hz - 1; k >= 0; --k) zf[k] = 2 * zf[k + 1] - zf[k + 2];
            for (int k = Hz + Nz + 1; k <= NZ; ++k) zf[k] = 2 * zf[k - 1] - zf[k - 2];
            for (int k = 0; k < NZ; ++k) dzc[k] = zf[k + 1] - zf[k];
            for (int k = 0; k < NZ; ++k) zc[k] = (zf[k] + zf[k + 1]) / 2;
            dzf[0] = dzc[0];
            for (int k = 1; k < NZ; ++k) dzf[k] = zc[k] - zc[k - 1];
            dzf[NZ] = dzc[NZ - 1];
        }
        h_dzc.assign(dzc.begin() + Hz, dzc.begin() + Hz + Nz);
        h_dzf.assign(dzf.begin() + Hz, dzf.begin() + Hz + Nz + 1);
        h_wc.assign(Nz, 1.0);
        h_wf.assign(Nz + 1, 1.0);
        if (anel) {
            for (int k = 0; k < Nz; ++k) h_wc[k] = wc[Hz + k];
            for (int k = 0; k <= Nz; ++k) h_wf[k] = wf[Hz + k];
        }
        dz_min = dzc[Hz];
        for (int k = Hz; k < Hz + Nz; ++k) dz_min = std::min(dz_min, dzc[k]);
        // device vectors indexed by interior level k at (k + AEO_LH); storage level K = k + Hz
        const int L = Nz + 2 * AEO_LH + 2;
        const int NV = 13;
        std::vector<double> hv((size_t)NV * L, 0.0);
        auto put = [&](int vec, int K, double val) {
            int e = K - Hz + AEO_LH;
            if (e >= 0 && e < L) hv[(size_t)vec * L + e] = val;
        };
        for (int K = 0; K < NZ; ++K) {
            put(0, K, 1 / dzc[K]);
            put(2, K, 2 / (dzf[K] + dzf[K + 1]));
            put(7, K, std::pow(g.dx * g.dy * dzc[K], 1.0 / 3));
            put(8, K, zc[K]);
            if (K >= 1) {
                double sm = dzc[K - 1] + dzc[K];
                put(3, K, dzc[K] / (dzc[K - 1] + dzc[K]));
                put(4, K, dzc[K - 1] / (dzc[K - 1] + dzc[K]));
                put(5, K, dzc[K - 1] / sm);
                put(6, K, dzc[K] / sm);
            }
        }
        for (int K = 0; K <= NZ; ++K) {
            put(1, K, 1 / dzf[K]);
            put(9, K, zf[K]);
        }
        if (anel) {
            for (int K = 0; K < NZ; ++K) put(10, K, wc[K]);
            for (int K = 0; K <= NZ; ++K) put(11, K, wf[K]);
            if (thf)
                for (int K = 0; K <= NZ; ++K) put(12, K, thf[K]);
        }
        if (aeo_status s = alloc(&levels, hv.size())) return s;
        CK(cudaMemcpyAsync(levels, hv.data(), hv.size() * sizeof(double), cudaMemcpyHostToDevice, st));
        g.idzc = levels + 0 * L; g.idzf = levels + 1 * L; g.idz_off = levels + 2 * L;
        g.wlo = levels + 3 * L; g.whi = levels + 4 * L; g.alo = levels + 5 * L; g.ahi = levels + 6 * L;
        g.delta = levels + 7 * L; g.zc = levels + 8 * L; g.zf = levels + 9 * L;
        g.wc = anel ? levels + 10 * L : nullptr;
        g.wf = anel ? levels + 11 * L : nullptr;
        g.thf = anel ? levels + 12 * L : nullptr;
        // the same factors in R, with the reciprocals, g/theta_f and the sponge
        // rates folded in (each rounded as the division or product in R rounds it)
        {
            std::vector<R> hr((size_t)LV_N * L, R(0));
            auto row = [&](int v, int e) { return hv[(size_t)v * L + e]; };
            const R zs = R(c.sponge_zstart), al = R(c.sponge_alpha);
            const R sinv = R(1.0 / (c.z0 + c.lz - c.sponge_zstart));
            auto rate = [&](double z) -> R {
                if (c.sponge_alpha == 0.0 || !(z >= (double)zs)) return R(0);
                R arg = R(0.5 * 3.14159265358979323846) * (R(z) - zs) * sinv;
                R sn = R(std::sin((double)arg));
                return al * sn * sn;
            };
            for (int e = 0; e < L; ++e) {
                auto put_r = [&](int f, R v) { hr[(size_t)f * L + e] = v; };
                put_r(LV_IDZC, R(row(0, e)));
                put_r(LV_IDZF, R(row(1, e)));
                put_r(LV_IDZOFF, R(row(2, e)));
                put_r(LV_WLO, R(row(3, e)));
                put_r(LV_WHI, R(row(4, e)));
                put_r(LV_ALO, R(row(5, e)));
                put_r(LV_AHI, R(row(6, e)));
                put_r(LV_DELTA, R(row(7, e)));
                const R wcr = R(row(10, e)), wfr = R(row(11, e)), thr = R(row(12, e));
                put_r(LV_WC, wcr);
                put_r(LV_WF, wfr);
                put_r(LV_IWC, wcr != R(0) ? R(1) / wcr : R(0));
                put_r(LV_IWF, wfr != R(0) ? R(1) / wfr : R(0));
                put_r(LV_THF, R(row(12, e) - th_off));   // the buoyancy's reference in stored units
                put_r(LV_GTHF, thr != R(0) ? R(c.g) / thr : R(0));
                put_r(LV_SPC, rate(row(8, e)));
                put_r(LV_SPF, rate(row(9, e)));
                put_r(LV_BGC, amd_bg());   // the sound-proof core's levels come from aeo_set_sgs_buoyancy
            }
            if (aeo_status s = alloc(&levels_r, hr.size())) return s;
            CK(cudaMemcpyAsync(levels_r, hr.data(), hr.size() * sizeof(R), cudaMemcpyHostToDevice, st));
            g.lvr = levels_r;
            g.lvn = L;
        }

        // ---- eigenvalues and column coefficients
        const int Nx = c.nx, Ny = c.ny, Mh = Nx / 2 + 1;
        std::vector<double> hkx(Mh), hky(Ny), hkz(Nz);
        if (c.solver == AEO_SOLVER_FFT) {
            // src/PressureSolvers.jl:128-130
            for (int m = 0; m < Mh; ++m) { double s = std::sin(M_PI * m / Nx); hkx[m] = 4 / (g.dx * g.dx) * (s * s); }
            for (int m = 0; m < Ny; ++m) { double s = std::sin(M_PI * m / Ny); hky[m] = 4 / (g.dy * g.dy) * (s * s); }
            for (int m = 0; m < Nz; ++m) { double s = std::sin(M_PI * m / Nz); hkz[m] = 4 / (g.dz * g.dz) * (s * s); }
        } else {
            // _r2r_eigen, src/PressureSolvers.jl:618-624
            for (int m = 0; m < Mh; ++m) { int mm = std::min(m, Nx - m); double s = std::sin(M_PI * mm / Nx); hkx[m] = 4 / (g.dx * g.dx) * (s * s); }
            for (int m = 0; m < Ny; ++m) { int mm = std::min(m, Ny - m); double s = std::sin(M_PI * mm / Ny); hky[m] = 4 / (g.dy * g.dy) * (s * s); }
        }
        if (aeo_status s = alloc(&kx2, Mh)) return s;
        if (aeo_status s = alloc(&ky2, Ny)) return s;
        if (aeo_status s = alloc(&kz2, Nz)) return s;
        CK(cudaMemcpyAsync(kx2, hkx.data(), Mh * sizeof(double), cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(ky2, hky.data(), Ny * sizeof(double), cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(kz2, hkz.data(), Nz * sizeof(double), cudaMemcpyHostToDevice, st));
        if (c.solver == AEO_SOLVER_COLUMN) {
            std::vector<double> lo(Nz), up(Nz), hw(Nz), me(Nz), io(Nz + 1), ga(Nz);
            for (int k = 0; k < Nz; ++k) {
                int K = Hz + k;
                if (anel) {
                    if (uni) {
                        // DirectWeightedPoissonSolver, src/Anelastic.jl:1013-1019
                        double idz2 = 1 / (g.dz * g.dz);
                        lo[k] = k > 0 ? wf[K] * idz2 : 0.0;
                        up[k] = k < Nz - 1 ? wf[K + 1] * idz2 : 0.0;
                        hw[k] = wc[K]; me[k] = g.dz * g.dz; ga[k] = 1.0;
                    } else {
                        lo[k] = k > 0 ? wf[K] / (dzc[K] * dzf[K]) : 0.0;
                        up[k] = k < Nz - 1 ? wf[K + 1] / (dzc[K] * dzf[K + 1]) : 0.0;
                        hw[k] = wc[K]; me[k] = dzc[K]; ga[k] = dzc[K];
                    }
                } else {
                    // ColumnTridiagonalSolver(dzc, dzf), src/PressureSolvers.jl:686-700
                    lo[k] = k > 0 ? 1 / (dzc[K] * dzf[K]) : 0.0;
                    up[k] = k < Nz - 1 ? 1 / (dzc[K] * dzf[K + 1]) : 0.0;
                    hw[k] = 1.0; me[k] = dzc[K]; ga[k] = dzc[K];
                }
            }
            for (int k = 0; k <= Nz; ++k) {
                int K = Hz + k;
                io[k] = anel ? (uni ? 1 / wf[K] : dzf[K] / wf[K]) : dzf[K];
            }
            double ms = 0, gs = 0;
            for (int k = 0; k < Nz; ++k) { ms += me[k]; gs += ga[k]; }
            if (aeo_status s = alloc(&colc, 6 * (size_t)(Nz + 1))) return s;
            std::vector<double> hc(6 * (size_t)(Nz + 1), 0.0);
            std::copy(lo.begin(), lo.end(), hc.begin());
            std::copy(up.begin(), up.end(), hc.begin() + (Nz + 1));
            std::copy(hw.begin(), hw.end(), hc.begin() + 2 * (Nz + 1));
            std::copy(me.begin(), me.end(), hc.begin() + 3 * (Nz + 1));
            std::copy(io.begin(), io.end(), hc.begin() + 4 * (Nz + 1));
            std::copy(ga.begin(), ga.end(), hc.begin() + 5 * (Nz + 1));
            CK(cudaMemcpyAsync(colc, hc.data(), hc.size() * sizeof(double), cudaMemcpyHostToDevice, st));
            cc.lower = colc; cc.upper = colc + (Nz + 1); cc.hw = colc + 2 * (Nz + 1);
            cc.meas = colc + 3 * (Nz + 1); cc.iota = colc + 4 * (Nz + 1); cc.gauge = colc + 5 * (Nz + 1);
            cc.meas_sum = ms; cc.gauge_sum = gs; cc.kx2 = kx2; cc.ky2 = ky2;
        }

        // ---- twiddles
        NT = next_pow2(std::max(std::max(Nx, Ny), c.solver == AEO_SOLVER_FFT ? Nz : 1));
        {
            std::vector<cplx<R>> ht(NT);
            for (int m = 0; m < NT; ++m) {
                double a = -2.0 * M_PI * (double)m / (double)NT;
                ht[m].x = (R)std::cos(a);
                ht[m].y = (R)std::sin(a);
            }
            if (aeo_status s = alloc(&tw, NT)) return s;
            CK(cudaMemcpyAsync(tw, ht.data(), NT * sizeof(cplx<R>), cudaMemcpyHostToDevice, st));
        }
        rows_x = std::max(1, 2048 / (Nx / 2));
        tpx_y = std::max(1, std::min(16, 2048 / Ny));
        tpx_z = std::max(1, std::min(16, 2048 / Nz));

        // ---- fields
        const long long np = padded_count();
        for (int s = 0; s < 4; ++s)
            for (int f = 0; f < 4; ++f)
                if (aeo_status e = alloc(&P[s][f], np)) return e;
        for (int f = 0; f < 3; ++f)
            if (aeo_status e = alloc(&Q[f], g.nin)) return e;
        if (sgs)
            if (aeo_status e = alloc(&nut, np)) return e;
        if (aeo_status e = alloc(&phi, g.nin)) return e;
        if (aeo_status e = alloc(&pres, g.nin)) return e;
        const long long ns = (long long)Mh * Ny * Nz;
        if (aeo_status e = alloc(&S, ns)) return e;
        if (c.solver == AEO_SOLVER_COLUMN) {
            // the elimination factors m and c' of every column in the working precision
            if (aeo_status e = alloc(&cps, sizeof(R) == sizeof(double) ? 2 * ns : ns)) return e;
            R* ftab = reinterpret_cast<R*>(cps);
            const long long cols = (long long)Ny * Mh;
            thomas_factor_kernel<R><<<(unsigned)((cols + 255) / 256), 256, 0, st>>>(g, ftab, ftab + ns, cc);
            CKL();
        }
        if (c.solver == AEO_SOLVER_PCG) {
            pcg = true;
            if (aeo_status e = alloc(&apx, (size_t)(Nx + 1) * Ny * Nz)) return e;
            if (aeo_status e = alloc(&apy, (size_t)Nx * (Ny + 1) * Nz)) return e;
            if (aeo_status e = alloc(&apz, (size_t)Nx * Ny * (Nz + 1))) return e;
            if (aeo_status e = make_pcg(nullptr, nullptr, nullptr)) return e;
        }
        host_n = (long long)(c.nx + 2 * c.hx) * (c.ny + 2 * c.hy) * (c.nz + 2 * c.hz);
        if (aeo_status e = alloc(&d_stage, std::max<long long>(host_n, g.nin))) return e;
        if (aeo_status e = alloc(&d_part, 4 * (size_t)(Nz + 1))) return e;
        if (dyncl()) {
            dws.sx = g.nx + 2;
            dws.sy = g.ny + 2;
            const size_t ns = (size_t)dws.sx * dws.sy * (g.nz + 2);
            for (int f = 0; f < DYN_N; ++f)
                if (aeo_status e = alloc(&dws.f[f], ns)) return e;
            dyn_nb = (g.nx * g.ny + 255) / 256;
            if (aeo_status e = alloc(&d_dynpart, 2 * (size_t)dyn_nb * g.nz)) return e;
            if (aeo_status e = alloc(&d_cs2, (size_t)g.nz)) return e;
            if (dyn_local() || lag())
                if (aeo_status e = alloc(&d_cs2f, padded_count())) return e;
            dyn_d2 = std::pow(g.dx * g.dy * g.dz, 2.0 / 3.0);
        }
        if (tke()) {
            if (aeo_status e = alloc(&d_tke, padded_count())) return e;
            if (aeo_status e = alloc(&d_tk2, padded_count())) return e;
            if (aeo_status e = alloc(&d_tkt, padded_count())) return e;
            if (aeo_status e = alloc(&d_tke_keep, padded_count())) return e;
            if (aeo_status e = alloc(&pos_fx, (size_t)(g.nx + 1) * g.ny * g.nz)) return e;
            if (aeo_status e = alloc(&pos_fy, (size_t)g.nx * (g.ny + 1) * g.nz)) return e;
            if (aeo_status e = alloc(&pos_fz, (size_t)g.nx * g.ny * (g.nz + 1))) return e;
            if (aeo_status e = alloc(&pos_r, (size_t)g.nin)) return e;
            const bool buoy = cfg.theta0 > 0 && cfg.g > 0;
            tkeA.ck = cfg.c_s; tkeA.ce0 = 0.19; tkeA.ce1 = 0.51; tkeA.cl = 0.76;
            tkeA.delta = std::pow(g.dx * g.dy * g.dz, 1.0 / 3);
            tkeA.bg = buoy ? cfg.g / cfg.theta0 : 0.0;
            tkeA.pb1 = buoy ? cfg.g / cfg.theta0 * cfg.flux_bot / 2 : 0.0;
            tkeA.pb2 = buoy ? cfg.g / cfg.theta0 * cfg.flux_top / 2 : 0.0;
            tkeA.exact = 0;
            g.tke = d_tke;
            g.tke_ck = tkeA.ck; g.tke_cl = tkeA.cl; g.tke_delta = tkeA.delta; g.tke_bg = tkeA.bg;
        }
        if (lag()) {
            for (int b = 0; b < 2; ++b)
                for (int f = 0; f < 5; ++f)
                    if (aeo_status e = alloc(&lagA.mem[b][f], (size_t)g.nin)) return e;
            if (aeo_status e = alloc(&d_lag_state, 4)) return e;   // [0, 1] live, [2, 3] the copy
            lagA.state = d_lag_state;
            lagA.idx = 1.0 / g.dx; lagA.idy = 1.0 / g.dy; lagA.idz = 1.0 / g.dz;
            lagA.cs2max = cfg.c_s * cfg.c_s;
        }
        if (aeo_status e = alloc(&d_flag, 1)) return e;
        if (aeo_status e = alloc(&d_steps, 1)) return e;
        if (aeo_status e = alloc(&d_sc, 1)) return e;
        set_scalar_kernel<<<1, 1, 0, st>>>(&d_sc->one, 1.0);
        CKL();
        if (lag()) {
            lagA.dtp = &d_sc->dt;
            if (aeo_status e = lag_refresh()) return e;
        }
        if (aeo_status e = make_tensor_maps()) return e;
        kchunk = std::min(g.nz, TileShape<R, 0, false>::KCH);
        CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, cfg.device));
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&fin_per_sm, finite_check_kernel<R>, 256, 0));
        fin_per_sm = std::max(fin_per_sm, 1);
        {
            // the paired WENO sweep: the chunk length that minimises whole waves x
            // (levels + the 6-plane start of a chunk)
            const long long tiles = (long long)((g.nx + WPairShape::TX - 1) / WPairShape::TX) *
                                    ((g.ny + WPairShape::TY - 1) / WPairShape::TY);
            const long long slots = (long long)WPairShape::CTAS_PER_SM * nsm;
            long long best = -1;
            for (int c : {16, 32, 64}) {
                const int kc = std::min(c, g.nz);
                const long long waves = (tiles * ((g.nz + kc - 1) / kc) + slots - 1) / slots;
                const long long cost = waves * (kc + 6);
                if (best < 0 || cost < best) { best = cost; wchunk = kc; }
            }
        }
        CK(cudaStreamSynchronize(st));
        launches = 3 * (9 + dyn_launches()) + lag_launches() + tke_launches();
        return AEO_OK;
    }

    // The apertures (host FP64 in the face layout of aeolus_b200_mgpcg.h, NULL:
    // every face open; the wall faces of a bounded z are blocked whatever is
    // given), their device copies, and the MG-PCG handle of the a^2 operator.
    aeo_status make_pcg(const double* axh, const double* ayh, const double* azh) {
        const int Nx = g.nx, Ny = g.ny, Nz = g.nz;
        const size_t n[3] = {(size_t)(Nx + 1) * Ny * Nz, (size_t)Nx * (Ny + 1) * Nz, (size_t)Nx * Ny * (Nz + 1)};
        const double* src[3] = {axh, ayh, azh};
        std::vector<double> a[3], c2[3];
        for (int d = 0; d < 3; ++d) {
            a[d].assign(n[d], 1.0);
            if (src[d]) std::copy(src[d], src[d] + n[d], a[d].begin());
            for (double v : a[d])
                if (!(v >= 0.0 && v <= 1.0)) { fail("set_pcg: apertures must lie in [0, 1]"); return AEO_ERR_ARGUMENT; }
        }
        if (g.bc_z == 1)
            for (size_t q = 0; q < (size_t)Nx * Ny; ++q) {
                a[2][q] = 0.0;
                a[2][(size_t)Nz * Nx * Ny + q] = 0.0;
            }
        for (int d = 0; d < 3; ++d) h_ap[d] = a[d];
        R* dst[3] = {apx, apy, apz};
        // c = a^2 on the uniform Boussinesq column; with density weights or a
        // stretched column, the symmetric form (aeo_cutcell.cuh): W_c a^2 dz_c/h_z
        // on x and y faces, W_f a^2 h_z/dz_f on z faces
        const bool weighted = anel || !uni;
        const size_t rowx = (size_t)(Nx + 1) * Ny, rowy = (size_t)Nx * (Ny + 1), rowz = (size_t)Nx * Ny;
        for (int d = 0; d < 3; ++d) {
            std::vector<R> ar(n[d]);
            c2[d].resize(n[d]);
            for (size_t q = 0; q < n[d]; ++q) {
                ar[q] = R(a[d][q]);
                c2[d][q] = a[d][q] * a[d][q];
                if (weighted) {
                    if (d < 2) {
                        const int k = (int)(q / (d == 0 ? rowx : rowy));
                        c2[d][q] *= h_wc[k] * (h_dzc[k] / g.dz);
                    } else {
                        const int k = (int)(q / rowz);
                        c2[d][q] *= h_wf[k] * (g.dz / h_dzf[k]);
                    }
                }
            }
            CK(cudaMemcpyAsync(dst[d], ar.data(), n[d] * sizeof(R), cudaMemcpyHostToDevice, st));
            CK(cudaStreamSynchronize(st));
        }
        // open faces: the operator couples nothing across them (the Neumann
        // condition of phi, src/boundary_conditions/open_boundary.jl:485-531);
        // the divergence keeps their apertures (the prescribed flux)
        if (open_x)
            for (size_t r = 0; r < (size_t)Ny * Nz; ++r) c2[0][r * (Nx + 1)] = c2[0][r * (Nx + 1) + Nx] = 0.0;
        if (open_y)
            for (int k = 0; k < Nz; ++k)
                for (int i = 0; i < Nx; ++i)
                    c2[1][(size_t)k * (Ny + 1) * Nx + i] = c2[1][((size_t)k * (Ny + 1) + Ny) * Nx + i] = 0.0;
        aeo_mg_config mc{};
        mc.nx = Nx; mc.ny = Ny; mc.nz = Nz;
        mc.dx = g.dx; mc.dy = g.dy; mc.dz = g.dz;
        mc.bc_x = open_x ? AEO_MG_NEUMANN : AEO_MG_PERIODIC;
        mc.bc_y = open_y ? AEO_MG_NEUMANN : AEO_MG_PERIODIC;
        mc.bc_z = g.bc_z == 1 ? AEO_MG_NEUMANN : AEO_MG_PERIODIC;
        mc.precision = cfg.precision;
        mc.precond = AEO_PC_VCYCLE;
        mc.flexible = cfg.precision == AEO_PREC_FP64 ? 0 : 1;
        mc.tol = pcg_tol;
        mc.maxit = pcg_maxit;
        mc.nu1 = 2; mc.nu2 = 2; mc.coarse_sweeps = 50; mc.min_size = 4;
        mc.device = cfg.device;
        CK(cudaStreamSynchronize(st));   // no solve of the old handle in flight
        drop_graphs();                   // the step graphs hold the old handle's nodes
        if (mg) { aeo_mg_destroy(mg); mg = nullptr; }
        if (aeo_status e = aeo_mg_create(&mc, c2[0].data(), c2[1].data(), c2[2].data(), &mg)) {
            fail(std::string("the MG-PCG pressure solver: ") + aeo_mg_last_error(nullptr));
            return e;
        }
        aeo_mg_buffers(mg, &mg_b, &mg_x);
        return AEO_OK;
    }

    aeo_status set_pcg(const double* ax, const double* ay, const double* az, double tol, int maxit) override {
        if (!pcg) { fail("set_pcg: the domain was not created with solver = AEO_SOLVER_PCG"); return AEO_ERR_STATE; }
        if (!(tol > 0) || maxit < 1) { fail("set_pcg: tol > 0 and maxit >= 1 required"); return AEO_ERR_ARGUMENT; }
        if ((ax == nullptr) != (ay == nullptr) || (ax == nullptr) != (az == nullptr)) {
            fail("set_pcg: give all three aperture arrays or none");
            return AEO_ERR_ARGUMENT;
        }
        pcg_tol = tol;
        pcg_maxit = maxit;
        return make_pcg(ax, ay, az);
    }

    // a PCG substage: sweep, cc_div, the solve graph, cc_correct, halo fill
    int step_launches() override {
        if (!pcg) return launches;
        aeo_mg_stats o{};
        if (cudaStreamSynchronize(st) != cudaSuccess || aeo_mg_read_stats(mg, &o)) return 0;
        return 3 * (4 + dyn_launches() + aeo_mg_launches_per_solve(mg, o.iterations)) + lag_launches() + tke_launches();
    }

    // the implicit IBM correction after every predictor (aeo_set_ibm)
    unsigned char* ibm_mask = nullptr;
    unsigned char* ibm_alloc = nullptr;
    double ibm_tau = 0.0;
    aeo_status set_ibm(const uint8_t* mask, double tau) override {
        if (pcg) { fail("set_ibm: the PCG solver takes obstacles as apertures (aeo_set_pcg)"); return AEO_ERR_STATE; }
        if (!(tau >= 0)) { fail("set_ibm: tau >= 0 required"); return AEO_ERR_ARGUMENT; }
        CK(cudaStreamSynchronize(st));
        drop_graphs();   // the step graphs gain or lose the correction
        if (!mask) {
            ibm_mask = nullptr;
            launches = 3 * (9 + dyn_launches()) + lag_launches() + tke_launches();
            return AEO_OK;
        }
        std::vector<unsigned char> m((size_t)g.nin);
        const long long HX = cfg.nx + 2LL * cfg.hx, HY = cfg.ny + 2LL * cfg.hy;
        for (int k = 0; k < g.nz; ++k)
            for (int j = 0; j < g.ny; ++j)
                for (int i = 0; i < g.nx; ++i)
                    m[(size_t)i + (size_t)g.nx * ((size_t)j + (size_t)g.ny * k)] =
                        mask[(i + cfg.hx) + HX * ((j + cfg.hy) + HY * (long long)(k + cfg.hz))] ? 1 : 0;
        if (!ibm_alloc)
            if (aeo_status e = alloc(&ibm_alloc, (size_t)g.nin)) return e;
        CK(cudaMemcpyAsync(ibm_alloc, m.data(), m.size(), cudaMemcpyHostToDevice, st));
        CK(cudaStreamSynchronize(st));
        ibm_mask = ibm_alloc;
        ibm_tau = tau;
        launches = 3 * (10 + dyn_launches()) + lag_launches() + tke_launches();
        return AEO_OK;
    }

    aeo_status pcg_stats(aeo_mg_stats* o) override {
        if (!pcg) { fail("pcg_stats: the domain was not created with solver = AEO_SOLVER_PCG"); return AEO_ERR_STATE; }
        CK(cudaStreamSynchronize(st));
        return aeo_mg_read_stats(mg, o);
    }

    aeo_status pcg_set_learned(aeo_unet* net, double stagnation) override {
        if (!pcg) { fail("pcg_set_learned: the domain was not created with solver = AEO_SOLVER_PCG"); return AEO_ERR_STATE; }
        CK(cudaStreamSynchronize(st));
        drop_graphs();   // the solve's loop body changes with the preconditioner
        if (aeo_status e = aeo_mg_set_learned(mg, net, stagnation)) {
            fail(std::string("pcg_set_learned: ") + aeo_mg_last_error(mg));
            return e;
        }
        pcg_learned = net != nullptr;
        return AEO_OK;
    }

    // The right-hand side of the last projection's solve (the run's own
    // snapshot), solved again from zero by the plain MG-preconditioned CG with
    // the residual and iterate of its first `cap` iterations recorded.
    aeo_status pcg_harvest(int cap, double* b, double* x, double* rh, double* xh, int* count) override {
        if (!pcg) { fail("pcg_harvest: the domain was not created with solver = AEO_SOLVER_PCG"); return AEO_ERR_STATE; }
        if (pcg_learned) {
            fail("pcg_harvest: pairs come from plain solves; switch the learned preconditioner off first");
            return AEO_ERR_STATE;
        }
        CK(cudaStreamSynchronize(st));
        aeo_mg_stats o{};
        if (aeo_status e = aeo_mg_read_stats(mg, &o)) { fail(std::string("pcg_harvest: ") + aeo_mg_last_error(mg)); return e; }
        if (!(o.bnorm > 0)) { fail("pcg_harvest: no projection with a non-zero right-hand side has run yet"); return AEO_ERR_STATE; }
        CK(cudaMemcpy(b, mg_b, sizeof(double) * (size_t)g.nin, cudaMemcpyDeviceToHost));
        if (aeo_status e = aeo_mg_solve_harvest(mg, b, x, &o, rh, xh, cap, count)) {
            fail(std::string("pcg_harvest: ") + aeo_mg_last_error(mg));
            return e;
        }
        return AEO_OK;
    }

    // Open lateral faces (open_boundary_conditions,
    // src/boundary_conditions/open_boundary.jl:532-638): the plane buffers in
    // the layout of OpenSet (host FP64), per-field modes (0 plane, 1 mirror);
    // the PCG operator is rebuilt with the Neumann condition on the open axes
    // and the state's halos refilled.
    aeo_status set_open(int ox, int oy, const double* xp, const double* yp, const int* modes) override {
        if (!pcg) { fail("set_open: open faces need the PCG projection (solver = AEO_SOLVER_PCG)"); return AEO_ERR_STATE; }
        if (anel || !uni) { fail("set_open: open faces are built on the uniform Boussinesq core"); return AEO_ERR_STATE; }
        if (g.bc_z != 1) { fail("set_open: open lateral faces need walls in z"); return AEO_ERR_STATE; }
        if (sgs && cfg.sgs_model >= AEO_SGS_DYNAMIC) {
            fail("set_open: open faces take the static SGS closures (Smagorinsky, Vreman, sigma, AMD)");
            return AEO_ERR_STATE;
        }
        if ((ox && !xp) || (oy && !yp) || ((ox || oy) && !modes)) { fail("set_open: NULL plane array"); return AEO_ERR_ARGUMENT; }
        if (ox || oy)
            for (int f = 0; f < 4; ++f)
                if (modes[f] != 0 && !(f == 3 && modes[f] == 1)) {
                    fail("set_open: the velocities take their planes (mode 0), theta its plane or the mirror (1)");
                    return AEO_ERR_ARGUMENT;
                }
        CK(cudaStreamSynchronize(st));
        drop_graphs();
        const int H = AEO_H, NX = g.nx + 2 * H, NY = g.ny + 2 * H, NZ = g.nz + 2 * H, L = H + 1;
        const size_t nxp = (size_t)8 * NZ * NY * L, nyp = (size_t)8 * NZ * L * NX;
        if (!ob.xp) {
            R *a = nullptr, *b = nullptr, *c = nullptr, *d = nullptr, *e = nullptr, *f = nullptr;
            if (aeo_status x = alloc(&a, nxp)) return x;
            if (aeo_status x = alloc(&b, nyp)) return x;
            if (aeo_status x = alloc(&c, (size_t)g.ny * g.nz)) return x;
            if (aeo_status x = alloc(&d, (size_t)g.ny * g.nz)) return x;
            if (aeo_status x = alloc(&e, (size_t)g.nx * g.nz)) return x;
            if (aeo_status x = alloc(&f, (size_t)g.nx * g.nz)) return x;
            ob.xp = a; ob.yp = b; ob.bw = c; ob.be = d; ob.bs = e; ob.bn = f;
        }
        ob.L = L;
        for (int f = 0; f < 4; ++f) ob.mode[f] = (ox || oy) ? modes[f] : 0;
        // theta is stored as its deviation from th_off
        auto conv = [&](const double* src, size_t n, size_t per_field) {
            std::vector<R> out(n, R(0));
            if (src)
                for (size_t q = 0; q < n; ++q) out[q] = R(src[q] - (q / per_field == 3 ? th_off : 0.0));
            return out;
        };
        std::vector<R> hx = conv(ox ? xp : nullptr, nxp, nxp / 4), hy = conv(oy ? yp : nullptr, nyp, nyp / 4);
        std::vector<R> bw((size_t)g.ny * g.nz), be(bw.size()), bs((size_t)g.nx * g.nz), bn(bs.size());
        for (int k = 0; k < g.nz; ++k) {
            for (int j = 0; j < g.ny; ++j) {
                bw[(size_t)k * g.ny + j] = hx[(((size_t)0 * NZ + k + H) * NY + j + H) * L + H];
                be[(size_t)k * g.ny + j] = hx[(((size_t)1 * NZ + k + H) * NY + j + H) * L + 0];
            }
            for (int i = 0; i < g.nx; ++i) {
                bs[(size_t)k * g.nx + i] = hy[(((size_t)2 * NZ + k + H) * L + H) * NX + i + H];
                bn[(size_t)k * g.nx + i] = hy[(((size_t)3 * NZ + k + H) * L + 0) * NX + i + H];
            }
        }
        CK(cudaMemcpy((void*)ob.xp, hx.data(), nxp * sizeof(R), cudaMemcpyHostToDevice));
        CK(cudaMemcpy((void*)ob.yp, hy.data(), nyp * sizeof(R), cudaMemcpyHostToDevice));
        CK(cudaMemcpy((void*)ob.bw, bw.data(), bw.size() * sizeof(R), cudaMemcpyHostToDevice));
        CK(cudaMemcpy((void*)ob.be, be.data(), be.size() * sizeof(R), cudaMemcpyHostToDevice));
        CK(cudaMemcpy((void*)ob.bs, bs.data(), bs.size() * sizeof(R), cudaMemcpyHostToDevice));
        CK(cudaMemcpy((void*)ob.bn, bn.data(), bn.size() * sizeof(R), cudaMemcpyHostToDevice));
        ob.ox = ox ? 1 : 0;
        ob.oy = oy ? 1 : 0;
        open_x = ox != 0;
        open_y = oy != 0;
        g.ox = ob.ox;     // the sweeps' closure fields take the mirror across open faces
        g.oy = ob.oy;
        ob_rad = false;   // Dirichlet until set_open_outflow
        for (int q = 0; q < 4; ++q) ob.rad[q] = 0;
        if (aeo_status e = make_pcg(h_ap[0].data(), h_ap[1].data(), h_ap[2].data())) return e;
        R* f[4] = {P[cur][0], P[cur][1], P[cur][2], P[cur][3]};
        int l[4] = {LOC_FX, LOC_FY, LOC_FZ, LOC_C};
        if (aeo_status e = halo(f, l, 4)) return e;
        CK(cudaStreamSynchronize(st));
        return AEO_OK;
    }

    // The radiating outflow of the open faces already set (set_open): per side
    // (west, east, south, north) 1 = :convective, the correction mode and the
    // raw data planes (before the correction) in the buffers' layout; the
    // step then refills, radiates and corrects the buffers before every
    // projection (update_open_boundaries!, open_boundary.jl:1137-1152).
    aeo_status set_open_outflow(const int* rad, int corr, const double* xd, const double* yd, const double* xw,
                                const double* yw) override {
        if (!(open_x || open_y)) { fail("set_open_outflow: no open face (aeo_set_open first)"); return AEO_ERR_STATE; }
        if (!rad || corr < 0 || corr > 2) { fail("set_open_outflow: NULL flags or a correction mode outside 0..2"); return AEO_ERR_ARGUMENT; }
        bool any = false;
        for (int q = 0; q < 4; ++q) {
            if (rad[q] < 0 || rad[q] > 2) { fail("set_open_outflow: a side's mode is 0 dirichlet, 1 convective or 2 orlanski"); return AEO_ERR_ARGUMENT; }
            if (rad[q] && !(q < 2 ? open_x : open_y)) { fail("set_open_outflow: a radiating side that is not open"); return AEO_ERR_ARGUMENT; }
            any = any || rad[q];
        }
        if (any && ((open_x && !xd) || (open_y && !yd))) { fail("set_open_outflow: NULL data planes"); return AEO_ERR_ARGUMENT; }
        CK(cudaStreamSynchronize(st));
        drop_graphs();
        ob.corr = corr;
        for (int q = 0; q < 4; ++q) ob.rad[q] = rad[q];
        ob_rad = any;
        if (!any) return AEO_OK;
        const int H = AEO_H, NX = g.nx + 2 * H, NY = g.ny + 2 * H, NZ = g.nz + 2 * H, L = H + 1;
        const size_t nxp = (size_t)8 * NZ * NY * L, nyp = (size_t)8 * NZ * L * NX;
        const size_t ntx = (size_t)8 * NZ * NY, nty = (size_t)8 * NZ * NX;
        if (!ob.xs) {
            R* b[12] = {};
            const size_t n[12] = {nxp, nyp, nxp, nyp, nxp, nyp, ntx, nty, ntx, nty, ntx, nty};
            for (int q = 0; q < 12; ++q)
                if (aeo_status e = alloc(&b[q], n[q])) return e;
            double* led = nullptr;
            if (aeo_status e = alloc(&led, 4)) return e;
            double *dxw = nullptr, *dyw = nullptr;
            if (aeo_status e = alloc(&dxw, (size_t)2 * g.nz * g.ny)) return e;
            if (aeo_status e = alloc(&dyw, (size_t)2 * g.nz * g.nx)) return e;
            ob.xw = dxw;
            ob.yw = dyw;
            R *hx_ = nullptr, *hy_ = nullptr;
            if (aeo_status e = alloc(&hx_, ntx)) return e;
            if (aeo_status e = alloc(&hy_, nty)) return e;
            int* hok = nullptr;
            double* ldt = nullptr;
            if (aeo_status e = alloc(&hok, 1)) return e;
            if (aeo_status e = alloc(&ldt, 1)) return e;
            ob.xh = hx_; ob.yh = hy_; ob.hist_ok = hok; ob.last_dt = ldt;
            ob.xd = b[0]; ob.yd = b[1]; ob.xs = b[2]; ob.ys = b[3]; ob.xv = b[4]; ob.yv = b[5];
            ob.xc = b[6]; ob.yc = b[7]; ob.x1 = b[8]; ob.y1 = b[9]; ob.x2 = b[10]; ob.y2 = b[11];
            ob.led = led;
        }
        std::vector<R> hx(nxp, R(0)), hy(nyp, R(0));
        if (open_x)
            for (size_t q = 0; q < nxp; ++q) hx[q] = R(xd[q] - (q / (nxp / 4) == 3 ? th_off : 0.0));
        if (open_y)
            for (size_t q = 0; q < nyp; ++q) hy[q] = R(yd[q] - (q / (nyp / 4) == 3 ? th_off : 0.0));
        CK(cudaMemcpy((void*)ob.xd, hx.data(), nxp * sizeof(R), cudaMemcpyHostToDevice));
        CK(cudaMemcpy((void*)ob.yd, hy.data(), nyp * sizeof(R), cudaMemcpyHostToDevice));
        CK(cudaMemset(ob.hist_ok, 0, sizeof(int)));   // the Orlanski history starts empty
        std::vector<double> wx((size_t)2 * g.nz * g.ny, 1.0), wy((size_t)2 * g.nz * g.nx, 1.0);
        if (xw) std::copy(xw, xw + wx.size(), wx.begin());
        if (yw) std::copy(yw, yw + wy.size(), wy.begin());
        for (double v : wx) if (!(v >= 0.0 && v <= 1.0)) { fail("set_open_outflow: face weights lie in [0, 1]"); return AEO_ERR_ARGUMENT; }
        for (double v : wy) if (!(v >= 0.0 && v <= 1.0)) { fail("set_open_outflow: face weights lie in [0, 1]"); return AEO_ERR_ARGUMENT; }
        CK(cudaMemcpy((void*)ob.xw, wx.data(), wx.size() * sizeof(double), cudaMemcpyHostToDevice));
        CK(cudaMemcpy((void*)ob.yw, wy.data(), wy.size() * sizeof(double), cudaMemcpyHostToDevice));
        return AEO_OK;
    }

    // The current plane buffers (state of a radiating open set: at its outflow
    // points they hold radiated values the data cannot reproduce;
    // open_boundary_checkpoint, open_boundary.jl:1282-1305), FP64 in
    // aeo_set_open's layout (theta with its offset added back)
    aeo_status get_open_planes(double* xo, double* yo) override {
        if (!(open_x || open_y)) { fail("get_open_planes: no open face"); return AEO_ERR_STATE; }
        CK(cudaStreamSynchronize(st));
        const size_t nxp = ob_nxp(), nyp = ob_nyp();
        std::vector<R> hx(nxp), hy(nyp);
        CK(cudaMemcpy(hx.data(), ob.xp, nxp * sizeof(R), cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(hy.data(), ob.yp, nyp * sizeof(R), cudaMemcpyDeviceToHost));
        if (xo) for (size_t q = 0; q < nxp; ++q) xo[q] = (double)hx[q] + (q / (nxp / 4) == 3 ? th_off : 0.0);
        if (yo) for (size_t q = 0; q < nyp; ++q) yo[q] = (double)hy[q] + (q / (nyp / 4) == 3 ? th_off : 0.0);
        return AEO_OK;
    }

    // The planes back from a checkpoint (the buffers only: the data, weights
    // and modes are the set's own), the projection's boundary faces from them,
    // the state's halos refilled
    aeo_status set_open_planes(const double* xi, const double* yi) override {
        if (!(open_x || open_y)) { fail("set_open_planes: no open face"); return AEO_ERR_STATE; }
        if (!xi || !yi) { fail("set_open_planes: NULL plane array"); return AEO_ERR_ARGUMENT; }
        CK(cudaStreamSynchronize(st));
        const int H = AEO_H, NX = g.nx + 2 * H, NY = g.ny + 2 * H, NZ = g.nz + 2 * H, L = H + 1;
        const size_t nxp = ob_nxp(), nyp = ob_nyp();
        std::vector<R> hx(nxp), hy(nyp);
        for (size_t q = 0; q < nxp; ++q) hx[q] = R(xi[q] - (q / (nxp / 4) == 3 ? th_off : 0.0));
        for (size_t q = 0; q < nyp; ++q) hy[q] = R(yi[q] - (q / (nyp / 4) == 3 ? th_off : 0.0));
        std::vector<R> bw((size_t)g.ny * g.nz), be(bw.size()), bs((size_t)g.nx * g.nz), bn(bs.size());
        for (int k = 0; k < g.nz; ++k) {
            for (int j = 0; j < g.ny; ++j) {
                bw[(size_t)k * g.ny + j] = hx[(((size_t)0 * NZ + k + H) * NY + j + H) * L + H];
                be[(size_t)k * g.ny + j] = hx[(((size_t)1 * NZ + k + H) * NY + j + H) * L + 0];
            }
            for (int i = 0; i < g.nx; ++i) {
                bs[(size_t)k * g.nx + i] = hy[(((size_t)2 * NZ + k + H) * L + H) * NX + i + H];
                bn[(size_t)k * g.nx + i] = hy[(((size_t)3 * NZ + k + H) * L + 0) * NX + i + H];
            }
        }
        CK(cudaMemcpy((void*)ob.xp, hx.data(), nxp * sizeof(R), cudaMemcpyHostToDevice));
        CK(cudaMemcpy((void*)ob.yp, hy.data(), nyp * sizeof(R), cudaMemcpyHostToDevice));
        CK(cudaMemcpy((void*)ob.bw, bw.data(), bw.size() * sizeof(R), cudaMemcpyHostToDevice));
        CK(cudaMemcpy((void*)ob.be, be.data(), be.size() * sizeof(R), cudaMemcpyHostToDevice));
        CK(cudaMemcpy((void*)ob.bs, bs.data(), bs.size() * sizeof(R), cudaMemcpyHostToDevice));
        CK(cudaMemcpy((void*)ob.bn, bn.data(), bn.size() * sizeof(R), cudaMemcpyHostToDevice));
        R* f[4] = {P[cur][0], P[cur][1], P[cur][2], P[cur][3]};
        int l[4] = {LOC_FX, LOC_FY, LOC_FZ, LOC_C};
        if (aeo_status e = halo(f, l, 4)) return e;
        CK(cudaStreamSynchronize(st));
        return AEO_OK;
    }

    // The Orlanski history of a radiating set (hx [f][side][NZ][NY], hy
    // [f][side][NZ][NX], the interior layer at the last step start) and sc =
    // (history set, the last step's length): read (set = false) or written
    aeo_status open_state(double* hx, double* hy, double* sc, bool set) override {
        if (!ob_rad) { fail("open_state: no radiating open face"); return AEO_ERR_STATE; }
        if (!hx || !hy || !sc) { fail("open_state: NULL array"); return AEO_ERR_ARGUMENT; }
        CK(cudaStreamSynchronize(st));
        const size_t ntx = (size_t)8 * (g.nz + 2 * AEO_H) * (g.ny + 2 * AEO_H), nty = (size_t)8 * (g.nz + 2 * AEO_H) * (g.nx + 2 * AEO_H);
        std::vector<R> bx(ntx), by(nty);
        int ok = 0;
        double ldt = 0.0;
        if (set) {
            for (size_t q = 0; q < ntx; ++q) bx[q] = R(hx[q] - ((q / (ntx / 4)) == 3 ? th_off : 0.0));
            for (size_t q = 0; q < nty; ++q) by[q] = R(hy[q] - ((q / (nty / 4)) == 3 ? th_off : 0.0));
            ok = sc[0] != 0.0;
            ldt = sc[1];
            CK(cudaMemcpy(ob.xh, bx.data(), ntx * sizeof(R), cudaMemcpyHostToDevice));
            CK(cudaMemcpy(ob.yh, by.data(), nty * sizeof(R), cudaMemcpyHostToDevice));
            CK(cudaMemcpy(ob.hist_ok, &ok, sizeof(int), cudaMemcpyHostToDevice));
            CK(cudaMemcpy(ob.last_dt, &ldt, sizeof(double), cudaMemcpyHostToDevice));
        } else {
            CK(cudaMemcpy(bx.data(), ob.xh, ntx * sizeof(R), cudaMemcpyDeviceToHost));
            CK(cudaMemcpy(by.data(), ob.yh, nty * sizeof(R), cudaMemcpyDeviceToHost));
            CK(cudaMemcpy(&ok, ob.hist_ok, sizeof(int), cudaMemcpyDeviceToHost));
            CK(cudaMemcpy(&ldt, ob.last_dt, sizeof(double), cudaMemcpyDeviceToHost));
            for (size_t q = 0; q < ntx; ++q) hx[q] = (double)bx[q] + ((q / (ntx / 4)) == 3 ? th_off : 0.0);
            for (size_t q = 0; q < nty; ++q) hy[q] = (double)by[q] + ((q / (nty / 4)) == 3 ? th_off : 0.0);
            sc[0] = ok;
            sc[1] = ldt;
        }
        return AEO_OK;
    }

    aeo_status open_ledger(double* out) override {
        if (!ob_rad) { fail("open_ledger: no radiating open face"); return AEO_ERR_STATE; }
        CK(cudaStreamSynchronize(st));
        CK(cudaMemcpy(out, ob.led, 3 * sizeof(double), cudaMemcpyDeviceToHost));
        return AEO_OK;
    }

    // the radiating outflow's step-start, stage-start, update and combination
    unsigned ob_blocks() const {
        const long long n = 8LL * (g.nz + 2 * AEO_H) * ((g.ny + 2 * AEO_H) + (g.nx + 2 * AEO_H));
        return (unsigned)((n + 255) / 256);
    }
    // step_adaptive's keep of the radiated state (the planes, the boundary
    // faces and the Orlanski history) before a step, written back before a retry
    void* ob_kept[10] = {};
    aeo_status ob_keep(bool back) {
        const size_t ntx = (size_t)8 * (g.nz + 2 * AEO_H) * (g.ny + 2 * AEO_H), nty = (size_t)8 * (g.nz + 2 * AEO_H) * (g.nx + 2 * AEO_H);
        void* live[10] = {ob.xp, ob.yp, ob.bw, ob.be, ob.bs, ob.bn, ob.xh, ob.yh, ob.hist_ok, ob.last_dt};
        const size_t bytes[10] = {ob_nxp() * sizeof(R), ob_nyp() * sizeof(R), (size_t)g.ny * g.nz * sizeof(R),
                                  (size_t)g.ny * g.nz * sizeof(R), (size_t)g.nx * g.nz * sizeof(R),
                                  (size_t)g.nx * g.nz * sizeof(R), ntx * sizeof(R), nty * sizeof(R), sizeof(int),
                                  sizeof(double)};
        for (int q = 0; q < 10; ++q) {
            if (!ob_kept[q]) {
                unsigned char* b = nullptr;
                if (aeo_status e = alloc(&b, bytes[q])) return e;
                ob_kept[q] = b;
            }
            CK(cudaMemcpyAsync(back ? live[q] : ob_kept[q], back ? ob_kept[q] : live[q], bytes[q],
                               cudaMemcpyDeviceToDevice, st));
        }
        return AEO_OK;
    }

    size_t ob_nxp() const { return (size_t)8 * (g.nz + 2 * AEO_H) * (g.ny + 2 * AEO_H) * (AEO_H + 1); }
    size_t ob_nyp() const { return (size_t)8 * (g.nz + 2 * AEO_H) * (AEO_H + 1) * (g.nx + 2 * AEO_H); }
    aeo_status ob_prepare(int s_state) {
        CK(cudaMemcpyAsync(ob.xs, ob.xp, ob_nxp() * sizeof(R), cudaMemcpyDeviceToDevice, st));
        CK(cudaMemcpyAsync(ob.ys, ob.yp, ob_nyp() * sizeof(R), cudaMemcpyDeviceToDevice, st));
        R** f = P[s_state];
        ob_phase_kernel<R><<<ob_blocks(), 256, 0, st>>>(g, ob, f[0], f[1], f[2], f[3], &d_sc->dt);
        CKL();
        ob_hist_kernel<<<1, 1, 0, st>>>(ob.hist_ok, ob.last_dt, &d_sc->dt);
        CKL();
        return AEO_OK;
    }
    aeo_status ob_update(int s_in) {
        (void)s_in;
        CK(cudaMemcpyAsync(ob.xv, ob.xp, ob_nxp() * sizeof(R), cudaMemcpyDeviceToDevice, st));
        CK(cudaMemcpyAsync(ob.yv, ob.yp, ob_nyp() * sizeof(R), cudaMemcpyDeviceToDevice, st));
        CK(cudaMemcpyAsync(ob.xp, ob.xd, ob_nxp() * sizeof(R), cudaMemcpyDeviceToDevice, st));
        CK(cudaMemcpyAsync(ob.yp, ob.yd, ob_nyp() * sizeof(R), cudaMemcpyDeviceToDevice, st));
        ob_radiate_kernel<R><<<ob_blocks(), 256, 0, st>>>(g, ob, &d_sc->dt);
        CKL();
        ob_correct_kernel<R><<<1, 1024, 0, st>>>(g, ob);
        CKL();
        return AEO_OK;
    }
    aeo_status ob_combine(R ca, R cb) {
        ob_combine_kernel<R><<<296, 256, 0, st>>>(ob.xp, ob.xs, (long long)ob_nxp(), ca, cb);
        CKL();
        ob_combine_kernel<R><<<296, 256, 0, st>>>(ob.yp, ob.ys, (long long)ob_nyp(), ca, cb);
        CKL();
        return AEO_OK;
    }

    aeo_status make_tensor_maps() {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        CK(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q));
        if (!fn || q != cudaDriverEntryPointSuccess) { fail("cuTensorMapEncodeTiled is unavailable"); return AEO_ERR_CUDA; }
        auto encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
        const int HH = cfg.advection != AEO_ADV_CENTRED ? 3 : 2;
        pair = sizeof(R) == sizeof(float) && cfg.advection == AEO_ADV_CENTRED;
        cuuint64_t dims[3] = {(cuuint64_t)g.px, (cuuint64_t)g.py, (cuuint64_t)(g.nz + 2 * AEO_H)};
        cuuint64_t strides[2] = {(cuuint64_t)g.sy * sizeof(R), (cuuint64_t)g.sz * sizeof(R)};
        cuuint32_t box[3] = {pair ? 64u + 8u : 32u + 8u, (cuuint32_t)(8 + 2 * HH), 1};
        cuuint32_t es[3] = {1, 1, 1};
        CUtensorMapDataType dt = sizeof(R) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
        for (int s = 0; s < 4; ++s) {
            CUtensorMap* m[4] = {&tmaps[s].u, &tmaps[s].v, &tmaps[s].w, &tmaps[s].t};
            for (int f = 0; f < 4; ++f) {
                CUresult r = encode(m[f], dt, 3, (void*)P[s][f], dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                    CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
                if (r != CUDA_SUCCESS) { fail("cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")"); return AEO_ERR_CUDA; }
            }
        }
        return AEO_OK;
    }

    // ---- launch helpers -------------------------------------------------------------
    dim3 blk3() const { return dim3(32, 4, 2); }
    dim3 grd3() const { return dim3((g.nx + 31) / 32, (g.ny + 3) / 4, (g.nz + 1) / 2); }
    // 256-thread blocks over the interior, 16 / sizeof(R) x-consecutive cells a thread
    unsigned gvec() const { return (unsigned)((g.nin / Vec16<R>::N + 255) / 256); }

    aeo_status halo(R* const* f, const int* loc, int nf) {
        if (open_x || open_y) {
            for (int b = 0; b < nf; b += 4) {
                HaloSet<R> hs{};
                int pid[4] = {-1, -1, -1, -1};
                const int m = std::min(4, nf - b);
                for (int q = 0; q < m; ++q) {
                    hs.f[q] = f[b + q];
                    hs.loc[q] = loc[b + q];
                    for (int c = 0; c < 4; ++c)
                        for (int s4 = 0; s4 < 4; ++s4)
                            if (f[b + q] && f[b + q] == P[s4][c]) pid[q] = c;
                    // the boundary face of the normal velocity (interior index 0)
                    if (pid[q] == 0 && open_x) {
                        open_face_kernel<R><<<dim3((unsigned)((g.ny + 127) / 128), (unsigned)g.nz), 128, 0, st>>>(
                            g, f[b + q], ob, 0);
                        CKL();
                    }
                    if (pid[q] == 1 && open_y) {
                        open_face_kernel<R><<<dim3((unsigned)((g.nx + 127) / 128), (unsigned)g.nz), 128, 0, st>>>(
                            g, f[b + q], ob, 1);
                        CKL();
                    }
                }
                hs.nf = m;
                const long long n = shell_count(g);
                open_halo_fill_kernel<R><<<(unsigned)((n + 255) / 256), 256, 0, st>>>(
                    g, hs, ob, make_int4(pid[0], pid[1], pid[2], pid[3]));
                CKL();
            }
            return AEO_OK;
        }
        HaloSet<R> hs{};
        for (int q = 0; q < nf; ++q) { hs.f[q] = f[q]; hs.loc[q] = loc[q]; }
        hs.nf = nf;
        long long n = shell_count(g);
        halo_fill_kernel<R><<<(unsigned)((n + 255) / 256), 256, 0, st>>>(g, hs);
        CKL();
        return AEO_OK;
    }

    template <int ADV, bool SG, bool AN, bool UN>
    void launch_sweep_t(int s_in, const SweepArgs<R>& a) {
        if constexpr (ADV == 0 && sizeof(R) == sizeof(float)) {
            if (pair) {
                using PS = PairShape<SG>;
                // persistent: the SMs' worth of CTAs, each an equal range of (tile, level) items
                const int ntx = (g.nx + PS::TX - 1) / PS::TX, nty = (g.ny + PS::TY - 1) / PS::TY;
                const int items = ntx * nty * g.nz;
                const dim3 grid((unsigned)std::min(items, PS::CTAS_PER_SM * nsm));
                if constexpr (SG && UN) {
                    if (amd()) {
                        SweepArgs<R> b = a;
                        b.kofs = PS::KT_OFS;
                        cudaFuncSetAttribute(sweep_pair_kernel<SG, AN, UN, 1>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)PS::SMEM_AMD);
                        sweep_pair_kernel<SG, AN, UN, 1><<<grid, dim3(PS::TXT, PS::TY), PS::SMEM_AMD, st>>>(
                            tmaps[s_in], b, ntx, items, d_flag);
                        return;
                    }
                }
                if constexpr (SG && !AN && UN) {
                    if (tke()) {
                        SweepArgs<R> b = a;
                        b.kofs = PS::KT_OFS;
                        cudaFuncSetAttribute(sweep_pair_kernel<SG, AN, UN, 3>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)PS::SMEM_AMD);
                        sweep_pair_kernel<SG, AN, UN, 3><<<grid, dim3(PS::TXT, PS::TY), PS::SMEM_AMD, st>>>(
                            tmaps[s_in], b, ntx, items, d_flag);
                        return;
                    }
                }
                if constexpr (SG && UN) {
                    if (dyncl()) {
                        cudaFuncSetAttribute(sweep_pair_kernel<SG, AN, UN, 2>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)PS::SMEM);
                        sweep_pair_kernel<SG, AN, UN, 2><<<grid, dim3(PS::TXT, PS::TY), PS::SMEM, st>>>(
                            tmaps[s_in], a, ntx, items, d_flag);
                        return;
                    }
                }
                cudaFuncSetAttribute(sweep_pair_kernel<SG, AN, UN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)PS::SMEM);
                sweep_pair_kernel<SG, AN, UN><<<grid, dim3(PS::TXT, PS::TY), PS::SMEM, st>>>(tmaps[s_in], a, ntx,
                                                                                           items, d_flag);
                return;
            }
        }
        if constexpr (ADV > 0 && !SG && !AN && UN && sizeof(R) == sizeof(float)) {
            // FP32 WENO without a closure: cell pairs, every face once
            using WS = WPairShape;
            const dim3 grid((g.nx + WS::TX - 1) / WS::TX, (g.ny + WS::TY - 1) / WS::TY, (g.nz + wchunk - 1) / wchunk);
            cudaFuncSetAttribute(sweep_wpair_kernel<ADV>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)WS::SMEM);
            sweep_wpair_kernel<ADV><<<grid, dim3(WS::TXT, WS::TY), WS::SMEM, st>>>(tmaps[s_in], a, wchunk, d_flag);
            return;
        }
        using TS = TileShape<R, ADV, SG>;
        dim3 grid((g.nx + TS::TX - 1) / TS::TX, (g.ny + TS::TY - 1) / TS::TY, (g.nz + kchunk - 1) / kchunk);
        if constexpr (SG && UN) {
            if (amd()) {
                SweepArgs<R> b = a;
                b.kofs = TS::KT_OFS;
                cudaFuncSetAttribute(sweep_tile_kernel<R, ADV, SG, AN, UN, 1>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TS::SMEM_AMD);
                sweep_tile_kernel<R, ADV, SG, AN, UN, 1><<<grid, dim3(TS::TX, TS::TY), TS::SMEM_AMD, st>>>(
                    tmaps[s_in], b, kchunk, d_flag);
                return;
            }
        }
        if constexpr (SG && !AN && UN) {
            if (tke()) {
                SweepArgs<R> b = a;
                b.kofs = TS::KT_OFS;
                cudaFuncSetAttribute(sweep_tile_kernel<R, ADV, SG, AN, UN, 3>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TS::SMEM_AMD);
                sweep_tile_kernel<R, ADV, SG, AN, UN, 3><<<grid, dim3(TS::TX, TS::TY), TS::SMEM_AMD, st>>>(
                    tmaps[s_in], b, kchunk, d_flag);
                return;
            }
        }
        if constexpr (SG && UN) {
            if (dyncl()) {
                cudaFuncSetAttribute(sweep_tile_kernel<R, ADV, SG, AN, UN, 2>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TS::SMEM);
                sweep_tile_kernel<R, ADV, SG, AN, UN, 2><<<grid, dim3(TS::TX, TS::TY), TS::SMEM, st>>>(
                    tmaps[s_in], a, kchunk, d_flag);
                return;
            }
        }
        const size_t sm = TS::SMEM;
        cudaFuncSetAttribute(sweep_tile_kernel<R, ADV, SG, AN, UN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        sweep_tile_kernel<R, ADV, SG, AN, UN><<<grid, dim3(TS::TX, TS::TY), sm, st>>>(tmaps[s_in], a, kchunk, d_flag);
    }

    aeo_status launch_sweep(int s_in, const SweepArgs<R>& a) {
        const int adv = cfg.advection;
        if (anel) {
            if (uni) { if (sgs) launch_sweep_t<0, true, true, true>(s_in, a); else launch_sweep_t<0, false, true, true>(s_in, a); }
            else { if (sgs) launch_sweep_t<0, true, true, false>(s_in, a); else launch_sweep_t<0, false, true, false>(s_in, a); }
        } else if (!uni) {
            if (sgs) launch_sweep_t<0, true, false, false>(s_in, a); else launch_sweep_t<0, false, false, false>(s_in, a);
        } else if (adv == AEO_ADV_CENTRED) {
            if (sgs) launch_sweep_t<0, true, false, true>(s_in, a); else launch_sweep_t<0, false, false, true>(s_in, a);
        } else if (adv == AEO_ADV_WENO_JS5) {
            if (sgs) launch_sweep_t<1, true, false, true>(s_in, a); else launch_sweep_t<1, false, false, true>(s_in, a);
        } else {
            if (sgs) launch_sweep_t<2, true, false, true>(s_in, a); else launch_sweep_t<2, false, false, true>(s_in, a);
        }
        CKL();
        return AEO_OK;
    }

    // The pressure solve from the source (src == nullptr: divergence of Q) into phi.
    aeo_status solve(const R* src) {
        if (pcg) {
            const unsigned gb = (unsigned)((g.nin + 255) / 256);
            if (src) to_f64_kernel<R><<<gb, 256, 0, st>>>(g.nin, src, mg_b);
            else if (anel && uni) cc_div_kernel<R, true, true><<<gb, 256, 0, st>>>(g, Q[0], Q[1], Q[2], apx, apy, apz, mg_b);
            else if (anel) cc_div_kernel<R, true, false><<<gb, 256, 0, st>>>(g, Q[0], Q[1], Q[2], apx, apy, apz, mg_b);
            else if (!uni) cc_div_kernel<R, false, false><<<gb, 256, 0, st>>>(g, Q[0], Q[1], Q[2], apx, apy, apz, mg_b);
            else cc_div_kernel<R><<<gb, 256, 0, st>>>(g, Q[0], Q[1], Q[2], apx, apy, apz, mg_b,
                                                       open_x ? ob.bw : nullptr, open_x ? ob.be : nullptr,
                                                       open_y ? ob.bs : nullptr, open_y ? ob.bn : nullptr);
            CKL();
            mark(AEO_K_DIV_FFTX);
            if (aeo_status e = aeo_mg_enqueue(mg, st)) {
                fail(std::string("the MG-PCG pressure solve: ") + aeo_mg_last_error(mg));
                return e;
            }
            mark(AEO_K_ZSOLVE);
            if (src) {
                from_f64_kernel<R><<<gb, 256, 0, st>>>(g.nin, mg_x, phi);
                CKL();
            }
            return AEO_OK;
        }
        const int M = g.nx / 2;
        size_t smx = (size_t)rows_x * xrow(M) * sizeof(cplx<R>);
        unsigned gx = (unsigned)((g.ny * (long long)g.nz + rows_x - 1) / rows_x);
        const int lgx = ilog2i(M), lgy = ilog2i(g.ny), lgz = ilog2i(g.nz);
        if (src) {
            AEO_FFT_LEN(lgx, (src_fftx_kernel<R, LG><<<gx, FFT_THREADS(R), smx + roots_smem<R>(LG), st>>>(
                                 g, src, S, tw, NT, rows_x)));
        } else if (lgx >= 7 && lgx <= 9) {
            // the divergence formed in the r2c's staging (it never goes to memory)
            const int dv = (anel ? 2 : 1) | (uni ? 0 : 4);
#define AEO_SRC_DIV(D) AEO_FFT_LEN(lgx, (src_fftx_kernel<R, LG, D><<<gx, FFT_THREADS(R), smx + roots_smem<R>(LG), st>>>( \
                                             g, nullptr, S, tw, NT, rows_x, Q[0], Q[1], Q[2])))
            switch (dv) {
                case 1: AEO_SRC_DIV(1); break;
                case 2: AEO_SRC_DIV(2); break;
                case 5: AEO_SRC_DIV(5); break;
                default: AEO_SRC_DIV(6); break;
            }
#undef AEO_SRC_DIV
        } else {
            // the divergence into phi (overwritten by the c2r at the end), then its r2c
            if (anel && uni) div_kernel<R, true, true><<<gvec(), 256, 0, st>>>(g, Q[0], Q[1], Q[2], phi);
            else if (anel) div_kernel<R, true, false><<<gvec(), 256, 0, st>>>(g, Q[0], Q[1], Q[2], phi);
            else if (uni) div_kernel<R, false, true><<<gvec(), 256, 0, st>>>(g, Q[0], Q[1], Q[2], phi);
            else div_kernel<R, false, false><<<gvec(), 256, 0, st>>>(g, Q[0], Q[1], Q[2], phi);
            CKL();
            AEO_FFT_LEN(lgx, (src_fftx_kernel<R, LG><<<gx, FFT_THREADS(R), smx + roots_smem<R>(LG), st>>>(
                                 g, phi, S, tw, NT, rows_x)));
        }
        CKL();
        mark(AEO_K_DIV_FFTX);
        const int Mh = M + 1;
        dim3 gy((Mh + tpx_y - 1) / tpx_y, g.nz);
        size_t smy = (size_t)tpx_y * g.ny * sizeof(cplx<R>);
        AEO_FFT_LEN(lgy, (ffty_kernel<R, 0, LG><<<gy, FFT_THREADS(R), smy + roots_smem<R>(LG), st>>>(g, S, tw, NT, tpx_y)));
        CKL();
        mark(AEO_K_FFTY);
        if (cfg.solver == AEO_SOLVER_FFT) {
            dim3 gz((Mh + tpx_z - 1) / tpx_z, g.ny);
            size_t smz = (size_t)tpx_z * g.nz * sizeof(cplx<R>);
            double nrm = 1.0 / ((double)g.nx * g.ny * g.nz);
            AEO_FFT_LEN(lgz, (fftz_solve_kernel<R, LG><<<gz, FFT_THREADS(R), smz + roots_smem<R>(LG), st>>>(
                                 g, S, tw, NT, tpx_z, kx2, ky2, kz2, nrm)));
        } else {
            size_t smt = thomas_smem(g, true);
            if (smt > 48 * 1024)
                cudaFuncSetAttribute(thomas_kernel<R, true, R, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)smt);
            // d' in place in S; the factors m and c' from the tables made at set-up
            R* ftab = reinterpret_cast<R*>(cps);
            const long long ns = (long long)(g.nx / 2 + 1) * g.ny * g.nz;
            thomas_kernel<R, true, R, true><<<thomas_blocks(g), 32, smt, st>>>(g, S, S, ftab + ns, cc, ftab);
        }
        CKL();
        mark(AEO_K_ZSOLVE);
        AEO_FFT_LEN(lgy, (ffty_kernel<R, 1, LG><<<gy, FFT_THREADS(R), smy + roots_smem<R>(LG), st>>>(g, S, tw, NT, tpx_y)));
        CKL();
        mark(AEO_K_FFTY);
        R scale = cfg.solver == AEO_SOLVER_FFT ? R(1) : R(1.0 / ((double)g.nx * g.ny));
        AEO_FFT_LEN(lgx, (ifftx_kernel<R, LG><<<gx, FFT_THREADS(R), smx + roots_smem<R>(LG), st>>>(
                             g, S, phi, tw, NT, rows_x, scale)));
        CKL();
        mark(AEO_K_IFFTX);
        return AEO_OK;
    }

    aeo_status correct(R** out, int stage, R ca, R cb, const double* dtp, int s_u0) {
        R** u0 = P[s_u0];
        if (pcg) {
            if (uni)
                cc_correct_kernel<R, true><<<(unsigned)((g.nin + 255) / 256), 256, 0, st>>>(
                    g, Q[0], Q[1], Q[2], mg_x, apx, apy, apz, u0[0], u0[1], u0[2], out[0], out[1], out[2], pres, dtp,
                    ca, cb, stage, open_x ? ob.bw : nullptr, open_y ? ob.bs : nullptr);
            else
                cc_correct_kernel<R, false><<<(unsigned)((g.nin + 255) / 256), 256, 0, st>>>(
                    g, Q[0], Q[1], Q[2], mg_x, apx, apy, apz, u0[0], u0[1], u0[2], out[0], out[1], out[2], pres, dtp,
                    ca, cb, stage);
            CKL();
            return AEO_OK;
        }
        if (uni)
            correct_kernel<R, true><<<gvec(), 256, 0, st>>>(g, Q[0], Q[1], Q[2], phi, u0[0], u0[1], u0[2], out[0],
                                                               out[1], out[2], pres, dtp, ca, cb, stage);
        else
            correct_kernel<R, false><<<gvec(), 256, 0, st>>>(g, Q[0], Q[1], Q[2], phi, u0[0], u0[1], u0[2], out[0],
                                                                out[1], out[2], pres, dtp, ca, cb, stage);
        CKL();
        return AEO_OK;
    }

    // One projected substage: set s_in -> set s_out; stage c(x, s) = ca*s + cb*x
    // with the step-start set s_u0 (stages 2, 3).
    aeo_status substage(int s_in, int s_out, int s_u0, int stage, R ca, R cb) {
        R** out = P[s_out];
        if (ob_rad) {   // the stage-start interior layers of the radiating faces
            ob_mark_kernel<R><<<ob_blocks(), 256, 0, st>>>(g, ob, P[s_in][0], P[s_in][1], P[s_in][2], P[s_in][3]);
            CKL();
        }
        SweepArgs<R> a{};
        a.g = g;
        a.u = P[s_in][0]; a.v = P[s_in][1]; a.w = P[s_in][2]; a.th = P[s_in][3];
        a.nut = nullptr;
        a.th0 = P[s_u0][3];
        a.us = Q[0]; a.vs = Q[1]; a.ws = Q[2];
        a.th_out = out[3];
        a.dtp = &d_sc->dt;
        a.ca = ca; a.cb = cb; a.stage = stage;
        a.nu = R(cfg.nu); a.gacc = R(cfg.g); a.theta0 = R(cfg.theta0); a.fcor = R(cfg.f_coriolis);
        a.bref = R(cfg.theta0 - th_off);
        a.pr_t = R(cfg.pr_t);
        // the AMD closure brings its own kappa_t (the flux takes it unscaled)
        // and a buoyancy term with g / theta0
        a.inv_prt = own_kappa() ? R(1) : R(1.0 / cfg.pr_t);
        a.cs2 = d_cs2;
        a.cs2f = d_cs2f;
        a.dyn_d2 = dyn_d2;
        if (dyn())
            if (aeo_status e = enqueue_dynamic(P[s_in])) return e;
        a.flux_bot = R(cfg.flux_bot); a.flux_top = R(cfg.flux_top);
        a.sp_alpha = R(cfg.sponge_alpha); a.sp_zstart = R(cfg.sponge_zstart);
        a.c_s = R(cfg.c_s);
        double ztop = cfg.z0 + cfg.lz;
        a.sp_inv = R(1.0 / (ztop - cfg.sponge_zstart));
        if (aeo_status e = launch_sweep(s_in, a)) return e;
        if (ibm_mask) {
            ibm_kernel<R><<<(unsigned)((g.nin + 255) / 256), 256, 0, st>>>(g, Q[0], Q[1], Q[2], ibm_mask, &d_sc->dt,
                                                                         ibm_tau);
            CKL();
        }
        mark(AEO_K_SWEEP);
        if (ob_rad)     // 7c. open boundaries: data, radiation, mass-flux correction
            if (aeo_status e = ob_update(s_in)) return e;
        if (aeo_status e = solve(nullptr)) return e;
        if (aeo_status e = correct(out, stage, ca, cb, &d_sc->dt, s_u0)) return e;
        if (ob_rad && stage)   // the buffers combined like the fields (combine_open_boundaries!)
            if (aeo_status e = ob_combine(ca, cb)) return e;
        mark(AEO_K_CORRECT);
        R* f[4] = {out[0], out[1], out[2], out[3]};
        int l[4] = {LOC_FX, LOC_FY, LOC_FZ, LOC_C};
        aeo_status hs = halo(f, l, 4);
        mark(AEO_K_HALO);
        return hs;
    }

    aeo_status enqueue_pick(int s_state) {
        R** in = P[s_state];
        if (dyn())
            if (aeo_status e = enqueue_dynamic(in)) return e;
        if (uni) {
            if (sgs) cfl_levels_kernel<R, true, true><<<g.nz, 256, 0, st>>>(g, in[0], in[1], in[2], in[3], R(cfg.c_s), R(cfg.pr_t), d_cs2, dyn_d2, d_part, d_cs2f);
            else cfl_levels_kernel<R, true, false><<<g.nz, 256, 0, st>>>(g, in[0], in[1], in[2], in[3], R(cfg.c_s), R(cfg.pr_t), d_cs2, dyn_d2, d_part, d_cs2f);
        } else {
            if (sgs) cfl_levels_kernel<R, false, true><<<g.nz, 256, 0, st>>>(g, in[0], in[1], in[2], in[3], R(cfg.c_s), R(cfg.pr_t), d_cs2, dyn_d2, d_part, d_cs2f);
            else cfl_levels_kernel<R, false, false><<<g.nz, 256, 0, st>>>(g, in[0], in[1], in[2], in[3], R(cfg.c_s), R(cfg.pr_t), d_cs2, dyn_d2, d_part, d_cs2f);
        }
        CKL();
        dt_pick_kernel<<<1, 32, 0, st>>>(g, cflp, d_part, d_sc);
        CKL();
        return AEO_OK;
    }

    // One RK3 step from set c to set c^1 (src/Simulations.jl:854-904).
    aeo_status enqueue_rk3(int c, bool pick) {
        if (pick)
            if (aeo_status e = enqueue_pick(c)) return e;
        const R inv3 = R(1) / R(3), two3 = R(2) * inv3;
        if (ob_rad)
            if (aeo_status e = ob_prepare(c)) return e;
        if (aeo_status e = substage(c, 2, c, 0, R(0), R(0))) return e;
        if (aeo_status e = substage(2, 3, c, 1, R(0.75), R(0.25))) return e;
        if (aeo_status e = substage(3, c ^ 1, c, 1, inv3, two3)) return e;
        return commit_sgs(c ^ 1);
    }

    // the closure's once-per-step commit (advance_sgs!), after the projection
    aeo_status commit_sgs(int s_state) {
        if (!lag() && !tke()) return AEO_OK;
        aeo_status e = lag() ? enqueue_lag_commit(P[s_state]) : enqueue_tke_commit(P[s_state]);
        mark(AEO_K_SGS);
        return e;
    }

    // One step on the stream: the captured graph (solver = PCG: with the three
    // CG solves inside it as conditional WHILE nodes).
    aeo_status launch_step(bool pick) {
        cudaGraphExec_t ge;
        if (aeo_status e = graph_for(pick, &ge)) return e;
        if (pcg)
            if (aeo_status e = aeo_mg_order_before(mg, st)) {
                fail(std::string("the MG-PCG pressure solve: ") + aeo_mg_last_error(mg));
                return e;
            }
        CK(cudaGraphLaunch(ge, st));
        return AEO_OK;
    }

    aeo_status graph_for(bool pick, cudaGraphExec_t* out) {
        cudaGraphExec_t& ge = gexec[pick ? 1 : 0][cur];
        if (!ge) {
            // PCG: the handle's set-up work is complete before its nodes are
            // captured; the conditional-node capture of its CG loop runs in
            // relaxed mode, as the handle's own solve graph
            if (pcg) CK(cudaDeviceSynchronize());
            CK(cudaStreamBeginCapture(st, pcg ? cudaStreamCaptureModeRelaxed : cudaStreamCaptureModeThreadLocal));
            aeo_status e = enqueue_rk3(cur, pick);
            cudaGraph_t gr = nullptr;
            cudaError_t ce = cudaStreamEndCapture(st, &gr);
            if (e) { if (gr) cudaGraphDestroy(gr); return e; }
            if (ce != cudaSuccess) { fail(std::string("graph capture: ") + cudaGetErrorString(ce)); return AEO_ERR_CUDA; }
            cudaError_t ie = cudaGraphInstantiate(&ge, gr, 0);
            cudaGraphDestroy(gr);
            if (ie != cudaSuccess) { ge = nullptr; fail(std::string("graph instantiate: ") + cudaGetErrorString(ie)); return AEO_ERR_CUDA; }
        }
        *out = ge;
        return AEO_OK;
    }

    // The graph of n steps: WHILE(pairs left) { step cur -> cur^1; step cur^1 -> cur }.
    aeo_status multi_graph_for(cudaGraphExec_t* out) {
        cudaGraphExec_t& ge = gmulti[cur];
        if (!ge) {
            if (pcg) CK(cudaDeviceSynchronize());   // as graph_for: the handle's set-up is complete
            CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed));
            aeo_status e = AEO_OK;
            cudaError_t ce = cudaSuccess;
            cudaStreamCaptureStatus cs;
            cudaGraph_t g0 = nullptr;
            const cudaGraphNode_t* deps = nullptr;
            size_t nd = 0;
            cudaGraphConditionalHandle h{};
            cudaGraphNode_t node{};
            ce = cudaStreamGetCaptureInfo(st, &cs, nullptr, &g0, nullptr, nullptr);
            if (ce == cudaSuccess) ce = cudaGraphConditionalHandleCreate(&h, g0, 0, cudaGraphCondAssignDefault);
            if (ce == cudaSuccess) {
                steps_begin_kernel<<<1, 1, 0, st>>>(d_steps, h);
                ce = cudaGetLastError();
            }
            if (ce == cudaSuccess) ce = cudaStreamGetCaptureInfo(st, &cs, nullptr, &g0, &deps, &nd);
            cudaGraphNodeParams cp = {};
            if (ce == cudaSuccess) {
                cp.type = cudaGraphNodeTypeConditional;
                cp.conditional.handle = h;
                cp.conditional.type = cudaGraphCondTypeWhile;
                cp.conditional.size = 1;
                std::vector<cudaGraphNode_t> dv(deps, deps + nd);
                ce = cudaGraphAddNode(&node, g0, dv.data(), dv.size(), &cp);
            }
            if (ce == cudaSuccess)
                ce = cudaStreamBeginCaptureToGraph(st_loop, cp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                                   cudaStreamCaptureModeRelaxed);
            if (ce == cudaSuccess) {
                // the body: every launch of the two steps goes to st_loop
                std::swap(st, st_loop);
                e = enqueue_rk3(cur, false);
                if (!e) e = enqueue_rk3(cur ^ 1, false);
                if (!e) {
                    steps_next_kernel<<<1, 1, 0, st>>>(d_steps, h);
                    if (cudaGetLastError() != cudaSuccess) { fail("multi-step graph: loop kernel"); e = AEO_ERR_CUDA; }
                }
                std::swap(st, st_loop);
                cudaGraph_t bg = nullptr;
                cudaError_t be = cudaStreamEndCapture(st_loop, &bg);
                if (be != cudaSuccess && !e) { fail(std::string("multi-step body capture: ") + cudaGetErrorString(be)); e = AEO_ERR_CUDA; }
                if (!e) ce = cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies);
            }
            cudaGraph_t gr = nullptr;
            cudaError_t ee = cudaStreamEndCapture(st, &gr);
            if (!e && ce != cudaSuccess) { fail(std::string("multi-step graph: ") + cudaGetErrorString(ce)); e = AEO_ERR_CUDA; }
            if (!e && ee != cudaSuccess) { fail(std::string("multi-step graph capture: ") + cudaGetErrorString(ee)); e = AEO_ERR_CUDA; }
            if (e) { if (gr) cudaGraphDestroy(gr); return e; }
            cudaError_t ie = cudaGraphInstantiate(&ge, gr, 0);
            cudaGraphDestroy(gr);
            if (ie != cudaSuccess) { ge = nullptr; fail(std::string("multi-step graph instantiate: ") + cudaGetErrorString(ie)); return AEO_ERR_CUDA; }
        }
        *out = ge;
        return AEO_OK;
    }

    aeo_status step_rk3(double dt, int n, bool sync) override {
        if (aeo_status e = sgs_ready()) return e;
        set_scalar_kernel<<<1, 1, 0, st>>>(&d_sc->dt, dt);
        CKL();
        if (n >= 2) {
            // the pairs of steps as one launch of the multi-step graph
            cudaGraphExec_t ge;
            if (aeo_status e = multi_graph_for(&ge)) return e;
            steps_set_kernel<<<1, 1, 0, st>>>(d_steps, n / 2);
            CKL();
            if (pcg)
                if (aeo_status e = aeo_mg_order_before(mg, st)) {
                    fail(std::string("the MG-PCG pressure solve: ") + aeo_mg_last_error(mg));
                    return e;
                }
            CK(cudaGraphLaunch(ge, st));
            n -= 2 * (n / 2);   // the state is back in set cur
        }
        for (int s = 0; s < n; ++s) {
            if (aeo_status e = launch_step(false)) return e;
            cur ^= 1;
        }
        if (sync) {
            CK(cudaStreamSynchronize(st));
            return check_finite();
        }
        return AEO_OK;
    }

    aeo_status step_euler(double dt, int n) override {
        if (aeo_status e = sgs_ready()) return e;
        set_scalar_kernel<<<1, 1, 0, st>>>(&d_sc->dt, dt);
        CKL();
        for (int s = 0; s < n; ++s) {
            if (ob_rad)
                if (aeo_status e = ob_prepare(cur)) return e;
            if (aeo_status e = substage(cur, cur ^ 1, cur, 0, R(0), R(0))) return e;
            if (aeo_status e = commit_sgs(cur ^ 1)) return e;
            cur ^= 1;
        }
        CK(cudaStreamSynchronize(st));
        return check_finite();
    }

    void set_cfl(const aeo_cfl* c) {
        CflParams p{};
        p.c_adv = c->c_advective; p.c_diff = c->c_diffusive; p.c_buoy = c->c_buoyancy; p.c_cor = c->c_coriolis;
        p.dt_min = c->dt_min; p.dt_max = c->dt_max; p.growth = c->growth_max;
        p.nu = cfg.nu; p.pr_t = cfg.pr_t; p.fcor = cfg.f_coriolis; p.gacc = cfg.g; p.theta0 = cfg.theta0;
        p.th_off = th_off;
        p.dz_min = dz_min; p.sgs = sgs; p.anel = anel;
        p.buoy = anel ? (cfg.g != 0.0) : (cfg.theta0 != 0.0);
        if (!cflp_set || std::memcmp(&p, &cflp, sizeof(p)) != 0) {
            cflp = p;
            cflp_set = true;
            for (auto& e : gexec[1])
                if (e) { cudaGraphExecDestroy(e); e = nullptr; }
        }
    }

    aeo_status read_scalars(StepScalars* h) {
        CK(cudaMemcpyAsync(h, d_sc, sizeof(StepScalars), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        return AEO_OK;
    }

    // the post-step guard of set s: (finite, max |div|, max speed)
    aeo_status guard(int s, bool* finite, double* div, double* speed) {
        R** in = P[s];
        if (anel) {
            if (uni) guard_levels_kernel<R, true, true><<<g.nz, 256, 0, st>>>(g, in[0], in[1], in[2], in[3], pres, d_part);
            else guard_levels_kernel<R, true, false><<<g.nz, 256, 0, st>>>(g, in[0], in[1], in[2], in[3], pres, d_part);
        } else {
            if (uni) guard_levels_kernel<R, false, true><<<g.nz, 256, 0, st>>>(g, in[0], in[1], in[2], in[3], pres, d_part);
            else guard_levels_kernel<R, false, false><<<g.nz, 256, 0, st>>>(g, in[0], in[1], in[2], in[3], pres, d_part);
        }
        CKL();
        std::vector<double> h(3 * (size_t)g.nz);
        CK(cudaMemcpyAsync(h.data(), d_part, h.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        bool fin = true;
        double dm = 0, sm = 0;
        for (int k = 0; k < g.nz; ++k) {
            fin = fin && h[3 * k] == 0.0;
            dm = std::max(dm, h[3 * k + 1]);
            sm = std::max(sm, h[3 * k + 2]);
        }
        *finite = fin;
        *div = dm;
        *speed = sm;
        return AEO_OK;
    }

    aeo_status cfl(const aeo_cfl* c, double dt_prev, aeo_adaptive_stats* out) override {
        if (aeo_status e = sgs_ready()) return e;
        set_cfl(c);
        set_scalar_kernel<<<1, 1, 0, st>>>(&d_sc->dt_prev, dt_prev > 0 ? dt_prev : 0.0);
        CKL();
        if (aeo_status e = enqueue_pick(cur)) return e;
        StepScalars h;
        if (aeo_status e = read_scalars(&h)) return e;
        std::memset(out, 0, sizeof(*out));
        out->dt = h.dt;
        out->limiter = h.limiter;
        out->advective_rate = h.rate;
        out->nut_max = h.nut_max;
        out->brunt_vaisala = h.N;
        return AEO_OK;
    }

    // step_adaptive! (src/TimeIntegration.jl:808-938): CFL pick on the
    // device, the step, the guard; on a failed guard the state (set cur,
    // untouched) is kept and the step retried with half the dt.
    aeo_status step_adaptive(const aeo_cfl* c, int n, double* dt_prev_io, aeo_adaptive_stats* stats) override {
        if (aeo_status e = sgs_ready()) return e;
        set_cfl(c);
        double dt_prev = (dt_prev_io && *dt_prev_io > 0) ? *dt_prev_io : 0.0;
        set_scalar_kernel<<<1, 1, 0, st>>>(&d_sc->dt_prev, dt_prev);
        CKL();
        aeo_adaptive_stats acc{};
        for (int s = 0; s < n; ++s) {
            // the closure's memory as committed before the step: a retry starts from it
            if (lag()) CK(cudaMemcpyAsync(d_lag_state + 2, d_lag_state, 2 * sizeof(int), cudaMemcpyDeviceToDevice, st));
            if (tke()) CK(cudaMemcpyAsync(d_tke_keep, d_tke, padded_count() * sizeof(R), cudaMemcpyDeviceToDevice, st));
            // a radiating open set's planes and history: the step rewrites them in place
            if (ob_rad)
                if (aeo_status e = ob_keep(false)) return e;
            if (aeo_status e = launch_step(true)) return e;
            StepScalars h;
            if (aeo_status e = read_scalars(&h)) return e;
            double dt = h.dt;
            int retries = 0;
            while (true) {
                bool fin;
                double dv, sp;
                if (aeo_status e = guard(cur ^ 1, &fin, &dv, &sp)) return e;
                bool ok = fin && std::isfinite(dv) && dv <= c->divergence_tol && sp <= c->max_velocity;
                int flag = 0;
                CK(cudaMemcpyAsync(&flag, d_flag, sizeof(int), cudaMemcpyDeviceToHost, st));
                CK(cudaStreamSynchronize(st));
                if (flag & AEO_ERR_FLAG_TMA) { fail("a tile load did not complete within its wait limit"); return AEO_ERR_CUDA; }
                if (ok) {
                    acc.max_divergence = dv;
                    acc.max_speed = sp;
                    break;
                }
                if (lag()) {
                    // the committed memory and its coefficient again (the failed commit wrote cs2f)
                    CK(cudaMemcpyAsync(d_lag_state, d_lag_state + 2, 2 * sizeof(int), cudaMemcpyDeviceToDevice, st));
                    if (aeo_status e = lag_refresh()) return e;
                }
                if (tke()) CK(cudaMemcpyAsync(d_tke, d_tke_keep, padded_count() * sizeof(R), cudaMemcpyDeviceToDevice, st));
                if (ob_rad)
                    if (aeo_status e = ob_keep(true)) return e;
                if (retries >= c->max_retries) {
                    fail(std::string("step_adaptive: step failed (") + (!fin ? "nonfinite" : (dv > c->divergence_tol ? "divergence" : "velocity")) +
                         ") after " + std::to_string(retries) + " retries; the state is the one before the step");
                    return AEO_ERR_NUMERICAL;
                }
                double dt_new = std::max(dt / 2, c->dt_min);
                if (dt_new == dt) {
                    fail("step_adaptive: step failed at dt_min; the state is the one before the step");
                    return AEO_ERR_NUMERICAL;
                }
                dt = dt_new;
                ++retries;
                set_scalar_kernel<<<1, 1, 0, st>>>(&d_sc->dt, dt);
                CKL();
                if (aeo_status e = launch_step(false)) return e;
            }
            cur ^= 1;
            set_scalar_kernel<<<1, 1, 0, st>>>(&d_sc->dt_prev, dt);
            CKL();
            acc.dt = dt;
            acc.t_advanced += dt;
            acc.retries += retries;
            acc.limiter = retries ? 8 : h.limiter;
            acc.advective_rate = h.rate;
            acc.nut_max = h.nut_max;
            acc.brunt_vaisala = h.N;
        }
        if (dt_prev_io && n > 0) *dt_prev_io = acc.dt;
        if (stats) *stats = acc;
        return AEO_OK;
    }

    aeo_status profile_step(double dt, double* ms, int ncls) override {
        if (aeo_status e = sgs_ready()) return e;
        set_scalar_kernel<<<1, 1, 0, st>>>(&d_sc->dt, dt);
        CKL();
        profiling = true;
        marks.clear();
        mark(-1);
        aeo_status e = enqueue_rk3(cur, false);
        profiling = false;
        if (e) return e;
        CK(cudaStreamSynchronize(st));
        cur ^= 1;
        for (int c = 0; c < ncls; ++c) ms[c] = 0.0;
        for (size_t q = 1; q < marks.size(); ++q) {
            float t = 0.f;
            cudaEventElapsedTime(&t, marks[q - 1].second, marks[q].second);
            int c = marks[q].first;
            if (c >= 0 && c < ncls) ms[c] += (double)t;
        }
        for (auto& m : marks) cudaEventDestroy(m.second);
        marks.clear();
        return check_finite();
    }

    aeo_status check_finite() {
        // one resident wave: every CTA loops over its share of each field
        const long long vecs = g.nin / Vec16<R>::N;
        const unsigned nb = (unsigned)std::min<long long>((vecs + 255) / 256, (long long)fin_per_sm * nsm);
        finite_check_kernel<R><<<nb, 256, 0, st>>>(g, P[cur][0], P[cur][1], P[cur][2], P[cur][3], d_flag);
        CKL();
        int h = 0;
        CK(cudaMemcpyAsync(&h, d_flag, sizeof(int), cudaMemcpyDeviceToHost, st));
        CK(cudaMemsetAsync(d_flag, 0, sizeof(int), st));
        CK(cudaStreamSynchronize(st));
        if (h & AEO_ERR_FLAG_TMA) { fail("a tile load did not complete within its wait limit"); return AEO_ERR_CUDA; }
        if (h) { fail("non-finite value in the state after the step"); return AEO_ERR_NUMERICAL; }
        return AEO_OK;
    }

    R* field_ptr(int id, int* padded, int* loc) {
        *padded = 1;
        switch (id) {
            case AEO_FIELD_U: *loc = LOC_FX; return P[cur][0];
            case AEO_FIELD_V: *loc = LOC_FY; return P[cur][1];
            case AEO_FIELD_W: *loc = LOC_FZ; return P[cur][2];
            case AEO_FIELD_THETA: *loc = LOC_C; return P[cur][3];
            case AEO_FIELD_P: *padded = 0; *loc = -1; return pres;
            case AEO_FIELD_NUT: *loc = -1; return nut;
            default: return nullptr;
        }
    }

    aeo_status set_field(int id, const double* host) override { return set_field_t<double>(id, host); }
    aeo_status get_field(int id, double* host) override { return get_field_t<double>(id, host); }
    aeo_status set_field_f32(int id, const float* host) override { return set_field_t<float>(id, host); }
    aeo_status get_field_f32(int id, float* host) override { return get_field_t<float>(id, host); }

    // the host array (FP64 or FP32, the reference storage layout) through the
    // staging buffer into the device field, and back
    template <typename S>
    aeo_status set_field_t(int id, const S* host) {
        int padded, loc;
        R* d = field_ptr(id, &padded, &loc);
        if (!d) { fail("set_field: unknown or unavailable field"); return AEO_ERR_ARGUMENT; }
        S* stage = reinterpret_cast<S*>(d_stage);
        CK(cudaMemcpyAsync(stage, host, host_n * sizeof(S), cudaMemcpyHostToDevice, st));
        dim3 gb((g.nx + 127) / 128, g.ny, g.nz);
        unpack_host_kernel<R, S><<<gb, 128, 0, st>>>(g, stage, cfg.hx, cfg.hy, cfg.hz, d, padded,
                                                     id == AEO_FIELD_THETA ? th_off : 0.0);
        CKL();
        if (padded && loc >= 0) {
            if (loc == LOC_FZ && g.bc_z == 1) {
                wall_face_zero_kernel<R><<<dim3((g.nx + 127) / 128, g.ny), 128, 0, st>>>(g, d);
                CKL();
            }
            R* f[1] = {d};
            int l[1] = {loc};
            if (aeo_status e = halo(f, l, 1)) return e;
        }
        CK(cudaStreamSynchronize(st));
        return AEO_OK;
    }

    template <typename S>
    aeo_status get_field_t(int id, S* host) {
        int padded, loc;
        R* d = field_ptr(id, &padded, &loc);
        if (!d) { fail("get_field: unknown or unavailable field"); return AEO_ERR_ARGUMENT; }
        if (id == AEO_FIELD_NUT) {
            // the step keeps nut in shared memory: evaluate it for the current state
            if (dyn())
                if (aeo_status e = enqueue_dynamic(P[cur])) return e;
            if (uni) smagorinsky_kernel<R, true><<<grd3(), blk3(), 0, st>>>(g, P[cur][0], P[cur][1], P[cur][2], P[cur][3], nut, R(cfg.c_s), R(cfg.pr_t), d_cs2, dyn_d2, d_cs2f);
            else smagorinsky_kernel<R, false><<<grd3(), blk3(), 0, st>>>(g, P[cur][0], P[cur][1], P[cur][2], P[cur][3], nut, R(cfg.c_s), R(cfg.pr_t), d_cs2, dyn_d2, d_cs2f);
            CKL();
        }
        S* stage = reinterpret_cast<S*>(d_stage);
        pack_host_kernel<R, S><<<(unsigned)((host_n + 255) / 256), 256, 0, st>>>(g, stage, cfg.hx, cfg.hy, cfg.hz, d,
                                                                                 padded, loc,
                                                                                 id == AEO_FIELD_THETA ? th_off : 0.0);
        CKL();
        CK(cudaMemcpyAsync(host, stage, host_n * sizeof(S), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        return AEO_OK;
    }

    aeo_status pressure_solve(const double* src, double* out) override {
        CK(cudaMemcpyAsync(d_stage, src, g.nin * sizeof(double), cudaMemcpyHostToDevice, st));
        convert_kernel<R><<<(unsigned)((g.nin + 255) / 256), 256, 0, st>>>(g.nin, d_stage, Q[0]);
        CKL();
        if (aeo_status e = solve(Q[0])) return e;
        convert_back_kernel<R><<<(unsigned)((g.nin + 255) / 256), 256, 0, st>>>(g.nin, phi, d_stage);
        CKL();
        CK(cudaMemcpyAsync(out, d_stage, g.nin * sizeof(double), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        return AEO_OK;
    }

    // advect_positive! on caller arrays in the reference storage layout: device
    // arrays of the working precision (host = false, enqueued on the stream),
    // or host FP64 arrays staged through the device (host = true, synchronous)
    R *pos_fx = nullptr, *pos_fy = nullptr, *pos_fz = nullptr, *pos_r = nullptr, *pos_st = nullptr;
    aeo_status advect_positive(const void* u, const void* v, const void* w, const void* phi, void* tend, double dt,
                               int scheme, int accumulate, bool host) override {
        if (scheme != AEO_ADV_WENO_JS5 && scheme != AEO_ADV_WENO_Z5) {
            fail("advect_positive: scheme must be WENO-JS5 or WENO-Z5");
            return AEO_ERR_ARGUMENT;
        }
        if (!uni) { fail("advect_positive: a uniform grid is required (the WENO stencils assume it)"); return AEO_ERR_ARGUMENT; }
        if (cfg.hx < 3 || cfg.hy < 3 || cfg.hz < 3) { fail("advect_positive: halos >= 3 required"); return AEO_ERR_ARGUMENT; }
        if (!(dt >= 0)) { fail("advect_positive: dt >= 0 required"); return AEO_ERR_ARGUMENT; }
        if (!pos_fx) {
            if (aeo_status e = alloc(&pos_fx, (size_t)(g.nx + 1) * g.ny * g.nz)) return e;
            if (aeo_status e = alloc(&pos_fy, (size_t)g.nx * (g.ny + 1) * g.nz)) return e;
            if (aeo_status e = alloc(&pos_fz, (size_t)g.nx * g.ny * (g.nz + 1))) return e;
            if (aeo_status e = alloc(&pos_r, (size_t)g.nin)) return e;
        }
        const R* a[4] = {static_cast<const R*>(u), static_cast<const R*>(v), static_cast<const R*>(w),
                         static_cast<const R*>(phi)};
        R* t = static_cast<R*>(tend);
        const unsigned hb = (unsigned)((host_n + 255) / 256);
        if (host) {
            if (!pos_st)
                if (aeo_status e = alloc(&pos_st, 5 * (size_t)host_n)) return e;
            const double* hs[5] = {static_cast<const double*>(u), static_cast<const double*>(v),
                                   static_cast<const double*>(w), static_cast<const double*>(phi),
                                   static_cast<const double*>(tend)};
            for (int f = 0; f < 5; ++f) {
                if (f == 4 && !accumulate) break;
                CK(cudaMemcpyAsync(d_stage, hs[f], host_n * sizeof(double), cudaMemcpyHostToDevice, st));
                convert_kernel<R><<<hb, 256, 0, st>>>(host_n, d_stage, pos_st + f * host_n);
                CKL();
            }
            for (int f = 0; f < 4; ++f) a[f] = pos_st + f * host_n;
            t = pos_st + 4 * host_n;
        }
        set_scalar_kernel<<<1, 1, 0, st>>>(&d_sc->pos_dt, dt);
        CKL();
        PosGeo pg{};
        pg.nx = g.nx; pg.ny = g.ny; pg.nz = g.nz;
        pg.hx = cfg.hx; pg.hy = cfg.hy; pg.hz = cfg.hz;
        pg.sx = 1;
        pg.sy = g.nx + 2LL * cfg.hx;
        pg.sz = pg.sy * (g.ny + 2LL * cfg.hy);
        pg.idx = g.idx; pg.idy = g.idy; pg.idz = g.idz;
        const dim3 gf((unsigned)((g.nx + 1 + 127) / 128), (unsigned)(g.ny + 1), (unsigned)(g.nz + 1));
        if (scheme == AEO_ADV_WENO_Z5)
            pos_flux_kernel<R, AEO_ADV_WENO_Z5><<<gf, 128, 0, st>>>(pg, a[0], a[1], a[2], a[3], pos_fx, pos_fy, pos_fz);
        else
            pos_flux_kernel<R, AEO_ADV_WENO_JS5><<<gf, 128, 0, st>>>(pg, a[0], a[1], a[2], a[3], pos_fx, pos_fy, pos_fz);
        CKL();
        const dim3 gc((unsigned)((g.nx + 127) / 128), (unsigned)g.ny, (unsigned)g.nz);
        pos_ratio_kernel<R><<<gc, 128, 0, st>>>(pg, a[0], a[1], a[2], a[3], pos_fx, pos_fy, pos_fz, &d_sc->pos_dt, pos_r);
        CKL();
        pos_apply_kernel<R><<<gc, 128, 0, st>>>(pg, a[0], a[1], a[2], a[3], pos_fx, pos_fy, pos_fz, pos_r, t, accumulate);
        CKL();
        if (host) {
            convert_back_kernel<R><<<hb, 256, 0, st>>>(host_n, t, d_stage);
            CKL();
            CK(cudaMemcpyAsync(tend, d_stage, host_n * sizeof(double), cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
        }
        return AEO_OK;
    }

    // One Chorin projection of the state with dt = 1 (the config driver's
    // _project!(sim, 1.0), src/config/simulation_driver.jl:1316).
    aeo_status project() override {
        dim3 gb((g.nx + 127) / 128, g.ny, g.nz);
        for (int f = 0; f < 3; ++f) {
            padded_to_interior_kernel<R><<<gb, 128, 0, st>>>(g, P[cur][f], Q[f]);
            CKL();
        }
        if (aeo_status e = solve(nullptr)) return e;
        if (aeo_status e = correct(P[cur], 0, R(0), R(0), &d_sc->one, cur)) return e;
        R* f[3] = {P[cur][0], P[cur][1], P[cur][2]};
        int l[3] = {LOC_FX, LOC_FY, LOC_FZ};
        if (aeo_status e = halo(f, l, 3)) return e;
        CK(cudaStreamSynchronize(st));
        return AEO_OK;
    }

    // isotropic_turbulence_field! on the device, then the optional projection
    // and rescaling to a target per-component rms.
    aeo_status init_isotropic(double u_rms, double k_peak, uint64_t seed, double kmax, int proj,
                              double target_rms) override {
        if (cfg.solver != AEO_SOLVER_FFT || !uni) {
            fail("init_isotropic: a triply periodic uniform grid is required (src/operators/spectra.jl:316)");
            return AEO_ERR_ARGUMENT;
        }
        const int Mh = g.nx / 2 + 1, M = g.nx / 2;
        const long long ns = (long long)Mh * g.ny * g.nz;
        dim3 gy((Mh + tpx_y - 1) / tpx_y, g.nz);
        size_t smy = (size_t)tpx_y * g.ny * sizeof(cplx<R>);
        dim3 gz((Mh + tpx_z - 1) / tpx_z, g.ny);
        size_t smz = (size_t)tpx_z * g.nz * sizeof(cplx<R>);
        size_t smx = (size_t)rows_x * xrow(M) * sizeof(cplx<R>);
        unsigned gx = (unsigned)((g.ny * (long long)g.nz + rows_x - 1) / rows_x);
        dim3 gb((g.nx + 127) / 128, g.ny, g.nz);
        for (int comp = 0; comp < 3; ++comp) {
            IsoParams p{};
            p.u_rms = u_rms; p.k_peak = k_peak; p.kmax = kmax > 0 ? kmax : 1.0 / 0.0;
            p.lx = cfg.lx; p.ly = cfg.ly; p.lz = cfg.lz;
            p.x1 = cfg.x0 + (comp == 0 ? 0.0 : 0.5 * g.dx);
            p.y1 = cfg.y0 + (comp == 1 ? 0.0 : 0.5 * g.dy);
            p.z1 = cfg.z0 + (comp == 2 ? 0.0 : 0.5 * g.dz);
            p.seed = seed;
            p.comp = comp;
            iso_modes_kernel<R><<<(unsigned)((ns + 255) / 256), 256, 0, st>>>(g, S, p);
            CKL();
            fftz_inv_kernel<R><<<gz, FFT_THREADS(R), smz, st>>>(g, S, tw, NT, tpx_z);
            CKL();
            ffty_kernel<R, 1><<<gy, FFT_THREADS(R), smy, st>>>(g, S, tw, NT, tpx_y);
            CKL();
            ifftx_kernel<R><<<gx, FFT_THREADS(R), smx, st>>>(g, S, phi, tw, NT, rows_x, R(1));
            CKL();
            interior_to_padded_kernel<R><<<gb, 128, 0, st>>>(g, phi, P[cur][comp], R(1));
            CKL();
        }
        R* f[3] = {P[cur][0], P[cur][1], P[cur][2]};
        int l[3] = {LOC_FX, LOC_FY, LOC_FZ};
        if (aeo_status e = halo(f, l, 3)) return e;
        if (proj)
            if (aeo_status e = project()) return e;
        if (target_rms > 0) {
            sumsq_levels_kernel<R><<<g.nz, 256, 0, st>>>(g, P[cur][0], P[cur][1], P[cur][2], d_part);
            CKL();
            std::vector<double> h(g.nz);
            CK(cudaMemcpyAsync(h.data(), d_part, g.nz * sizeof(double), cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            double sum = 0.0;
            for (int k = 0; k < g.nz; ++k) sum += h[k];
            double rms = std::sqrt(sum / (3.0 * (double)g.nin));
            if (!(rms > 0)) { fail("init_isotropic: the generated field is zero"); return AEO_ERR_NUMERICAL; }
            for (int c = 0; c < 3; ++c) {
                scale_padded_kernel<R><<<gb, 128, 0, st>>>(g, P[cur][c], target_rms / rms);
                CKL();
            }
            if (aeo_status e = halo(f, l, 3)) return e;
        }
        CK(cudaStreamSynchronize(st));
        return AEO_OK;
    }

    aeo_status kinetic_energy(double* out) override {
        if (uni) ke_levels_kernel<R, true><<<g.nz, 256, 0, st>>>(g, P[cur][0], P[cur][1], P[cur][2], d_part);
        else ke_levels_kernel<R, false><<<g.nz, 256, 0, st>>>(g, P[cur][0], P[cur][1], P[cur][2], d_part);
        CKL();
        std::vector<double> h(g.nz);
        CK(cudaMemcpyAsync(h.data(), d_part, g.nz * sizeof(double), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        double t = 0.0;
        for (int k = 0; k < g.nz; ++k) t += h[k];
        *out = uni ? 0.5 * t * (g.dx * g.dy * g.dz) : 0.5 * t * g.dx * g.dy;
        return AEO_OK;
    }

    aeo_status max_divergence(double* out) override {
        R** s = P[cur];
        if (pcg) {
            if (anel && uni) cc_maxdiv_levels_kernel<R, true, true><<<g.nz, 256, 0, st>>>(g, s[0], s[1], s[2], apx, apy, apz, d_part);
            else if (anel) cc_maxdiv_levels_kernel<R, true, false><<<g.nz, 256, 0, st>>>(g, s[0], s[1], s[2], apx, apy, apz, d_part);
            else if (!uni) cc_maxdiv_levels_kernel<R, false, false><<<g.nz, 256, 0, st>>>(g, s[0], s[1], s[2], apx, apy, apz, d_part);
            else cc_maxdiv_levels_kernel<R><<<g.nz, 256, 0, st>>>(g, s[0], s[1], s[2], apx, apy, apz, d_part);
            CKL();
            std::vector<double> h((size_t)g.nz);
            CK(cudaMemcpyAsync(h.data(), d_part, h.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            double m = 0.0;
            for (double v : h) m = std::max(m, v);
            *out = m;
            return AEO_OK;
        }
        if (anel) {
            if (uni) maxdiv_levels_kernel<R, true, true><<<g.nz, 256, 0, st>>>(g, s[0], s[1], s[2], d_part);
            else maxdiv_levels_kernel<R, true, false><<<g.nz, 256, 0, st>>>(g, s[0], s[1], s[2], d_part);
        } else {
            if (uni) maxdiv_levels_kernel<R, false, true><<<g.nz, 256, 0, st>>>(g, s[0], s[1], s[2], d_part);
            else maxdiv_levels_kernel<R, false, false><<<g.nz, 256, 0, st>>>(g, s[0], s[1], s[2], d_part);
        }
        CKL();
        std::vector<double> h(g.nz);
        CK(cudaMemcpyAsync(h.data(), d_part, g.nz * sizeof(double), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        double m = 0.0;
        for (int k = 0; k < g.nz; ++k) m = std::max(m, h[k]);
        *out = m;
        return AEO_OK;
    }

    aeo_status fill_uniform(int id, uint64_t seed, uint32_t stream, double amp, int mode) override {
        int padded, loc;
        R* d = field_ptr(id, &padded, &loc);
        if (!d || loc < 0) { fail("fill_uniform: field must be u, v, w or theta"); return AEO_ERR_ARGUMENT; }
        philox_fill_kernel<R><<<(unsigned)((g.nin + 255) / 256), 256, 0, st>>>(g, d, padded, seed, stream, amp, mode,
                                                                               id == AEO_FIELD_THETA ? th_off : 0.0);
        CKL();
        if (loc == LOC_FZ && g.bc_z == 1) {
            wall_face_zero_kernel<R><<<dim3((g.nx + 127) / 128, g.ny), 128, 0, st>>>(g, d);
            CKL();
        }
        R* f[1] = {d};
        int l[1] = {loc};
        if (aeo_status e = halo(f, l, 1)) return e;
        CK(cudaStreamSynchronize(st));
        return AEO_OK;
    }
};

// ====================================================================================
// C-ABI
// ====================================================================================

static aeo_status validate(const aeo_config* c, const double* zf, const double* wc, const double* wf, std::string* m) {
    if (!c) { *m = "config is NULL"; return AEO_ERR_ARGUMENT; }
    if (c->nx < 4 || c->ny < 4 || c->nz < 2) { *m = "grid too small (nx, ny >= 4, nz >= 2)"; return AEO_ERR_ARGUMENT; }
    if (!is_pow2(c->nx) || !is_pow2(c->ny)) { *m = "nx and ny must be powers of two"; return AEO_ERR_ARGUMENT; }
    if (c->nx / 2 > 2048 || c->ny > 2048) { *m = "nx/2 and ny must not exceed 2048"; return AEO_ERR_ARGUMENT; }
    if (c->bc_x != AEO_BC_PERIODIC || c->bc_y != AEO_BC_PERIODIC) { *m = "x and y must be periodic"; return AEO_ERR_ARGUMENT; }
    if (c->bc_z != AEO_BC_PERIODIC && c->bc_z != AEO_BC_WALL) { *m = "bc_z must be periodic or wall"; return AEO_ERR_ARGUMENT; }
    if (c->hx < 0 || c->hy < 0 || c->hz < 0 || c->hx > 8 || c->hy > 8 || c->hz > 8) { *m = "host halo widths must be in 0..8"; return AEO_ERR_ARGUMENT; }
    if (c->solver == AEO_SOLVER_FFT) {
        if (c->bc_z != AEO_BC_PERIODIC) { *m = "the FFT solver needs a periodic z"; return AEO_ERR_ARGUMENT; }
        if (!is_pow2(c->nz) || c->nz > 2048) { *m = "the FFT solver needs nz a power of two <= 2048"; return AEO_ERR_ARGUMENT; }
    } else if (c->solver == AEO_SOLVER_COLUMN) {
        if (c->bc_z != AEO_BC_WALL) { *m = "the column solver needs walls in z"; return AEO_ERR_ARGUMENT; }
        if (c->nz > AEO_COLUMN_NZ_MAX) { *m = "the column solver needs nz <= " + std::to_string(AEO_COLUMN_NZ_MAX); return AEO_ERR_ARGUMENT; }
    } else if (c->solver == AEO_SOLVER_PCG) {
        // any core and column: the density weights and the stretched metric
        // enter the multigrid operator in its symmetric form (aeo_cutcell.cuh)
    } else { *m = "unknown solver"; return AEO_ERR_ARGUMENT; }
    if (c->advection < 0 || c->advection > 2) { *m = "unknown advection scheme"; return AEO_ERR_ARGUMENT; }
    if (c->advection != AEO_ADV_CENTRED && (c->stretched || c->core == AEO_CORE_ANELASTIC)) {
        *m = "WENO advection is defined on a uniform Boussinesq grid (src/AdvectionSchemes.jl:731)";
        return AEO_ERR_ARGUMENT;
    }
    if (c->core == AEO_CORE_ANELASTIC && (!wc || !wf || c->bc_z != AEO_BC_WALL)) {
        *m = "the anelastic core needs wc, wf and walls in z";
        return AEO_ERR_ARGUMENT;
    }
    if (c->core != AEO_CORE_BOUSSINESQ && c->core != AEO_CORE_ANELASTIC) { *m = "unknown core"; return AEO_ERR_ARGUMENT; }
    if (c->stretched && (!zf || c->bc_z != AEO_BC_WALL)) { *m = "a stretched grid needs zf and walls in z"; return AEO_ERR_ARGUMENT; }
    if (c->precision != AEO_PREC_FP64 && c->precision != AEO_PREC_FP32_MIXED) { *m = "unknown precision"; return AEO_ERR_ARGUMENT; }
    if (c->c_s != 0.0 && !(c->pr_t > 0.0)) { *m = "pr_t must be positive with SGS"; return AEO_ERR_ARGUMENT; }
    if (c->sgs_model != AEO_SGS_SMAGORINSKY && c->sgs_model != AEO_SGS_VREMAN && c->sgs_model != AEO_SGS_SIGMA &&
        c->sgs_model != AEO_SGS_AMD && c->sgs_model != AEO_SGS_DYNAMIC && c->sgs_model != AEO_SGS_DYNAMIC_LOCAL &&
        c->sgs_model != AEO_SGS_LAGRANGIAN && c->sgs_model != AEO_SGS_TKE) {
        *m = "unknown SGS closure";
        return AEO_ERR_ARGUMENT;
    }
    if (c->sgs_model != AEO_SGS_SMAGORINSKY && c->stretched) {
        *m = "the Vreman, sigma, AMD and dynamic closures take a uniform grid (src/operators/sgs_amd_vreman.jl:102-107, "
             ":280-284, src/operators/sigma_closure.jl:208-212, src/Operators.jl:555)";
        return AEO_ERR_ARGUMENT;
    }
    if (c->sgs_model == AEO_SGS_TKE && c->c_s != 0.0 &&
        (c->core != AEO_CORE_BOUSSINESQ || c->hx < 3 || c->hy < 3 || c->hz < 3)) {
        *m = "the TKE closure runs on the Boussinesq core (theta0 its buoyancy reference) with host halos >= 3 "
             "(the WENO-Z5 transport of e, src/PrognosticSGS.jl:354-356)";
        return AEO_ERR_ARGUMENT;
    }
    if ((c->sgs_model == AEO_SGS_DYNAMIC || c->sgs_model == AEO_SGS_DYNAMIC_LOCAL || c->sgs_model == AEO_SGS_LAGRANGIAN) &&
        c->c_s != 0.0 && (c->hx < 2 || c->hy < 2 || c->hz < 2)) {
        *m = "the dynamic Smagorinsky closures need host halos of at least 2 (src/Operators.jl:556-557, "
             "src/operators/lagrangian_sgs.jl:170-171)";
        return AEO_ERR_ARGUMENT;
    }
    return AEO_OK;
}

extern "C" {

aeo_status aeo_create(const aeo_config* cfg, const double* zf, const double* wc, const double* wf, const double* thf,
                      aeo_sim** out) {
    if (!out) { g_create_error = "out is NULL"; return AEO_ERR_ARGUMENT; }
    *out = nullptr;
    std::string m;
    if (aeo_status s = validate(cfg, zf, wc, wf, &m)) { g_create_error = m; return s; }
    cudaError_t e = cudaSetDevice(cfg->device);
    if (e != cudaSuccess) { g_create_error = std::string("cudaSetDevice: ") + cudaGetErrorString(e); return AEO_ERR_CUDA; }
    CoreBase* c = cfg->precision == AEO_PREC_FP64 ? (CoreBase*)new (std::nothrow) Core<double>()
                                                  : (CoreBase*)new (std::nothrow) Core<float>();
    if (!c) { g_create_error = "out of host memory"; return AEO_ERR_CUDA; }
    c->cfg = *cfg;
    aeo_status s = c->init(zf, wc, wf, thf);
    if (s) { g_create_error = c->err; delete c; return s; }
    aeo_sim* h = new (std::nothrow) aeo_sim;
    if (!h) { delete c; g_create_error = "out of host memory"; return AEO_ERR_CUDA; }
    h->core = c;
    *out = h;
    return AEO_OK;
}

aeo_status aeo_destroy(aeo_sim* h) {
    if (!h) return AEO_OK;
    cudaSetDevice(h->core->cfg.device);
    delete h->core;
    delete h;
    return AEO_OK;
}

#define ENTER(h)                                                       \
    if (!h) return AEO_ERR_ARGUMENT;                                   \
    if (cudaSetDevice(h->core->cfg.device) != cudaSuccess) {           \
        h->core->fail("cudaSetDevice failed");                         \
        return AEO_ERR_CUDA;                                           \
    }

aeo_status aeo_set_field(aeo_sim* h, int32_t field, const double* host) {
    ENTER(h);
    if (!host) { h->core->fail("host pointer is NULL"); return AEO_ERR_ARGUMENT; }
    return h->core->set_field(field, host);
}

aeo_status aeo_get_field(aeo_sim* h, int32_t field, double* host) {
    ENTER(h);
    if (!host) { h->core->fail("host pointer is NULL"); return AEO_ERR_ARGUMENT; }
    return h->core->get_field(field, host);
}

aeo_status aeo_set_field_f32(aeo_sim* h, int32_t field, const float* host) {
    ENTER(h);
    if (!host) { h->core->fail("host pointer is NULL"); return AEO_ERR_ARGUMENT; }
    return h->core->set_field_f32(field, host);
}

aeo_status aeo_get_field_f32(aeo_sim* h, int32_t field, float* host) {
    ENTER(h);
    if (!host) { h->core->fail("host pointer is NULL"); return AEO_ERR_ARGUMENT; }
    return h->core->get_field_f32(field, host);
}

aeo_status aeo_step_rk3(aeo_sim* h, double dt, int32_t nsteps) {
    ENTER(h);
    if (!(dt > 0) || nsteps < 0) { h->core->fail("dt must be positive and nsteps >= 0"); return AEO_ERR_ARGUMENT; }
    return h->core->step_rk3(dt, nsteps, true);
}

aeo_status aeo_step_rk3_async(aeo_sim* h, double dt, int32_t nsteps) {
    ENTER(h);
    if (!(dt > 0) || nsteps < 0) { h->core->fail("dt must be positive and nsteps >= 0"); return AEO_ERR_ARGUMENT; }
    return h->core->step_rk3(dt, nsteps, false);
}

aeo_status aeo_synchronize(aeo_sim* h) {
    ENTER(h);
    cudaError_t e = cudaStreamSynchronize(h->core->st);
    if (e != cudaSuccess) { h->core->fail(cudaGetErrorString(e)); return AEO_ERR_CUDA; }
    return AEO_OK;
}

aeo_status aeo_step_euler(aeo_sim* h, double dt, int32_t nsteps) {
    ENTER(h);
    if (!(dt > 0) || nsteps < 0) { h->core->fail("dt must be positive and nsteps >= 0"); return AEO_ERR_ARGUMENT; }
    return h->core->step_euler(dt, nsteps);
}

aeo_status aeo_step_adaptive(aeo_sim* h, const aeo_cfl* c, int32_t nsteps, double* dt_prev,
                             aeo_adaptive_stats* stats) {
    ENTER(h);
    if (!c || nsteps < 0 || !(c->c_advective > 0) || !(c->c_diffusive > 0) || !(c->c_buoyancy > 0) ||
        !(c->c_coriolis > 0) || !(c->dt_min > 0) || !(c->dt_min <= c->dt_max) || !(c->growth_max >= 1) ||
        c->max_retries < 0) {
        h->core->fail("step_adaptive: invalid CFL constraints (CFLConstraints, src/TimeIntegration.jl:137-153)");
        return AEO_ERR_ARGUMENT;
    }
    return h->core->step_adaptive(c, nsteps, dt_prev, stats);
}

aeo_status aeo_cfl_diagnostics(aeo_sim* h, const aeo_cfl* c, double dt_prev, aeo_adaptive_stats* out) {
    ENTER(h);
    if (!c || !out || !(c->c_advective > 0) || !(c->c_diffusive > 0) || !(c->dt_min > 0) || !(c->dt_min <= c->dt_max) ||
        !(c->growth_max >= 1)) {
        h->core->fail("cfl_diagnostics: invalid CFL constraints");
        return AEO_ERR_ARGUMENT;
    }
    return h->core->cfl(c, dt_prev, out);
}

aeo_status aeo_init_isotropic(aeo_sim* h, double u_rms, double k_peak, uint64_t seed, double kmax, int32_t project,
                              double target_rms) {
    ENTER(h);
    if (!(u_rms > 0) || !(k_peak > 0)) { h->core->fail("init_isotropic: u_rms and k_peak must be positive"); return AEO_ERR_ARGUMENT; }
    return h->core->init_isotropic(u_rms, k_peak, seed, kmax, project, target_rms);
}

aeo_status aeo_project(aeo_sim* h) {
    ENTER(h);
    return h->core->project();
}

aeo_status aeo_pressure_solve(aeo_sim* h, const double* src, double* phi) {
    ENTER(h);
    if (!src || !phi) { h->core->fail("NULL array"); return AEO_ERR_ARGUMENT; }
    return h->core->pressure_solve(src, phi);
}

aeo_status aeo_advect_positive(aeo_sim* h, const double* u, const double* v, const double* w, const double* phi,
                               double* tend, double dt, int32_t scheme, int32_t accumulate) {
    ENTER(h);
    if (!u || !v || !w || !phi || !tend) { h->core->fail("NULL array"); return AEO_ERR_ARGUMENT; }
    return h->core->advect_positive(u, v, w, phi, tend, dt, scheme, accumulate, true);
}

aeo_status aeo_advect_positive_device(aeo_sim* h, const void* u, const void* v, const void* w, const void* phi,
                                      void* tend, double dt, int32_t scheme, int32_t accumulate) {
    ENTER(h);
    if (!u || !v || !w || !phi || !tend) { h->core->fail("NULL array"); return AEO_ERR_ARGUMENT; }
    return h->core->advect_positive(u, v, w, phi, tend, dt, scheme, accumulate, false);
}

aeo_status aeo_set_ibm(aeo_sim* h, const uint8_t* mask, double tau) {
    ENTER(h);
    return h->core->set_ibm(mask, tau);
}

aeo_status aeo_set_sgs_buoyancy(aeo_sim* h, const double* bg) {
    ENTER(h);
    return h->core->set_sgs_buoyancy(bg);
}

aeo_status aeo_set_lagrangian(aeo_sim* h, double c0, double theta, double memory_time) {
    ENTER(h);
    return h->core->set_lagrangian(c0, theta, memory_time);
}

aeo_status aeo_set_tke(aeo_sim* h, double c_eps0, double c_eps1, double c_l, int32_t exact) {
    ENTER(h);
    return h->core->set_tke(c_eps0, c_eps1, c_l, exact);
}

aeo_status aeo_get_sgs_state(aeo_sim* h, double* out) {
    ENTER(h);
    return h->core->get_sgs_state(out);
}

aeo_status aeo_set_sgs_state(aeo_sim* h, const double* in) {
    ENTER(h);
    return h->core->set_sgs_state(in);
}

aeo_status aeo_set_pcg(aeo_sim* h, const double* ax, const double* ay, const double* az, double tol, int32_t maxit) {
    ENTER(h);
    return h->core->set_pcg(ax, ay, az, tol, maxit);
}

aeo_status aeo_pcg_stats(aeo_sim* h, int32_t* iterations, int32_t* status, double* residual, double* bnorm) {
    ENTER(h);
    aeo_mg_stats o{};
    if (aeo_status e = h->core->pcg_stats(&o)) return e;
    if (iterations) *iterations = o.iterations;
    if (status) *status = o.status;
    if (residual) *residual = o.residual;
    if (bnorm) *bnorm = o.bnorm;
    return AEO_OK;
}

aeo_status aeo_pcg_set_learned(aeo_sim* h, struct aeo_unet* net, double stagnation) {
    ENTER(h);
    return h->core->pcg_set_learned(net, stagnation);
}

aeo_status aeo_set_open(aeo_sim* h, int32_t open_x, int32_t open_y, const double* x_planes, const double* y_planes,
                        const int32_t* modes) {
    ENTER(h);
    return h->core->set_open(open_x, open_y, x_planes, y_planes, modes);
}

aeo_status aeo_set_open_outflow(aeo_sim* h, const int32_t* radiate, int32_t correction, const double* x_data,
                                const double* y_data, const double* x_weights, const double* y_weights) {
    ENTER(h);
    return h->core->set_open_outflow(radiate, correction, x_data, y_data, x_weights, y_weights);
}

aeo_status aeo_get_open_planes(aeo_sim* h, double* x_planes, double* y_planes) {
    ENTER(h);
    return h->core->get_open_planes(x_planes, y_planes);
}

aeo_status aeo_set_open_planes(aeo_sim* h, const double* x_planes, const double* y_planes) {
    ENTER(h);
    return h->core->set_open_planes(x_planes, y_planes);
}

aeo_status aeo_get_open_history(aeo_sim* h, double* x_hist, double* y_hist, double* scalars) {
    ENTER(h);
    return h->core->open_state(x_hist, y_hist, scalars, false);
}

aeo_status aeo_set_open_history(aeo_sim* h, const double* x_hist, const double* y_hist, const double* scalars) {
    ENTER(h);
    return h->core->open_state(const_cast<double*>(x_hist), const_cast<double*>(y_hist), const_cast<double*>(scalars),
                               true);
}

aeo_status aeo_open_ledger(aeo_sim* h, double* out) {
    ENTER(h);
    if (!out) return AEO_ERR_ARGUMENT;
    return h->core->open_ledger(out);
}

aeo_status aeo_pcg_harvest(aeo_sim* h, int32_t cap, double* b, double* x, double* r_hist, double* x_hist,
                           int32_t* count) {
    ENTER(h);
    if (!b || !x || !r_hist || !x_hist || !count || cap < 1) {
        h->core->fail("pcg_harvest: NULL array or cap < 1");
        return AEO_ERR_ARGUMENT;
    }
    return h->core->pcg_harvest(cap, b, x, r_hist, x_hist, count);
}

aeo_status aeo_kinetic_energy(aeo_sim* h, double* out) {
    ENTER(h);
    if (!out) return AEO_ERR_ARGUMENT;
    return h->core->kinetic_energy(out);
}

aeo_status aeo_max_divergence(aeo_sim* h, double* out) {
    ENTER(h);
    if (!out) return AEO_ERR_ARGUMENT;
    return h->core->max_divergence(out);
}

aeo_status aeo_profile_step(aeo_sim* h, double dt, double* ms_per_class, int32_t nclass) {
    ENTER(h);
    if (!(dt > 0) || !ms_per_class || nclass < 0) { h->core->fail("bad profile arguments"); return AEO_ERR_ARGUMENT; }
    return h->core->profile_step(dt, ms_per_class, nclass);
}

aeo_status aeo_launches_per_step(aeo_sim* h, int32_t* out) {
    if (!h || !out) return AEO_ERR_ARGUMENT;
    *out = h->core->step_launches();
    return AEO_OK;
}

void* aeo_stream(aeo_sim* h) { return h ? (void*)h->core->st : nullptr; }

aeo_status aeo_fill_uniform(aeo_sim* h, int32_t field, uint64_t seed, uint32_t stream, double amp, int32_t mode) {
    ENTER(h);
    return h->core->fill_uniform(field, seed, stream, amp, mode);
}

const char* aeo_last_error(const aeo_sim* h) { return h ? h->core->err.c_str() : g_create_error.c_str(); }

const char* aeo_version(void) { return "aeolus_b200 0.1 (sm_100a)"; }

}  // extern "C"
