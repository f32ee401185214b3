/*
 * aeolus_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU FP64 restatement of the Aeolus.jl dynamical-core step (the checker the
 * CUDA library is compared against).  Nothing in the product path links,
 * loads or calls this code; only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / --impl reference legs of bench.py do.
 *
 * Arrays crossing this interface use the reference storage layout: a field
 * on a grid of Nx x Ny x Nz interior cells with halos (Hx, Hy, Hz) is a
 * column-major (x fastest) array of (Nx+2Hx)(Ny+2Hy)(Nz+2Hz) doubles, the
 * interior at 0-based indices [H, H+N).  FaceX index i is the west face of
 * cell i, FaceY the south face, FaceZ the bottom face (src/Grids.jl:52-80).
 */
#ifndef AEOLUS_ORACLE_H
#define AEOLUS_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { OC_BC_PERIODIC = 0, OC_BC_WALL = 1 };
enum { OC_CORE_BOUSSINESQ = 0, OC_CORE_ANELASTIC = 1 };
enum { OC_ADV_CENTRED = 0, OC_ADV_WENO_JS5 = 1, OC_ADV_WENO_Z5 = 2 };
enum { OC_SOLVER_FFT = 0, OC_SOLVER_COLUMN = 1, OC_SOLVER_PCG = 2 };
enum { OC_U = 0, OC_V = 1, OC_W = 2, OC_THETA = 3, OC_P = 4, OC_NUT = 5, OC_PHI = 6, OC_KT = 7 };
enum { OC_SGS_SMAGORINSKY = 0, OC_SGS_VREMAN = 1, OC_SGS_SIGMA = 2, OC_SGS_AMD = 3, OC_SGS_DYNAMIC = 4,
       OC_SGS_DYNAMIC_LOCAL = 5,     /* 5: averaging = :local, src/Operators.jl:873-880 */
       OC_SGS_LAGRANGIAN = 6,        /* 6: LagrangianDynamicSmagorinsky, src/operators/lagrangian_sgs.jl */
       OC_SGS_TKE = 7 };             /* 7: TKEClosure (Deardorff 1980), src/PrognosticSGS.jl; c_s is c_k */

typedef struct {
    int32_t nx, ny, nz, hx, hy, hz;
    double lx, ly, lz, x0, y0, z0;
    int32_t stretched;        /* 0: uniform z; 1: zf[] gives the Nz+1 interior faces */
    int32_t bc_x, bc_y, bc_z; /* x, y: periodic only; z: periodic or wall */
    int32_t core, advection, solver;
    double nu, theta0, g, f_coriolis, c_s, pr_t;
    double flux_bot, flux_top, sponge_alpha, sponge_zstart;
    int32_t sgs_model;        /* OC_SGS_* when c_s > 0 (Vreman, sigma, AMD: uniform grids;
                                 AMD: c_s is its constant C, Boussinesq core;
                                 dynamic Smagorinsky: c_s is the clip cs_max) */
} oc_params;

typedef struct oc_sim oc_sim;

/* zf: Nz+1 interior face heights (stretched only, else NULL).
 * wc (Nz+2Hz), wf (Nz+2Hz+1), thf (Nz+2Hz+1): padded weights and the face
 * reference potential temperature of the anelastic core (NULL otherwise). */
oc_sim* oc_create(const oc_params* p, const double* zf, const double* wc,
                  const double* wf, const double* thf);
void oc_destroy(oc_sim* s);
int64_t oc_storage_size(const oc_sim* s);
int oc_set_field(oc_sim* s, int id, const double* src);
int oc_get_field(const oc_sim* s, int id, double* dst);
void oc_fill_state_halos(oc_sim* s);
int oc_step_rk3(oc_sim* s, double dt, int nsteps);
int oc_step_euler(oc_sim* s, double dt, int nsteps);
/* Chorin projection of the current velocity (dt = 1). */
int oc_project(oc_sim* s);

/* CFLConstraints (src/TimeIntegration.jl:127-153) */
typedef struct { double c_adv, c_diff, c_buoy, c_cor, dt_min, dt_max, growth; } oc_cfl;
double oc_adaptive_dt(oc_sim* s, const oc_cfl* c, double dt_prev, int* limiter);
int oc_step_adaptive(oc_sim* s, const oc_cfl* c, int nsteps, double* dt_prev, double* dts);
/* Tendencies of the current state (halos filled first) into tu..tθ (storage). */
int oc_tendencies(oc_sim* s, double* tu, double* tv, double* tw, double* tt);
/* Solve the projection's Poisson problem: src and phi are interior-sized
 * (Nx*Ny*Nz, x fastest). */
int oc_pressure_solve(oc_sim* s, const double* src, double* phi);
/* Apply the discrete operator the solver inverts (interior-sized in/out). */
int oc_apply_poisson_operator(oc_sim* s, const double* phi, double* out);
double oc_kinetic_energy(oc_sim* s);
/* max |divergence|; solver = OC_SOLVER_PCG: the aperture-weighted one */
double oc_max_divergence(oc_sim* s);
/* solver = OC_SOLVER_PCG (uniform Boussinesq grid): the face apertures in
 * [0, 1] in the interior face layout of mgpcg_oracle.h (all NULL: every face
 * open; the wall faces of a bounded z are blocked whatever is given) and the
 * multigrid-preconditioned CG's relative tolerance and iteration cap.  The
 * projection solves sum_faces a^2 (phi_nbr - phi) / h^2 = the
 * aperture-weighted divergence and corrects u = u* - a d(phi) on every face
 * (zero on a blocked face).  0 on success. */
int oc_set_apertures(oc_sim* s, const double* ax, const double* ay, const double* az, double tol, int maxit);
/* the AMD closure's buoyancy parameter g/theta_bar(z_k) of the Nz interior
 * levels (the sound-proof core; src/operators/sgs_amd_vreman.jl:331-345) */
int oc_set_sgs_buoyancy(oc_sim* s, const double* bg);
/* the Lagrangian closure's C0 (0.16), theta (1.5) and memory_time (<= 0:
 * MLC96's T), src/operators/lagrangian_sgs.jl:163-199 */
int oc_set_lagrangian(oc_sim* s, double c0, double theta, double memory_time);
/* sgs_state / restore_sgs_state! of the Lagrangian closure
 * (src/operators/lagrangian_sgs.jl:372-381): 5 Nx Ny Nz + 1 values, I_LM,
 * I_MM and the cell-centred u, v, w of the memory (x fastest), then the
 * initialised flag (0 / 1).  0 on success. */
int oc_get_sgs_state(const oc_sim* s, double* out);
/* the TKE closure's c_eps0 (0.19), c_eps1 (0.51), c_l (0.76) and dissipation
 * form (0 :semi_implicit, 1 :exact), src/PrognosticSGS.jl:326-375; its
 * sgs_state is e on the interior (Nx Ny Nz values, x fastest) */
int oc_set_tke(oc_sim* s, double c_eps0, double c_eps1, double c_l, int exact);
int oc_set_sgs_state(oc_sim* s, const double* in);
/* the implicit IBM correction after every predictor (implicit_ibm_correction!,
 * src/IBM.jl:295-300): mask storage-shaped, nonzero = solid (interior cells
 * count), NULL switches it off; tau >= 0 (0: the faces are zeroed); not with
 * OC_SOLVER_PCG.  0 on success. */
int oc_set_ibm(oc_sim* s, const unsigned char* mask, double tau);
/* iterations, status (mgpcg_oracle.h OCG_*), ||r|| and ||b|| of the last solve */
int oc_pcg_stats(const oc_sim* s, int* iterations, int* status, double* residual, double* bnorm);
/* open lateral faces: planes in the layout of aeo_set_open (FP64), modes[4] */
int oc_set_open(oc_sim* s, int open_x, int open_y, const double* xp, const double* yp, const int* modes);
/* radiating (:convective) outflow per side, the correction mode, the raw data planes */
int oc_set_open_outflow(oc_sim* s, const int* rad, int corr, const double* xd, const double* yd,
                        const double* xf, const double* yf);
/* Q, residual, delta of the last correction on the device-side update */
void oc_open_ledger(const oc_sim* s, double* out);
/* the current plane buffers (layout of oc_set_open) */
void oc_get_open_planes(const oc_sim* s, double* xp, double* yp);
/* a checkpoint's planes back (the halos refilled) */
int oc_set_open_planes(oc_sim* s, const double* xp, const double* yp);
/* the :orlanski history and (history set, last dt): read (set 0) or written */
int oc_open_history(oc_sim* s, double* xh, double* yh, double* sc, int set);
void oc_set_threads(int n);
/* advect_positive! (src/AdvectionSchemes.jl:1100-1160): add (accumulate) or
 * write -div(u phi) with the positivity limiter; storage arrays of the
 * domain's layout with filled halos (>= 3); scheme OC_ADV_WENO_JS5 or
 * OC_ADV_WENO_Z5; uniform grids.  0 on success. */
int oc_advect_positive(oc_sim* s, const double* u, const double* v, const double* w, const double* phi,
                       double* tend, double dt, int scheme, int accumulate);

/* Philox4x32-10 block function and the uniform fill of the synthetic inputs. */
void oc_philox4x32(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
void oc_uniform_fill(uint64_t seed, uint32_t stream, int64_t n, double amp, double* out);

#ifdef __cplusplus
}
#endif
#endif
