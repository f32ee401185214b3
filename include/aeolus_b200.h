/*
 * aeolus_b200.h -- the C-ABI of libaeolus_b200.so, the B200 (sm_100a)
 * dynamical-core step of the Aeolus.jl large-eddy-simulation model.
 *
 * One handle owns all device state of one domain (one simulation).  Host
 * arrays crossing this interface are in the reference's storage layout: a
 * Float64 field of Nx x Ny x Nz interior cells with halos (Hx, Hy, Hz) is a
 * column-major (x fastest) array of (Nx+2Hx)(Ny+2Hy)(Nz+2Hz) doubles, i.e.
 * the `Field.data` array of the reference (src/Fields.jl:21,
 * src/Grids.jl:98-130), so a Julia `ccall` passes it by pointer with no
 * reshuffle.  No host pointer is retained after a call returns.
 *
 * Every entry point returns an aeo_status; on failure aeo_last_error(h)
 * describes it.  A handle is not thread-safe; distinct handles are
 * independent.  Work is enqueued on the handle's own CUDA stream and every
 * call below returns after that stream has synchronised.
 *
 * Each entry point names the reference interface it replaces.
 */
#ifndef AEOLUS_B200_H
#define AEOLUS_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    AEO_OK = 0,
    AEO_ERR_ARGUMENT = 1,   /* maps to ArgumentError in the host shim */
    AEO_ERR_CUDA = 2,       /* CUDA runtime failure (message in aeo_last_error) */
    AEO_ERR_NUMERICAL = 3,  /* non-finite state or failed solve: NumericalFailure */
    AEO_ERR_STATE = 4       /* call out of order (e.g. no field set yet) */
} aeo_status;

enum { AEO_BC_PERIODIC = 0, AEO_BC_WALL = 1 };
enum { AEO_CORE_BOUSSINESQ = 0, AEO_CORE_ANELASTIC = 1 };
enum { AEO_ADV_CENTRED = 0, AEO_ADV_WENO_JS5 = 1, AEO_ADV_WENO_Z5 = 2 };
enum { AEO_SOLVER_FFT = 0, AEO_SOLVER_COLUMN = 1, AEO_SOLVER_PCG = 2 };
enum { AEO_PREC_FP64 = 0, AEO_PREC_FP32_MIXED = 1 };
enum { AEO_SGS_SMAGORINSKY = 0, AEO_SGS_VREMAN = 1, AEO_SGS_SIGMA = 2, AEO_SGS_AMD = 3, AEO_SGS_DYNAMIC = 4,
       AEO_SGS_DYNAMIC_LOCAL = 5, AEO_SGS_LAGRANGIAN = 6, AEO_SGS_TKE = 7 };
enum { AEO_FIELD_U = 0, AEO_FIELD_V = 1, AEO_FIELD_W = 2, AEO_FIELD_THETA = 3,
       AEO_FIELD_P = 4, AEO_FIELD_NUT = 5 };

/* Grid + physics of one domain.  Mirrors the keyword set of
 * BoussinesqSimulation (src/Simulations.jl:232-246) and of the sound-proof
 * MassWeightedSimulation (src/Anelastic.jl:1559), the mesh of RegularGrid /
 * StretchedGrid (src/Grids.jl:98, src/StretchedGrids.jl:345) and the
 * FieldBoundaryConditions kinds of src/BoundaryConditions.jl:54-74
 * (x, y periodic; z periodic or ImpermeableWall). */
typedef struct {
    int32_t nx, ny, nz;        /* interior cells (nx even)                     */
    int32_t hx, hy, hz;        /* halo widths of the HOST storage arrays       */
    double lx, ly, lz;         /* domain extent                                */
    double x0, y0, z0;         /* origin                                       */
    int32_t bc_x, bc_y, bc_z;  /* AEO_BC_*; x and y must be periodic           */
    int32_t stretched;         /* 1: zf gives the Nz+1 interior face heights   */
    int32_t core;              /* AEO_CORE_*                                   */
    int32_t advection;         /* AEO_ADV_* (momentum and theta)               */
    int32_t solver;            /* AEO_SOLVER_FFT (triply periodic), COLUMN, or
                                  PCG (any core and column: aeo_set_pcg)        */
    int32_t precision;         /* AEO_PREC_*                                   */
    double nu;                 /* molecular viscosity / diffusivity (0 = off)  */
    double theta0;             /* Boussinesq reference theta (0 = no buoyancy) */
    double g;                  /* gravitational acceleration                   */
    double f_coriolis;         /* Coriolis parameter (0 = off)                 */
    double c_s;                /* Smagorinsky constant (0 = no SGS)            */
    double pr_t;               /* turbulent Prandtl number                     */
    double flux_bot, flux_top; /* prescribed wall fluxes of theta              */
    double sponge_alpha;       /* Rayleigh sponge rate (0 = off)               */
    double sponge_zstart;      /* sponge bottom                                */
    int32_t device;            /* CUDA device ordinal                          */
    int32_t sgs_model;         /* AEO_SGS_* when c_s > 0: Smagorinsky (nu_t =
                                  (c_s Delta)^2 |S|), Vreman (2004), c =
                                  2.5 c_s^2 (compute_vreman_nut!,
                                  src/operators/sgs_amd_vreman.jl:280-298), or
                                  the sigma model, (c_s Delta)^2 D_sigma with
                                  c_s = C_sigma (compute_sigma_nut!,
                                  src/operators/sigma_closure.jl:208-222);
                                  or the anisotropic minimum-dissipation
                                  closure with c_s = its constant C (0.3 in
                                  the reference) and its own kappa_t
                                  (AMDClosure / compute_amd_coefficients!,
                                  src/operators/sgs_amd_vreman.jl:109-212,
                                  :325-354; g / theta_bar(z) on the sound-
                                  proof core, aeo_set_sgs_buoyancy); or dynamic
                                  Smagorinsky (Germano-Lilly, plane-averaged,
                                  test filter 3x3x3 with width ratio 3) with
                                  c_s = the clip cs_max (0.5 in the reference;
                                  DynamicSmagorinsky,
                                  src/Operators.jl:497-900), or the same with
                                  averaging = :local (each cell its own
                                  clipped ratio, _local_cs2_body!,
                                  src/Operators.jl:873-880), or the
                                  Lagrangian dynamic closure with c_s =
                                  cs_max (LagrangianDynamicSmagorinsky,
                                  aeo_set_lagrangian), or the prognostic-TKE
                                  closure with c_s = c_k (0.1; TKEClosure,
                                  aeo_set_tke; Boussinesq core, halos >= 3).
                                  Vreman, sigma, AMD, dynamic, Lagrangian
                                  and TKE on uniform grids                   */
} aeo_config;

typedef struct aeo_sim aeo_sim;

/* Create a domain.  zf: Nz+1 interior face heights when cfg->stretched
 * (StretchedGrid(stretching = (:custom, zf))), else NULL.  Anelastic core:
 * wc (Nz+2Hz) and wf (Nz+2Hz+1) are the halo-padded constraint weights
 * (ReferenceState.ρ̄c_pad / ρ̄f_pad, src/Anelastic.jl:232-233, :375-380) and
 * thf (Nz+2Hz+1) the padded face reference theta (θ̄f_pad) of the buoyancy;
 * NULL for the Boussinesq core.  Replaces the constructors
 * BoussinesqSimulation (src/Simulations.jl:232) and the sound-proof
 * simulation of src/Anelastic.jl:1559 together with their default pressure
 * solvers (_default_solver, src/Simulations.jl:1137; DirectWeightedPoissonSolver,
 * src/Anelastic.jl:997). */
aeo_status aeo_create(const aeo_config* cfg, const double* zf, const double* wc,
                      const double* wf, const double* thf, aeo_sim** out);

/* Release the domain and all its device memory. */
aeo_status aeo_destroy(aeo_sim* h);

/* Copy a host Field.data array (storage layout, halos ignored on input) into
 * the domain.  Replaces writes into sim.u/v/w/θ.data (src/Simulations.jl:201-206)
 * followed by fill_state_halos! (src/Simulations.jl:1028). */
aeo_status aeo_set_field(aeo_sim* h, int32_t field, const double* host);

/* Copy a field to a host Field.data array (storage layout).  u, v, w, θ come
 * back with halos filled from the interior by the boundary conditions
 * (fill_halos!, src/boundary_conditions/halo_sets.jl:176); p and νt with
 * zero halos.  νt (the `max_νt` diagnostic, src/Simulations.jl:1058) is the
 * Smagorinsky viscosity of the current state: the step itself keeps νt in
 * shared memory only. */
aeo_status aeo_get_field(aeo_sim* h, int32_t field, double* host);
/* The same with FP32 host arrays (half the host<->device bytes; the values
 * are the FP32 roundings of the FP64 ones, exact for an FP32-mixed domain's
 * stored state).  No reference counterpart: a Float32 host mirror of the
 * fields for AEO_PREC_FP32_MIXED domains. */
aeo_status aeo_set_field_f32(aeo_sim* h, int32_t field, const float* host);
aeo_status aeo_get_field_f32(aeo_sim* h, int32_t field, float* host);

/* nsteps projected SSP-RK3 steps of size dt: step_rk3! of the Boussinesq
 * core (src/Simulations.jl:843-904) or of the sound-proof core
 * (src/Anelastic.jl:1905-1948).  The whole step is one CUDA graph; with
 * nsteps >= 2 the pairs of steps run as one launch of a graph whose
 * conditional WHILE node loops over a two-step body (an odd last step is
 * launched on its own), bit-identical to single steps. */
aeo_status aeo_step_rk3(aeo_sim* h, double dt, int32_t nsteps);

/* nsteps forward-Euler projection steps: step! (src/Simulations.jl:481-650,
 * src/Anelastic.jl:1747-1876). */
aeo_status aeo_step_euler(aeo_sim* h, double dt, int32_t nsteps);

/* CFL constraints and guard limits of the adaptive step: CFLConstraints
 * (src/TimeIntegration.jl:127-153; defaults C_advective 0.5, C_diffusive
 * 0.25, C_buoyancy 0.5, C_coriolis 0.5, dt_min 1e-8, dt_max Inf,
 * growth_max 1.1) and step_adaptive!'s divergence_tol (1e-6), max_velocity
 * (Inf) and max_retries (3) (src/TimeIntegration.jl:823-835). */
typedef struct {
    double c_advective, c_diffusive, c_buoyancy, c_coriolis;
    double dt_min, dt_max, growth_max;
    double divergence_tol, max_velocity;
    int32_t max_retries;
} aeo_cfl;

/* What an adaptive step reports: the last accepted dt, the time advanced, the
 * limiter of the pick (0 advective, 1 diffusive, 2 buoyancy, 3 Coriolis,
 * 4 sgs, 5 growth, 6 dt_min, 7 dt_max, 8 retried), the retries, the pick's
 * advective rate max Σ|u_i|/Δx_i, max νt, Brunt-Väisälä frequency, and the
 * guard's max |∇·u| and max speed of the new state. */
typedef struct {
    double dt, t_advanced;
    int32_t limiter, retries;
    double advective_rate, nut_max, brunt_vaisala, max_divergence, max_speed;
} aeo_adaptive_stats;

/* nsteps adaptive SSP-RK3 steps: step_adaptive! (src/TimeIntegration.jl:808-938)
 * with adaptive_dt (:436-454) evaluated on the device inside the step's CUDA
 * graph.  *dt_prev in: the previous dt (<= 0: none, no growth limit); out: the
 * last accepted dt.  A step whose guard fails (non-finite state, divergence
 * above the tolerance, speed above the cap) is retried from the unchanged
 * step-start state with half the dt, up to max_retries times; then the call
 * returns AEO_ERR_NUMERICAL with the state of the start of that step. */
aeo_status aeo_step_adaptive(aeo_sim* h, const aeo_cfl* c, int32_t nsteps, double* dt_prev,
                             aeo_adaptive_stats* stats);

/* cfl_diagnostics + adaptive_dt of the current state (src/TimeIntegration.jl:291-454):
 * the dt the next adaptive step would take and its limiter, without stepping. */
aeo_status aeo_cfl_diagnostics(aeo_sim* h, const aeo_cfl* c, double dt_prev, aeo_adaptive_stats* out);

/* The projection's Poisson solve on interior-sized arrays (Nx*Ny*Nz, x
 * fastest): solve!(p, source, solver) / solve_source_buffer! of the
 * AbstractPressureSolver seam (src/PressureSolvers.jl:41-80, :162-174,
 * :712-732).  Zero-mean gauge (FFT) or the column solver's gauge. */
aeo_status aeo_pressure_solve(aeo_sim* h, const double* src, double* phi);

/* Project the current velocity onto the discretely solenoidal fields (one
 * Chorin projection with dt = 1, p = phi): the config driver's
 * `_project!(sim, 1.0)` of a noisy initial field
 * (src/config/simulation_driver.jl:1316; src/Simulations.jl:711-744). */
aeo_status aeo_project(aeo_sim* h);

/* Fill u, v, w with the random-phase isotropic field of the Passot-Pouquet
 * spectrum E(k) = 16 sqrt(2/pi) u_rms^2 k^4/k_peak^5 exp(-2 (k/k_peak)^2):
 * isotropic_turbulence_field! with PassotPouquetSpectrum
 * (src/operators/spectra.jl:248-343; SplitMix64 mode hash, modes with
 * |k| <= kmax, kmax <= 0 for no cut-off), generated on the device.  Then,
 * when `project` is non-zero, one Chorin projection (aeo_project), and when
 * target_rms > 0 a rescaling of u, v, w to that per-component rms.  Triply
 * periodic uniform grids only. */
aeo_status aeo_init_isotropic(aeo_sim* h, double u_rms, double k_peak, uint64_t seed, double kmax,
                              int32_t project, double target_rms);

/* kinetic_energy (src/Simulations.jl:992-1014) and max_divergence
 * (src/Simulations.jl:1045-1050; the W-normalised residual
 * (1/W)∇·(W u) for the anelastic core, src/Anelastic.jl:1134-1142). */
aeo_status aeo_kinetic_energy(aeo_sim* h, double* out);
aeo_status aeo_max_divergence(aeo_sim* h, double* out);

/* Device-resident stepping for benchmarks and graph-captured drivers: the
 * same as aeo_step_rk3 but returns without synchronising the stream. */
aeo_status aeo_step_rk3_async(aeo_sim* h, double dt, int32_t nsteps);
aeo_status aeo_synchronize(aeo_sim* h);

/* Kernel classes of one substage, for aeo_profile_step. */
enum { AEO_K_SGS = 0, AEO_K_SWEEP = 1, AEO_K_DIV_FFTX = 2, AEO_K_FFTY = 3, AEO_K_ZSOLVE = 4,
       AEO_K_IFFTX = 5, AEO_K_CORRECT = 6, AEO_K_HALO = 7, AEO_K_NCLASS = 8 };

/* One RK3 step run launch by launch (not as a graph) with CUDA events
 * recorded on the handle's stream between kernel groups; ms_per_class[c]
 * receives the summed device time of class c over the step.  Advances the
 * state like aeo_step_rk3.  The reference's per-stage wall times of
 * StepRecord (src/simulations/step_record.jl:1-263) are the analogue. */
aeo_status aeo_profile_step(aeo_sim* h, double dt, double* ms_per_class, int32_t nclass);

/* The implicit immersed-boundary correction after every predictor: replaces
 *   step!/step_rk3!(sim, dt; post_predictor! = (s, dt) -> implicit_ibm_correction!(s, sm; tau, dt = dt))
 *                                   src/IBM.jl:295-300, src/Simulations.jl:624-628
 * mask: storage-shaped bytes (the SolidMask of src/IBM.jl:33, nonzero =
 * solid; the interior cells count), NULL switches the correction off.  Every
 * predictor face of a solid cell is scaled by 1/(1 + dt/tau), once per solid
 * cell it touches (tau = 0: zeroed).  Not with AEO_SOLVER_PCG (obstacles are
 * apertures there). */
aeo_status aeo_set_ibm(aeo_sim* h, const uint8_t* mask, double tau);

/* Positivity-preserving scalar advection: replaces
 *   advect_positive!(tend, u, v, w, phi, dt; scheme, accumulate)
 *                                   src/AdvectionSchemes.jl:1141-1160
 * with the limiter of apply_positivity_limiter! (:998-1098, upwind low-order
 * fluxes, the one-layer periodic wrap of the ratio: no boundary conditions).
 * Adds (accumulate = 1) or writes -div(u phi) into the interior of tend so
 * that phi + dt * tend stays >= 0 where phi >= 0 and sum |u_d| dt/dx_d <= 1.
 * u, v, w, phi, tend are arrays of the domain's storage layout (the layout of
 * aeo_set_field), halos filled, hx, hy, hz >= 3; scheme AEO_ADV_WENO_JS5 or
 * AEO_ADV_WENO_Z5; a uniform grid.  The host form takes FP64 host arrays and
 * synchronises; the device form takes device arrays of the domain's working
 * precision (double for AEO_PREC_FP64, float for AEO_PREC_FP32_MIXED) and is
 * enqueued on the domain's stream (aeo_stream). */
aeo_status aeo_advect_positive(aeo_sim* h, const double* u, const double* v, const double* w, const double* phi,
                               double* tend, double dt, int32_t scheme, int32_t accumulate);
aeo_status aeo_advect_positive_device(aeo_sim* h, const void* u, const void* v, const void* w, const void* phi,
                                      void* tend, double dt, int32_t scheme, int32_t accumulate);

/* Number of kernel launches one RK3 step issues (for launch accounting).
   solver = AEO_SOLVER_PCG: counted with the iteration count of the last
   pressure solve for all three substages (synchronises the stream). */
aeo_status aeo_launches_per_step(aeo_sim* h, int32_t* out);

/* The handle's CUDA stream (a cudaStream_t) for callers that time kernels. */
void* aeo_stream(aeo_sim* h);

/* Philox4x32-10 uniform fill on the device: out[i] = amp*(2*U(seed, stream, i)-1)
 * for i < n, written into the given field's interior in storage order
 * (the synthetic-input generator of Backends.counter_rng, src/Backends.jl:1607-1739).
 * mode 0 overwrites, mode 1 adds. */
aeo_status aeo_fill_uniform(aeo_sim* h, int32_t field, uint64_t seed, uint32_t stream,
                            double amp, int32_t mode);

/* The column pressure solve (x, y periodic; zero-flux walls in z) without a
 * handle and without allocating device memory.  This entry point has no
 * counterpart in the reference.  It is for callers that cannot call
 * cudaMalloc: a host runtime whose device memory must all come from its own
 * pool or budget, an application that reserves every byte at start-up, or
 * a stepping loop that cannot afford cudaMalloc's implicit synchronisation.
 * Its scratch (twiddles, eigenvalues, coefficients and the (nx/2+1)*ny*nz
 * complex FP64 spectrum) lives in one static 32 MiB device array of this
 * library, held by every GPU that loads it until the process exits; a grid
 * whose scratch does not fit is rejected with AEO_ERR_ARGUMENT.  Operator:
 * the ColumnTridiagonalSolver coefficients lower, upper, hweight, measure
 * (nz each), inv_coupling (nz+1) and gauge (nz), host arrays; src and phi
 * are caller-owned device arrays of nx*ny*nz doubles (x fastest).  It runs
 * on `stream` on the current device: it copies the six host coefficient
 * arrays to the scratch, launches the solve and returns after that stream
 * has synchronised; a stream that is capturing a graph is refused with
 * AEO_ERR_ARGUMENT, as are a zero sum of measure or of gauge.  Every call
 * looks up the scratch array's device address on the current device (the
 * lookup allocates nothing, and after a cudaDeviceReset it finds the array
 * of the new context);
 * the first call on a device also loads the library's device code there,
 * so make that first call before any stream capture begins on the device.
 * Calls share the scratch: calls that overlap on the GPU (other streams,
 * other host threads) race. */
aeo_status aeo_pressure_solve_column_noalloc(int32_t nx, int32_t ny, int32_t nz, double lx, double ly,
                                             const double* lower, const double* upper,
                                             const double* hweight, const double* measure,
                                             const double* inv_coupling, const double* gauge,
                                             const double* src, double* phi, void* stream);

/* The AMD closure's buoyancy parameter of every interior level, Nz values:
 * g / theta_bar(z_k) of the sound-proof core's reference state at the cell
 * centres (sgs_buoyancy_parameter / _LevelBuoyancy,
 * src/operators/sgs_amd_vreman.jl:331-345, which AMDClosure passes to
 * compute_amd_coefficients!, :346-351).  Required before the first step of
 * an anelastic domain with the AMD closure (AEO_ERR_STATE otherwise); the
 * Boussinesq core uses g / theta0 and needs no call. */
aeo_status aeo_set_sgs_buoyancy(aeo_sim* h, const double* bg);

/* The Lagrangian dynamic closure (sgs_model = AEO_SGS_LAGRANGIAN;
 * LagrangianDynamicSmagorinsky(mesh; C0, theta, memory_time),
 * src/operators/lagrangian_sgs.jl:163-199, the scale-invariant model with
 * cadence 1 and no mask; c_s is cs_max): the initial coefficient C0 (0.16),
 * the time-scale factor theta (1.5) and a fixed memory_time (0: MLC96's T =
 * theta Delta (I_LM I_MM)^(-1/8)).  A new domain has the defaults; the call
 * recomputes the coefficient of the committed memory.  AEO_ERR_STATE on a
 * domain with another closure. */
aeo_status aeo_set_lagrangian(aeo_sim* h, double c0, double theta, double memory_time);

/* sgs_state / restore_sgs_state! of the closures with a memory.  The
 * Lagrangian closure (src/operators/lagrangian_sgs.jl:372-381): 5 Nx Ny Nz + 1
 * doubles -- the committed I_LM, I_MM and the cell-centred u, v, w the memory
 * was committed with (interior arrays, x fastest), then the initialised flag
 * (0 / 1); setting it recomputes the coefficient the next step uses.  The TKE
 * closure (src/PrognosticSGS.jl:1174-1197): e on the interior, Nx Ny Nz
 * doubles >= 0 (its initial value; a new domain has e = 0, a fixed point of
 * the TKE equation).  AEO_ERR_STATE on a domain whose closure keeps no
 * memory. */
aeo_status aeo_get_sgs_state(aeo_sim* h, double* out);

/* The TKE closure (sgs_model = AEO_SGS_TKE; TKEClosure(mesh; c_k, c_eps0,
 * c_eps1, c_l, dissipation), src/PrognosticSGS.jl:326-375, without a mask,
 * wall cap, first-level factor or surface value; c_s is c_k): c_eps0 (0.19),
 * c_eps1 (0.51), c_l (0.76) and the dissipation form (0 :semi_implicit, 1
 * :exact).  e is committed once per step after the projection (advance_sgs!,
 * :978-1002): WENO-Z5 flux-limited transport, div(2 nu_t grad e), the shear
 * production of the discrete dual of the momentum operator, the buoyancy
 * production (with (g/theta0) F / 2 of the surface heat fluxes in the wall
 * levels) and the implicit sinks.  AEO_ERR_STATE on another closure. */
aeo_status aeo_set_tke(aeo_sim* h, double c_eps0, double c_eps1, double c_l, int32_t exact);
aeo_status aeo_set_sgs_state(aeo_sim* h, const double* in);

/* The pressure solve of a domain created with solver = AEO_SOLVER_PCG:
 * conjugate gradients preconditioned by one multigrid V(2,2) cycle
 * (MGPreconditionedCG, src/Multigrid.jl:893-967, the urban :mg_cg slot of
 * src/components/urban/pressure_solver.jl:126) on cut-cell face apertures.
 * ax ((nx+1)*ny*nz), ay (nx*(ny+1)*nz), az (nx*ny*(nz+1)): host FP64
 * apertures in [0, 1] in the face layout of aeolus_b200_mgpcg.h (face i the
 * west / south / bottom face of cell i), all NULL for every face open; the
 * wall faces of a bounded z are blocked whatever is given.  The projection
 * solves the a^2-weighted Laplacian against the aperture-weighted
 * divergence of the predictor (cutcell_divergence! times vol_eff,
 * src/CutCell.jl:602-623) and corrects with the aperture-scaled gradient
 * (cutcell_gradient_x/y/z!, :666-700), so a blocked face carries no velocity
 * (apply_cutcell_velocity_bc!, :852-880) and the aperture-weighted
 * divergence after a projection is the solve's residual.  On the
 * sound-proof core the fluxes carry the density weights of
 * DensityWeightedPoissonSolver (src/Anelastic.jl:734-793: W_c on x and y
 * faces, W_f on z faces; the :density_weighted_cg slot,
 * src/components/urban/pressure_solver.jl:182-191) and on a stretched column
 * the z metrics, both in the symmetric form the multigrid hierarchy takes
 * (every equation times dz_c/h_z, h_z = lz/nz).  Every solve runs to
 * ||r|| <= tol ||b|| or maxit iterations (defaults 1e-8, 200); the solve's
 * CG loop is a conditional node inside the step's graph.  aeo_max_divergence
 * reports the aperture-weighted (density-weighted) divergence on these
 * domains.  No reference counterpart for the learned
 * preconditioner (aeo_pcg_set_learned: the U-Net of aeolus_b200_unet.h with
 * its stagnation fallback to the cycle; net NULL switches back). */
struct aeo_unet;
aeo_status aeo_set_pcg(aeo_sim* h, const double* ax, const double* ay, const double* az, double tol, int32_t maxit);
/* the statistics of the last projection's solve (iterations, AEO_MG_* status,
 * ||r||, ||b - mean(b)||); synchronises the handle's stream */
aeo_status aeo_pcg_stats(aeo_sim* h, int32_t* iterations, int32_t* status, double* residual, double* bnorm);
aeo_status aeo_pcg_set_learned(aeo_sim* h, struct aeo_unet* net, double stagnation);
/* Open lateral faces: Dirichlet halos from boundary data, the replacement of
 * OpenBoundary / open_boundary_conditions(mesh, data; x, y, ...) and its halo
 * fills (src/boundary_conditions/open_boundary.jl:485-638, :722-807).
 * open_x / open_y open both faces of an axis (the other axis stays
 * periodic); bottom and top stay walls.  x_planes: [field][side][NZ][NY][H+1],
 * y_planes: [field][side][NZ][H+1][NX] (FP64; field u, v, w, theta; side 0
 * west/south, 1 east/north; NX, NY, NZ the storage extents Nx+2H, Ny+2H,
 * Nz+2H; layer = storage index along the face normal on the low side, that
 * index - (H + N) on the high side, so the low side's layer H is the normal
 * velocity's boundary face, interior index 0): the data at those storage
 * points with the normal velocities already mass-corrected
 * (correct_boundary_mass_flux!, :1024-1083).  modes[4]: 0 the field takes its
 * plane, 1 the zero-gradient mirror (theta only: scalar_halo = :mirror); every
 * other field (the pressure) takes the mirror, so the projection's phi has
 * d phi / dn = 0 there and leaves the prescribed normal velocity unchanged.
 * Needs solver = AEO_SOLVER_PCG on the uniform Boussinesq core with walls in z;
 * of the SGS closures the static ones (Smagorinsky, Vreman, sigma, AMD), whose
 * nu_t takes the mirror across the open faces; the planes are steady (the
 * step does not refresh them).
 * open_x = open_y = 0 closes the faces again. */
aeo_status aeo_set_open(aeo_sim* h, int32_t open_x, int32_t open_y, const double* x_planes, const double* y_planes,
                        const int32_t* modes);
/* Radiating outflow of the open faces set by aeo_set_open (the :convective
 * outflow of open_boundary_conditions, src/boundary_conditions/outflow.jl):
 * radiate[4] (west, east, south, north) 0 = :dirichlet, 1 = :convective,
 * 2 = :orlanski (the tangential velocities and theta take the Orlanski 1976
 * phase speed of the interior layer next to the face between this and the
 * previous step start, clipped to [0, dn/dtau]; the normal velocity and the
 * first step the convective one; outflow.jl:136-182);
 * correction 0 :uniform, 1 :outflow_only, 2 :none; x_data / y_data the raw
 * boundary data (before the correction) in aeo_set_open's layout.  Each step
 * then fixes, at its start, the outflow points (outward normal velocity of
 * the boundary face > 0) and their phase speed c = that velocity
 * (prepare_open_boundaries!, open_boundary.jl:1189-1200); before every
 * projection it refills the planes from the data, advances the outflow
 * points by the second-order upstream radiation update from the stage-start
 * values, r = min(c dt / dn, 1), and applies the mass-flux correction
 * (update_open_boundaries!, :1137-1152; _radiate_body!, outflow.jl:262-285);
 * RK3 stages combine the planes like the fields (combine_open_boundaries!,
 * :1262-1280).  x_weights [side][Nz][Ny] / y_weights [side][Nz][Nx] (NULL: 1)
 * weight each normal boundary face in the correction: 0 a solid face
 * (mark_open_boundary_solids!, :809-868), else its open fraction (the
 * projection's aperture there, so the corrected planes carry no net flux the
 * cut-cell divergence sees).  Not with aeo_step_adaptive (AEO_ERR_STATE). */
aeo_status aeo_set_open_outflow(aeo_sim* h, const int32_t* radiate, int32_t correction, const double* x_data,
                                const double* y_data, const double* x_weights, const double* y_weights);
/* Q, residual and delta of the last mass-flux correction of a radiating open
 * set (open_boundary_ledger, open_boundary.jl:1437-1450); synchronises */
aeo_status aeo_open_ledger(aeo_sim* h, double* out);
/* The current open-face plane buffers in aeo_set_open's layout (FP64): on a
 * radiating face they are state, the radiated outflow points included
 * (open_boundary_checkpoint, src/boundary_conditions/open_boundary.jl:1282-1305);
 * synchronises */
aeo_status aeo_get_open_planes(aeo_sim* h, double* x_planes, double* y_planes);
/* A checkpoint's planes back into the buffers (restore_open_boundary_checkpoint!,
 * open_boundary.jl:1307-1350; the open set itself as built by aeo_set_open /
 * aeo_set_open_outflow); the state's halos refilled */
aeo_status aeo_set_open_planes(aeo_sim* h, const double* x_planes, const double* y_planes);
/* The Orlanski history of a radiating set (hist, t_hist, has_hist of the
 * checkpoint): x_hist [field][side][NZ][NY], y_hist [field][side][NZ][NX],
 * scalars = (history set, the last step's length) */
aeo_status aeo_get_open_history(aeo_sim* h, double* x_hist, double* y_hist, double* scalars);
aeo_status aeo_set_open_history(aeo_sim* h, const double* x_hist, const double* y_hist, const double* scalars);
/* Residual -> error pairs from the run's own snapshots (no reference
 * counterpart; it feeds the learned preconditioner): b receives the
 * right-hand side of the last projection's solve (the predictor's cut-cell
 * divergence of the last substage, nx*ny*nz FP64, x fastest), which the
 * plain MG-preconditioned CG solves again from a zero guess; x receives its
 * converged solution, r_hist / x_hist (cap * nx*ny*nz each) the residual
 * r_k and iterate x_k of iterations k = 0 .. count-1, so that A (x - x_k) =
 * r_k.  AEO_ERR_STATE while a learned preconditioner is set or before a
 * projection has run; synchronises the handle's stream. */
aeo_status aeo_pcg_harvest(aeo_sim* h, int32_t cap, double* b, double* x, double* r_hist, double* x_hist,
                           int32_t* count);

/* Last error message of the handle (or of the last failed aeo_create when h is NULL). */
const char* aeo_last_error(const aeo_sim* h);

/* Library version string. */
const char* aeo_version(void);

#ifdef __cplusplus
}
#endif
#endif
