/*
 * aeolus_b200_mgpcg.h -- C ABI of the multigrid-preconditioned conjugate
 * gradient solver for div(c grad phi) = b on a uniform Cartesian grid: the
 * cut-cell pressure solve (face coefficients c = aperture^2,
 * src/CutCell.jl:735-768, solved in the symmetric form vol_eff L,
 * src/CutCell.jl:705-716) and the variable-coefficient Poisson solve of the
 * reference's MultigridPoissonSolver / MGPreconditionedCG.
 *
 * Replaces (reference file:line)
 *   MGPreconditionedCG(mesh; coeff_x, coeff_y, coeff_z, bc_x, bc_y, bc_z,
 *                      tol, maxit, nu1, nu2, min_size, mg_cycles)
 *                                              src/Multigrid.jl:893-901  -> aeo_mg_create
 *   solve!(p, source, ::MGPreconditionedCG)    src/Multigrid.jl:955-967  -> aeo_mg_solve
 *   pcg!(A, M, x, b, ws; tol, maxit, project_mean, definite = :negative)
 *                                              src/Backends.jl:1511-1589 -> aeo_mg_solve
 *   mg_solve!(solver, phi, rhs)                src/Multigrid.jl:801-840  -> aeo_mg_vcycle_solve
 *   _apply_fine!(out, x, solver)               src/Multigrid.jl:911-919  -> aeo_mg_apply
 *   _mg_precond!(z, r, solver)                 src/Multigrid.jl:922-932  -> aeo_mg_precondition
 *   mg_level_count(solver)                     src/Multigrid.jl:670      -> aeo_mg_levels
 *
 * Arrays on this interface are interior-only FP64, x fastest: a cell array
 * is nx*ny*nz doubles; face coefficients are cx (nx+1)*ny*nz, cy
 * nx*(ny+1)*nz, cz nx*ny*(nz+1), face index i the west (south, bottom) face
 * of cell i.  Status codes are those of aeolus_b200.h.
 */
#ifndef AEOLUS_B200_MGPCG_H
#define AEOLUS_B200_MGPCG_H

#include <stdint.h>

#include "aeolus_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

enum { AEO_MG_PERIODIC = 0, AEO_MG_NEUMANN = 1 };
/* preconditioner of the CG iteration: none (plain CG), one multigrid cycle
 * per application (the reference's MGPreconditionedCG), or the learned U-Net
 * of aeolus_b200_unet.h (set by aeo_mg_set_learned; no reference counterpart) */
enum { AEO_PC_IDENTITY = 0, AEO_PC_VCYCLE = 1, AEO_PC_LEARNED = 2, AEO_PC_JACOBI = 3 };
/* AEO_PC_JACOBI: z = r / diag(A) (the Jacobi-preconditioned CG of the
 * density-weighted projection, DensityWeightedPoissonSolver,
 * src/components/urban/pressure_solver.jl:18-20) */
/* solve status (the reference's :converged, :maxit, :breakdown, :zero_rhs) */
enum { AEO_MG_CONVERGED = 0, AEO_MG_MAXIT = 1, AEO_MG_BREAKDOWN = 2, AEO_MG_ZERO_RHS = 3 };

typedef struct {
    int32_t nx, ny, nz;
    double dx, dy, dz;
    int32_t bc_x, bc_y, bc_z;  /* AEO_MG_PERIODIC / AEO_MG_NEUMANN per axis */
    int32_t precision;         /* AEO_PREC_FP64: every array FP64 (the reference's arithmetic);
                                  AEO_PREC_FP32_MIXED: the multigrid cycle in FP32, the Krylov
                                  vectors, the operator and every reduction in FP64 */
    int32_t precond;           /* AEO_PC_* */
    int32_t flexible;          /* 0: beta = (r.z)_new / (r.z)_old as the reference;
                                  1: Polak-Ribiere beta (flexible CG, robust to an inexact cycle) */
    double tol;                /* ||r|| <= tol ||b|| (reference default 1e-10) */
    int32_t maxit;             /* CG iterations (aeo_mg_solve) or cycles (aeo_mg_vcycle_solve) */
    int32_t nu1, nu2;          /* red-black Gauss-Seidel sweeps before / after the coarse correction */
    int32_t coarse_sweeps;     /* sweeps on the coarsest level (reference: 50) */
    int32_t min_size;          /* coarsen while every dimension is even and its half >= min_size */
    int32_t device;
} aeo_mg_config;

typedef struct {
    int32_t iterations;        /* CG iterations, or cycles for aeo_mg_vcycle_solve */
    int32_t status;            /* AEO_MG_* */
    double residual;           /* ||r|| of the last iterate (relative for aeo_mg_vcycle_solve) */
    double bnorm;              /* ||b - mean(b)|| */
    double curvature;          /* the last p.Ap formed (NaN if none) */
    int32_t fallback_at;       /* learned preconditioner: the iteration it was dropped for the
                                  multigrid cycle after stagnating, -1 if never */
} aeo_mg_stats;

typedef struct aeo_mg aeo_mg;
struct aeo_unet;

/* cx, cy, cz: host face coefficients, or all NULL for the constant-coefficient
 * Laplacian.  Fails with AEO_ERR_ARGUMENT when the coarsest level exceeds
 * 16384 cells (give the grid more factors of two). */
aeo_status aeo_mg_create(const aeo_mg_config* cfg, const double* cx, const double* cy, const double* cz,
                         aeo_mg** out);
aeo_status aeo_mg_destroy(aeo_mg* h);
/* number of levels, and their (nx, ny, nz) in dims[3*l..3*l+2] (dims may be NULL) */
aeo_status aeo_mg_levels(aeo_mg* h, int32_t* nlevels, int32_t* dims);
/* x = A^-1 b by preconditioned CG from a zero guess, x of zero mean when every
 * axis is periodic or Neumann; host arrays; synchronous */
aeo_status aeo_mg_solve(aeo_mg* h, const double* b, double* x, aeo_mg_stats* stats);
/* the same with FP64 device arrays on the handle's device */
aeo_status aeo_mg_solve_device(aeo_mg* h, const double* b_dev, double* x_dev, aeo_mg_stats* stats);
/* repeated multigrid cycles until the relative residual is below tol (mg_solve!) */
aeo_status aeo_mg_vcycle_solve(aeo_mg* h, const double* b, double* x, aeo_mg_stats* stats);
/* out = A x (host arrays) */
aeo_status aeo_mg_apply(aeo_mg* h, const double* x, double* out);
/* z = M r, one preconditioner application, z deflated to zero mean for a singular operator */
aeo_status aeo_mg_precondition(aeo_mg* h, const double* r, double* z);
/* Device time of `reps` back-to-back launches of one part, after warm-up:
 * what = 0 the whole solve of the right-hand side of the last solve call,
 * 1 one red-black colour pass on the finest level, 2 the operator with its
 * p.Ap reduction, 3 one preconditioner application, 4 the coarsest-level
 * solve, 5 the residual restriction of the finest level, 6 one whole
 * red-black sweep of the finest level as the cycle runs it (one fused pass,
 * or the two colour passes).  ms_out: mean ms. */
aeo_status aeo_mg_profile(aeo_mg* h, int32_t what, int32_t reps, double* ms_out);
/* The learned preconditioner (no reference counterpart): `net` (same grid;
 * NULL detaches it) preconditions flexible CG from the next solve on.  When
 * an iteration's residual falls by less than `stagnation` (ratio of norms)
 * twice in a row, the solve switches to the multigrid cycle for its
 * remaining iterations, on the device inside the solve graph; every solve
 * still stops at ||r|| <= tol ||b||. */
aeo_status aeo_mg_set_learned(aeo_mg* h, struct aeo_unet* net, double stagnation);
/* aeo_mg_solve that also returns its residuals and iterates: slot k of
 * r_hist / x_hist (cap slots of nx*ny*nz doubles each) holds r_k and x_k
 * after k updates (slot 0: b - mean b and 0); *count = the slots filled.
 * The pairs (r_k, x - x_k) are residual -> error pairs of this solve (no
 * reference counterpart: the training data of the learned preconditioner). */
aeo_status aeo_mg_solve_harvest(aeo_mg* h, const double* b, double* x, aeo_mg_stats* stats, double* r_hist,
                                double* x_hist, int32_t cap, int32_t* count);
/* kernel launches of one CG iteration (graph body) */
int32_t aeo_mg_launches_per_iteration(const aeo_mg* h);
const char* aeo_mg_last_error(const aeo_mg* h);

#ifdef __cplusplus
}
#endif
#endif
