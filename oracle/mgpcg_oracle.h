/*
 * mgpcg_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU FP64 restatement of the reference's geometric multigrid and its
 * multigrid-preconditioned conjugate gradients for the variable-coefficient
 * Poisson operator div(c grad phi) (src/Multigrid.jl:174-967 and
 * pcg!/_pcg! in src/Backends.jl:1262-1589).  The face coefficients of a
 * cut-cell grid are the squared apertures (src/CutCell.jl:735-768), so this
 * is also the cut-cell pressure solve.  Nothing in the product path links,
 * loads or calls this code.
 *
 * Arrays are interior-only, x fastest: a cell array is nx*ny*nz doubles;
 * face coefficients are cx (nx+1)*ny*nz, cy nx*(ny+1)*nz, cz nx*ny*(nz+1),
 * face index i the west (south, bottom) face of cell i.
 */
#ifndef MGPCG_ORACLE_H
#define MGPCG_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { OCG_BC_PERIODIC = 0, OCG_BC_NEUMANN = 1 };
enum { OCG_PC_IDENTITY = 0, OCG_PC_VCYCLE = 1 };
enum { OCG_CONVERGED = 0, OCG_MAXIT = 1, OCG_BREAKDOWN = 2, OCG_ZERO_RHS = 3 };

typedef struct {
    int32_t nx, ny, nz;
    double dx, dy, dz;
    int32_t bc_x, bc_y, bc_z;
    double tol;
    int32_t maxit;         /* PCG iterations (MGPreconditionedCG maxit) or V-cycles (mg_solve!) */
    int32_t nu1, nu2;      /* RB-GS pre/post sweeps */
    int32_t coarse_sweeps; /* RB-GS sweeps on the coarsest level */
    int32_t min_size;      /* stop coarsening below this */
    int32_t mg_cycles;     /* V-cycles per preconditioner application */
    int32_t precond;       /* OCG_PC_* */
} ocg_params;

typedef struct {
    int32_t iterations, status;
    double residual, bnorm, curvature;
} ocg_stats;

typedef struct ocg ocg;

/* cx/cy/cz NULL: the constant-coefficient Laplacian */
ocg* ocg_create(const ocg_params* p, const double* cx, const double* cy, const double* cz);
void ocg_destroy(ocg* s);
int ocg_nlevels(const ocg* s);
int ocg_level_dims(const ocg* s, int lev, int32_t dims[3]);
int ocg_level_coeff(const ocg* s, int lev, double* cx, double* cy, double* cz);
int ocg_apply(ocg* s, const double* x, double* out);          /* _apply_fine! */
int ocg_precondition(ocg* s, const double* r, double* z);     /* _mg_precond! */
int ocg_solve(ocg* s, const double* b, double* x, ocg_stats* st);      /* solve!(MGPreconditionedCG) */
int ocg_mg_solve(ocg* s, const double* b, double* x, ocg_stats* st);   /* mg_solve! */

#ifdef __cplusplus
}
#endif
#endif
