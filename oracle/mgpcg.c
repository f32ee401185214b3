/*
 * mgpcg.c -- TEST INFRASTRUCTURE ONLY.  FP64 restatement of the reference's
 * multigrid V-cycle (src/Multigrid.jl) and preconditioned conjugate
 * gradients (src/Backends.jl pcg!).  Each function cites the lines it
 * follows.  Sums are plane sums in (j, i) order folded serially over k, the
 * shape of the reference's canonical reductions (src/Backends.jl:1349-1357).
 */
#include "mgpcg_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
    int nx, ny, nz;
    double dx, dy, dz, ix2, iy2, iz2;
    double *phi, *b, *r;        /* (nx+2)(ny+2)(nz+2), single-cell halo */
    double *cx, *cy, *cz;       /* face coefficients or NULL */
} level;

struct ocg {
    ocg_params p;
    int nlev, singular;
    level L[24];
    double *x, *rr, *z, *pp, *Ap, *bb;   /* PCG work, interior-sized */
};

#define IX(L, i, j, k) ((size_t)(i) + (size_t)((L)->nx + 2) * ((size_t)(j) + (size_t)((L)->ny + 2) * (size_t)(k)))
#define CXI(L, i, j, k) ((size_t)(i) + (size_t)((L)->nx + 1) * ((size_t)(j) + (size_t)(L)->ny * (size_t)(k)))
#define CYI(L, i, j, k) ((size_t)(i) + (size_t)(L)->nx * ((size_t)(j) + (size_t)((L)->ny + 1) * (size_t)(k)))
#define CZI(L, i, j, k) ((size_t)(i) + (size_t)(L)->nx * ((size_t)(j) + (size_t)(L)->ny * (size_t)(k)))

static size_t ncells(const level* L) { return (size_t)L->nx * L->ny * L->nz; }

/* fill_unit_halo!: x, then y, then z; periodic wraps, Neumann mirrors
 * (src/Multigrid.jl:77-78). */
static void fill_halo(level* L, int bx, int by, int bz) {
    int nx = L->nx, ny = L->ny, nz = L->nz;
    double* f = L->phi;
    for (int k = 0; k < nz + 2; ++k)
        for (int j = 0; j < ny + 2; ++j) {
            f[IX(L, 0, j, k)] = bx == OCG_BC_PERIODIC ? f[IX(L, nx, j, k)] : f[IX(L, 1, j, k)];
            f[IX(L, nx + 1, j, k)] = bx == OCG_BC_PERIODIC ? f[IX(L, 1, j, k)] : f[IX(L, nx, j, k)];
        }
    for (int k = 0; k < nz + 2; ++k)
        for (int i = 0; i < nx + 2; ++i) {
            f[IX(L, i, 0, k)] = by == OCG_BC_PERIODIC ? f[IX(L, i, ny, k)] : f[IX(L, i, 1, k)];
            f[IX(L, i, ny + 1, k)] = by == OCG_BC_PERIODIC ? f[IX(L, i, 1, k)] : f[IX(L, i, ny, k)];
        }
    for (int j = 0; j < ny + 2; ++j)
        for (int i = 0; i < nx + 2; ++i) {
            f[IX(L, i, j, 0)] = bz == OCG_BC_PERIODIC ? f[IX(L, i, j, nz)] : f[IX(L, i, j, 1)];
            f[IX(L, i, j, nz + 1)] = bz == OCG_BC_PERIODIC ? f[IX(L, i, j, 1)] : f[IX(L, i, j, nz)];
        }
}

/* _Aphi for _ConstOp / _VarOp (src/Multigrid.jl:174-193); (i,j,k) storage */
static double Aphi(const level* L, const double* f, int i, int j, int k) {
    double c = f[IX(L, i, j, k)];
    if (!L->cx) {
        return (f[IX(L, i + 1, j, k)] - 2 * c + f[IX(L, i - 1, j, k)]) * L->ix2 +
               (f[IX(L, i, j + 1, k)] - 2 * c + f[IX(L, i, j - 1, k)]) * L->iy2 +
               (f[IX(L, i, j, k + 1)] - 2 * c + f[IX(L, i, j, k - 1)]) * L->iz2;
    }
    int ii = i - 1, jj = j - 1, kk = k - 1;
    double fxp = L->cx[CXI(L, ii + 1, jj, kk)], fxm = L->cx[CXI(L, ii, jj, kk)];
    double fyp = L->cy[CYI(L, ii, jj + 1, kk)], fym = L->cy[CYI(L, ii, jj, kk)];
    double fzp = L->cz[CZI(L, ii, jj, kk + 1)], fzm = L->cz[CZI(L, ii, jj, kk)];
    return (fxp * (f[IX(L, i + 1, j, k)] - c) - fxm * (c - f[IX(L, i - 1, j, k)])) * L->ix2 +
           (fyp * (f[IX(L, i, j + 1, k)] - c) - fym * (c - f[IX(L, i, j - 1, k)])) * L->iy2 +
           (fzp * (f[IX(L, i, j, k + 1)] - c) - fzm * (c - f[IX(L, i, j, k - 1)])) * L->iz2;
}

/* canonical interior sum of a level array (src/Multigrid.jl:227-232) */
static double isum(const level* L, const double* a) {
    double s = 0;
    for (int k = 1; k <= L->nz; ++k) {
        double pk = 0;
        for (int j = 1; j <= L->ny; ++j)
            for (int i = 1; i <= L->nx; ++i) pk += a[IX(L, i, j, k)];
        s += pk;
    }
    return s;
}

static void shift(level* L, double* a, double m) {
    for (int k = 1; k <= L->nz; ++k)
        for (int j = 1; j <= L->ny; ++j)
            for (int i = 1; i <= L->nx; ++i) a[IX(L, i, j, k)] -= m;
}

static void project_mean(level* L, double* a) { shift(L, a, isum(L, a) / (double)ncells(L)); }

/* _compute_residual! (src/Multigrid.jl:281-285) */
static void residual(ocg* s, level* L) {
    fill_halo(L, s->p.bc_x, s->p.bc_y, s->p.bc_z);
    for (int k = 1; k <= L->nz; ++k)
        for (int j = 1; j <= L->ny; ++j)
            for (int i = 1; i <= L->nx; ++i)
                L->r[IX(L, i, j, k)] = L->b[IX(L, i, j, k)] - Aphi(L, L->phi, i, j, k);
}

/* _rbgs_sweeps! (src/Multigrid.jl:311-353): per colour, the halo fill then
 * the cells with (i + j + k) & 1 == colour (1-based storage indices); a cell
 * whose |diag| < eps is skipped. */
static void rbgs(ocg* s, level* L, int nsweeps) {
    double* f = L->phi;
    for (int sw = 0; sw < nsweeps; ++sw)
        for (int colour = 0; colour < 2; ++colour) {
            fill_halo(L, s->p.bc_x, s->p.bc_y, s->p.bc_z);
            for (int k = 1; k <= L->nz; ++k)
                for (int j = 1; j <= L->ny; ++j)
                    for (int i = 1; i <= L->nx; ++i) {
                        if (((i + 1 + j + 1 + k + 1) & 1) != colour) continue;
                        double off, diag;
                        if (!L->cx) {
                            diag = -2 * (L->ix2 + L->iy2 + L->iz2);
                            off = (f[IX(L, i + 1, j, k)] + f[IX(L, i - 1, j, k)]) * L->ix2 +
                                  (f[IX(L, i, j + 1, k)] + f[IX(L, i, j - 1, k)]) * L->iy2 +
                                  (f[IX(L, i, j, k + 1)] + f[IX(L, i, j, k - 1)]) * L->iz2;
                        } else {
                            int ii = i - 1, jj = j - 1, kk = k - 1;
                            double fxp = L->cx[CXI(L, ii + 1, jj, kk)], fxm = L->cx[CXI(L, ii, jj, kk)];
                            double fyp = L->cy[CYI(L, ii, jj + 1, kk)], fym = L->cy[CYI(L, ii, jj, kk)];
                            double fzp = L->cz[CZI(L, ii, jj, kk + 1)], fzm = L->cz[CZI(L, ii, jj, kk)];
                            diag = -((fxp + fxm) * L->ix2 + (fyp + fym) * L->iy2 + (fzp + fzm) * L->iz2);
                            if (fabs(diag) < DBL_EPSILON) continue;
                            off = (fxp * f[IX(L, i + 1, j, k)] + fxm * f[IX(L, i - 1, j, k)]) * L->ix2 +
                                  (fyp * f[IX(L, i, j + 1, k)] + fym * f[IX(L, i, j - 1, k)]) * L->iy2 +
                                  (fzp * f[IX(L, i, j, k + 1)] + fzm * f[IX(L, i, j, k - 1)]) * L->iz2;
                        }
                        f[IX(L, i, j, k)] = (L->b[IX(L, i, j, k)] - off) / diag;
                    }
        }
}

/* _restrict! (src/Multigrid.jl:380-406): coarse b = mean of the eight fine
 * (r - m), summed in the reference's order */
static void restrict_(level* C, const level* F, double m) {
    for (int K = 1; K <= C->nz; ++K)
        for (int J = 1; J <= C->ny; ++J)
            for (int I = 1; I <= C->nx; ++I) {
                int i = 2 * I - 1, j = 2 * J - 1, k = 2 * K - 1;   /* 0-based of 1-based 2I-2 */
                const double* r = F->r;
                double sum = (r[IX(F, i, j, k)] - m) + (r[IX(F, i + 1, j, k)] - m) +
                             (r[IX(F, i, j + 1, k)] - m) + (r[IX(F, i + 1, j + 1, k)] - m) +
                             (r[IX(F, i, j, k + 1)] - m) + (r[IX(F, i + 1, j, k + 1)] - m) +
                             (r[IX(F, i, j + 1, k + 1)] - m) + (r[IX(F, i + 1, j + 1, k + 1)] - m);
                C->b[IX(C, I, J, K)] = sum * 0.125;
            }
}

/* _prolong_add! (src/Multigrid.jl:412-455): trilinear (3/4, 1/4) weights,
 * accumulated near before far, dk then dj then di */
static void prolong_add(ocg* s, level* F, level* C) {
    fill_halo(C, s->p.bc_x, s->p.bc_y, s->p.bc_z);
    const double n = 3.0 / 4, f = 1.0 / 4;
    const double w[8] = {n * n * n, f * n * n, n * f * n, f * f * n, n * n * f, f * n * f, n * f * f, f * f * f};
    for (int ks = 1; ks <= F->nz; ++ks)
        for (int js = 1; js <= F->ny; ++js)
            for (int is = 1; is <= F->nx; ++is) {
                /* reference: i = is - 1 with 1-based is; here is is 0-based
                 * storage, so the 1-based interior index is is */
                int i = is, j = js, k = ks;
                int Ih = ((i + 1) >> 1), Ix = Ih + ((i & 1) ? -1 : 1);
                int Jh = ((j + 1) >> 1), Jy = Jh + ((j & 1) ? -1 : 1);
                int Kh = ((k + 1) >> 1), Kz = Kh + ((k & 1) ? -1 : 1);
                const double* P = C->phi;
                double acc = 0;
                acc += w[0] * P[IX(C, Ih, Jh, Kh)];
                acc += w[1] * P[IX(C, Ix, Jh, Kh)];
                acc += w[2] * P[IX(C, Ih, Jy, Kh)];
                acc += w[3] * P[IX(C, Ix, Jy, Kh)];
                acc += w[4] * P[IX(C, Ih, Jh, Kz)];
                acc += w[5] * P[IX(C, Ix, Jh, Kz)];
                acc += w[6] * P[IX(C, Ih, Jy, Kz)];
                acc += w[7] * P[IX(C, Ix, Jy, Kz)];
                F->phi[IX(F, is, js, ks)] += acc;
            }
}

/* _restrict_coeff (src/Multigrid.jl:465-496): four-face means */
static void restrict_coeff(const level* F, level* C) {
    int cnx = C->nx, cny = C->ny, cnz = C->nz;
    int sx1 = F->nx + 1, sx2 = F->ny, sx3 = F->nz;
    int sy1 = F->nx, sy2 = F->ny + 1, sy3 = F->nz;
    int sz1 = F->nx, sz2 = F->ny, sz3 = F->nz + 1;
#define MINI(a, b) ((a) < (b) ? (a) : (b))
    for (int K = 1; K <= cnz; ++K)
        for (int J = 1; J <= cny; ++J)
            for (int I = 1; I <= cnx + 1; ++I) {
                int i = 2 * I - 1;
                double sum = 0;
                for (int dk = 0; dk <= 1; ++dk)
                    for (int dj = 0; dj <= 1; ++dj)
                        sum += F->cx[CXI(F, MINI(i, sx1) - 1, MINI(2 * J - 1 + dj, sx2) - 1, MINI(2 * K - 1 + dk, sx3) - 1)];
                C->cx[CXI(C, I - 1, J - 1, K - 1)] = sum * 0.25;
            }
    for (int K = 1; K <= cnz; ++K)
        for (int J = 1; J <= cny + 1; ++J)
            for (int I = 1; I <= cnx; ++I) {
                int j = 2 * J - 1;
                double sum = 0;
                for (int dk = 0; dk <= 1; ++dk)
                    for (int di = 0; di <= 1; ++di)
                        sum += F->cy[CYI(F, MINI(2 * I - 1 + di, sy1) - 1, MINI(j, sy2) - 1, MINI(2 * K - 1 + dk, sy3) - 1)];
                C->cy[CYI(C, I - 1, J - 1, K - 1)] = sum * 0.25;
            }
    for (int K = 1; K <= cnz + 1; ++K)
        for (int J = 1; J <= cny; ++J)
            for (int I = 1; I <= cnx; ++I) {
                int k = 2 * K - 1;
                double sum = 0;
                for (int dj = 0; dj <= 1; ++dj)
                    for (int di = 0; di <= 1; ++di)
                        sum += F->cz[CZI(F, MINI(2 * I - 1 + di, sz1) - 1, MINI(2 * J - 1 + dj, sz2) - 1, MINI(k, sz3) - 1)];
                C->cz[CZI(C, I - 1, J - 1, K - 1)] = sum * 0.25;
            }
#undef MINI
}

static void zero_all(level* L, double* a) {
    memset(a, 0, sizeof(double) * (size_t)(L->nx + 2) * (L->ny + 2) * (L->nz + 2));
}

/* mg_vcycle! (src/Multigrid.jl:706-739) with _solve_coarsest! (:681-685) */
static void vcycle(ocg* s, int lev) {
    level* L = &s->L[lev];
    int sing = s->singular;
    if (lev == s->nlev - 1) {
        rbgs(s, L, s->p.coarse_sweeps);
        if (sing) project_mean(L, L->phi);
        return;
    }
    level* C = &s->L[lev + 1];
    rbgs(s, L, s->p.nu1);
    if (sing) project_mean(L, L->phi);
    residual(s, L);
    restrict_(C, L, sing ? isum(L, L->r) / (double)ncells(L) : 0.0);
    if (sing) project_mean(C, C->b);
    zero_all(C, C->phi);
    vcycle(s, lev + 1);
    prolong_add(s, L, C);
    if (sing) project_mean(L, L->phi);
    rbgs(s, L, s->p.nu2);
    if (sing) project_mean(L, L->phi);
}

/* _load_rhs! (src/Multigrid.jl:766-775) */
static void load_rhs(ocg* s, const double* rhs) {
    level* L = &s->L[0];
    for (int k = 0; k < L->nz; ++k)
        for (int j = 0; j < L->ny; ++j)
            for (int i = 0; i < L->nx; ++i)
                L->b[IX(L, i + 1, j + 1, k + 1)] = rhs[i + (size_t)L->nx * (j + (size_t)L->ny * k)];
    if (s->singular) project_mean(L, L->b);
}

/* _store_solution! (src/Multigrid.jl:789-793) */
static void store_solution(ocg* s, double* out) {
    level* L = &s->L[0];
    double m = s->singular ? isum(L, L->phi) / (double)ncells(L) : 0.0;
    for (int k = 0; k < L->nz; ++k)
        for (int j = 0; j < L->ny; ++j)
            for (int i = 0; i < L->nx; ++i) {
                double v = L->phi[IX(L, i + 1, j + 1, k + 1)] - m;
                L->phi[IX(L, i + 1, j + 1, k + 1)] = v;
                out[i + (size_t)L->nx * (j + (size_t)L->ny * k)] = v;
            }
}

/* _mg_precond! (src/Multigrid.jl:922-932) */
int ocg_precondition(ocg* s, const double* r, double* z) {
    level* L = &s->L[0];
    load_rhs(s, r);
    zero_all(L, L->phi);
    int nc = s->p.mg_cycles > 1 ? s->p.mg_cycles : 1;
    for (int c = 0; c < nc; ++c) vcycle(s, 0);
    store_solution(s, z);
    return 0;
}

/* _apply_fine! (src/Multigrid.jl:911-919) */
int ocg_apply(ocg* s, const double* x, double* out) {
    level* L = &s->L[0];
    for (int k = 0; k < L->nz; ++k)
        for (int j = 0; j < L->ny; ++j)
            for (int i = 0; i < L->nx; ++i)
                L->phi[IX(L, i + 1, j + 1, k + 1)] = x[i + (size_t)L->nx * (j + (size_t)L->ny * k)];
    fill_halo(L, s->p.bc_x, s->p.bc_y, s->p.bc_z);
    for (int k = 0; k < L->nz; ++k)
        for (int j = 0; j < L->ny; ++j)
            for (int i = 0; i < L->nx; ++i)
                out[i + (size_t)L->nx * (j + (size_t)L->ny * k)] = Aphi(L, L->phi, i + 1, j + 1, k + 1);
    return 0;
}

/* canonical sums over an interior-sized array */
static double csum(const ocg* s, const double* a, const double* b) {
    int nx = s->p.nx, ny = s->p.ny, nz = s->p.nz;
    double t = 0;
    for (int k = 0; k < nz; ++k) {
        double pk = 0;
        for (size_t q = (size_t)nx * ny * k; q < (size_t)nx * ny * (k + 1); ++q) pk += b ? a[q] * b[q] : a[q];
        t += pk;
    }
    return t;
}

/* pcg!/_pcg! (src/Backends.jl:1511-1589) with the V-cycle (or identity)
 * preconditioner, zero initial guess, definite = :negative. */
int ocg_solve(ocg* s, const double* b, double* x, ocg_stats* st) {
    size_t n = (size_t)s->p.nx * s->p.ny * s->p.nz;
    double nd = (double)n;
    double *r = s->rr, *z = s->z, *p = s->pp, *Ap = s->Ap;
    int pm = s->singular;
    double mb = pm ? csum(s, b, NULL) / nd : 0.0;
    for (size_t q = 0; q < n; ++q) x[q] = 0.0;
    for (size_t q = 0; q < n; ++q) { r[q] = b[q] - mb; z[q] = s->p.precond == OCG_PC_IDENTITY ? r[q] : 0.0; }
    double b2 = csum(s, r, r);
    double bnorm = sqrt(b2);
    st->bnorm = bnorm;
    st->curvature = NAN;
    if (bnorm == 0) {
        st->iterations = 0; st->residual = 0; st->status = OCG_ZERO_RHS;
        return 0;
    }
    if (s->p.precond == OCG_PC_VCYCLE) ocg_precondition(s, r, z);
    double r2 = csum(s, r, r), rz = csum(s, r, z), Sz = csum(s, z, NULL), Sr = csum(s, r, NULL);
    double m = pm ? Sz / nd : 0.0;
    if (pm) rz -= m * Sr;
    for (size_t q = 0; q < n; ++q) p[q] = z[q] - m;
    double rnorm = sqrt(r2);
    int iters = 0, status = rnorm <= s->p.tol * bnorm ? OCG_CONVERGED : OCG_MAXIT;
    double pAp = NAN;
    while (status != OCG_CONVERGED && iters < s->p.maxit) {
        ocg_apply(s, p, Ap);
        pAp = csum(s, p, Ap);
        if (!(fabs(pAp) > DBL_EPSILON * fabs(rz))) { status = OCG_BREAKDOWN; break; }
        double alpha = rz / pAp;
        iters++;
        for (size_t q = 0; q < n; ++q) {
            x[q] = x[q] + alpha * p[q];
            r[q] = r[q] - alpha * Ap[q];
            if (s->p.precond == OCG_PC_IDENTITY) z[q] = r[q];
        }
        r2 = csum(s, r, r);
        double rzn = csum(s, r, z);
        Sz = csum(s, z, NULL); Sr = csum(s, r, NULL);
        rnorm = sqrt(r2);
        if (rnorm <= s->p.tol * bnorm) { status = OCG_CONVERGED; break; }
        if (s->p.precond == OCG_PC_VCYCLE) {
            ocg_precondition(s, r, z);
            rzn = csum(s, r, z); Sz = csum(s, z, NULL); Sr = csum(s, r, NULL);
        }
        m = pm ? Sz / nd : 0.0;
        if (pm) rzn -= m * Sr;
        double beta = rzn / rz;
        for (size_t q = 0; q < n; ++q) p[q] = (z[q] - m) + beta * p[q];
        rz = rzn;
    }
    if (pm) {
        double mx = csum(s, x, NULL) / nd;
        for (size_t q = 0; q < n; ++q) x[q] = x[q] - mx;
    }
    st->iterations = iters; st->residual = rnorm; st->status = status; st->curvature = pAp;
    return 0;
}

/* mg_solve! (src/Multigrid.jl:801-840), residual norm by _residual_norm! */
int ocg_mg_solve(ocg* s, const double* b, double* x, ocg_stats* st) {
    level* L = &s->L[0];
    load_rhs(s, b);
    zero_all(L, L->phi);
    double bn = sqrt(0.0);
    {
        double t = 0;
        for (int k = 1; k <= L->nz; ++k) {
            double pk = 0;
            for (int j = 1; j <= L->ny; ++j)
                for (int i = 1; i <= L->nx; ++i) pk += L->b[IX(L, i, j, k)] * L->b[IX(L, i, j, k)];
            t += pk;
        }
        bn = sqrt(t);
    }
    st->bnorm = bn; st->curvature = NAN;
    if (bn == 0) {
        memset(x, 0, sizeof(double) * ncells(L));
        st->iterations = 0; st->residual = 0; st->status = OCG_ZERO_RHS;
        return 0;
    }
    double rel = 1.0;
    int ncyc = 0, conv = 0;
    for (int c = 1; c <= s->p.maxit; ++c) {
        vcycle(s, 0);
        residual(s, L);
        double t = 0;
        if (s->singular) {
            double mr = isum(L, L->r) / (double)ncells(L);
            for (int k = 1; k <= L->nz; ++k) {
                double pk = 0;
                for (int j = 1; j <= L->ny; ++j)
                    for (int i = 1; i <= L->nx; ++i) {
                        double v = L->r[IX(L, i, j, k)] - mr;
                        L->r[IX(L, i, j, k)] = v;
                        pk += v * v;
                    }
                t += pk;
            }
        } else {
            for (int k = 1; k <= L->nz; ++k) {
                double pk = 0;
                for (int j = 1; j <= L->ny; ++j)
                    for (int i = 1; i <= L->nx; ++i) pk += L->r[IX(L, i, j, k)] * L->r[IX(L, i, j, k)];
                t += pk;
            }
        }
        rel = sqrt(t) / bn;
        ncyc = c;
        if (rel < s->p.tol) { conv = 1; break; }
    }
    store_solution(s, x);
    st->iterations = ncyc; st->residual = rel; st->status = conv ? OCG_CONVERGED : OCG_MAXIT;
    return 0;
}

static void level_init(level* L, int nx, int ny, int nz, double dx, double dy, double dz, int coeff) {
    L->nx = nx; L->ny = ny; L->nz = nz;
    L->dx = dx; L->dy = dy; L->dz = dz;
    L->ix2 = 1.0 / (dx * dx); L->iy2 = 1.0 / (dy * dy); L->iz2 = 1.0 / (dz * dz);
    size_t ns = (size_t)(nx + 2) * (ny + 2) * (nz + 2);
    L->phi = calloc(ns, sizeof(double));
    L->b = calloc(ns, sizeof(double));
    L->r = calloc(ns, sizeof(double));
    if (coeff) {
        L->cx = calloc((size_t)(nx + 1) * ny * nz, sizeof(double));
        L->cy = calloc((size_t)nx * (ny + 1) * nz, sizeof(double));
        L->cz = calloc((size_t)nx * ny * (nz + 1), sizeof(double));
    } else {
        L->cx = L->cy = L->cz = NULL;
    }
}

/* MultigridPoissonSolver / MGPreconditionedCG constructors
 * (src/Multigrid.jl:551-600, :893-901): full coarsening while every
 * dimension stays even and its half is >= min_size. */
ocg* ocg_create(const ocg_params* p, const double* cx, const double* cy, const double* cz) {
    if (p->nx < 1 || p->ny < 1 || p->nz < 1 || !(p->dx > 0) || !(p->dy > 0) || !(p->dz > 0)) return NULL;
    ocg* s = calloc(1, sizeof(ocg));
    s->p = *p;
    int nx = p->nx, ny = p->ny, nz = p->nz;
    double dx = p->dx, dy = p->dy, dz = p->dz;
    int coeff = cx != NULL;
    level_init(&s->L[0], nx, ny, nz, dx, dy, dz, coeff);
    if (coeff) {
        memcpy(s->L[0].cx, cx, sizeof(double) * (size_t)(nx + 1) * ny * nz);
        memcpy(s->L[0].cy, cy, sizeof(double) * (size_t)nx * (ny + 1) * nz);
        memcpy(s->L[0].cz, cz, sizeof(double) * (size_t)nx * ny * (nz + 1));
    }
    s->nlev = 1;
    while (s->nlev < 24) {
        int cxo = nx % 2 == 0 && nx / 2 >= p->min_size;
        int cyo = ny % 2 == 0 && ny / 2 >= p->min_size;
        int czo = nz % 2 == 0 && nz / 2 >= p->min_size;
        if (!(cxo && cyo && czo)) break;
        nx /= 2; ny /= 2; nz /= 2;
        dx *= 2; dy *= 2; dz *= 2;
        level_init(&s->L[s->nlev], nx, ny, nz, dx, dy, dz, coeff);
        if (coeff) restrict_coeff(&s->L[s->nlev - 1], &s->L[s->nlev]);
        s->nlev++;
    }
    s->singular = (p->bc_x == OCG_BC_PERIODIC || p->bc_x == OCG_BC_NEUMANN) &&
                  (p->bc_y == OCG_BC_PERIODIC || p->bc_y == OCG_BC_NEUMANN) &&
                  (p->bc_z == OCG_BC_PERIODIC || p->bc_z == OCG_BC_NEUMANN);
    size_t n = (size_t)p->nx * p->ny * p->nz;
    s->x = calloc(n, sizeof(double));
    s->rr = calloc(n, sizeof(double));
    s->z = calloc(n, sizeof(double));
    s->pp = calloc(n, sizeof(double));
    s->Ap = calloc(n, sizeof(double));
    s->bb = calloc(n, sizeof(double));
    return s;
}

void ocg_destroy(ocg* s) {
    if (!s) return;
    for (int l = 0; l < s->nlev; ++l) {
        free(s->L[l].phi); free(s->L[l].b); free(s->L[l].r);
        free(s->L[l].cx); free(s->L[l].cy); free(s->L[l].cz);
    }
    free(s->x); free(s->rr); free(s->z); free(s->pp); free(s->Ap); free(s->bb);
    free(s);
}

int ocg_nlevels(const ocg* s) { return s->nlev; }

int ocg_level_dims(const ocg* s, int lev, int32_t dims[3]) {
    if (lev < 0 || lev >= s->nlev) return 1;
    dims[0] = s->L[lev].nx; dims[1] = s->L[lev].ny; dims[2] = s->L[lev].nz;
    return 0;
}

int ocg_level_coeff(const ocg* s, int lev, double* cx, double* cy, double* cz) {
    if (lev < 0 || lev >= s->nlev || !s->L[lev].cx) return 1;
    const level* L = &s->L[lev];
    memcpy(cx, L->cx, sizeof(double) * (size_t)(L->nx + 1) * L->ny * L->nz);
    memcpy(cy, L->cy, sizeof(double) * (size_t)L->nx * (L->ny + 1) * L->nz);
    memcpy(cz, L->cz, sizeof(double) * (size_t)L->nx * L->ny * (L->nz + 1));
    return 0;
}
