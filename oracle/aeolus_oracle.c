/*
 * aeolus_oracle.c -- TEST INFRASTRUCTURE ONLY (the oracle).
 *
 * A CPU FP64 restatement of the Aeolus.jl dynamical-core time step, used as
 * the checker for the CUDA library and as the timed CPU baseline.  The
 * product path never links or calls this file.  Every function names the
 * reference lines (path:line inside the Aeolus.jl project) it restates; the
 * arithmetic follows the reference's expression order so that the oracle
 * differs from the reference by round-off only.
 *
 * Parity pins: the reference is Julia (not installable here), so the oracle
 * is pinned by the reference's own known-answer and analytic tests restated
 * in tests/ (Philox4x32-10 KATs of test/backends.jl:265-276, the discrete
 * Poisson identities of test/runtests.jl:168-260 and
 * test/pressure_column.jl:13-117, the projection's round-off divergence,
 * WENO design order of test/advection.jl:52-188, the TGV modified-wavenumber
 * decay of test/ka_step.jl:138-147).
 *
 * Build: oracle/Makefile (gcc -O2 -fopenmp -ffp-contract=off; no fast-math,
 * no FMA contraction, so that each operation rounds as Julia's does).
 */
#include "aeolus_oracle.h"
#include "mgpcg_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define LOC_C 0
#define LOC_FX 1
#define LOC_FY 2
#define LOC_FZ 3

typedef struct { double re, im; } cpx;

typedef struct {
    int n;          /* transform length */
    int pow2;       /* 1 when n is a power of two */
    cpx* tw;        /* e^{-2 pi i k / n}, k < n */
    int* rev;       /* bit reversal (pow2 only) */
} fft_plan;

struct oc_sim {
    oc_params p;
    int NX, NY, NZ;
    int64_t n;                   /* storage points */
    /* metrics (src/FiniteVolume.jl:71-186, src/StretchedGrids.jl:560-590) */
    int uniform;
    double dx, dy, dz, idx, idy, idx2, idy2, idz, idz2, delta_u;
    double *zf, *zc, *dzc, *dzf;                  /* storage levels */
    double *idzc, *idzf, *idz_off, *wlo, *whi, *alo, *ahi, *delta;
    /* anelastic weights (padded) */
    double *wc, *wf, *thf;
    /* fields (storage layout) */
    double *u, *v, *w, *th, *pr, *nut, *kt, *phi;
    double *tu, *tv, *tw, *tt;
    double *u0, *v0, *w0, *th0;
    /* pressure solver */
    double* src;                 /* interior-sized */
    cpx* hat;                    /* (Nx/2+1) x Ny x Nz */
    double *kx2, *ky2, *kz2;     /* eigenvalue pieces */
    double *lower, *upper, *hw, *meas, *iota, *gauge;
    double meas_sum, gauge_sum;
    fft_plan px, py, pz;         /* px: length Nx/2 (the packed r2c) */
    cpx* twx;                    /* e^{-2 pi i k / Nx}, k <= Nx/2 */
    /* the implicit IBM correction: solid cells (interior, x fastest) and tau */
    unsigned char* ibm;
    double ibm_tau;
    /* solver = PCG: face apertures (interior face layout), the CG of the a^2 operator */
    double *apx, *apy, *apz, *cgx;
    ocg* cg;
    ocg_stats cg_st;
    /* dynamic Smagorinsky: the ten pass-1 fields on the interior + one shell,
     * LM and MM (interior), the per-level coefficient */
    double* dyn[10];
    double *dyn_lm, *dyn_mm, *cs2;
    double* amd_bg;   /* g/theta_bar(z_k) of the sound-proof core's AMD closure (interior levels), or NULL */
    /* the Lagrangian closure: the memories I_LM, I_MM and the cell-centred
     * velocity of the memory (interior, x fastest), the coefficient of the
     * committed memory, the scratch of the relaxation, its parameters */
    double *lag_ilm, *lag_imm, *lag_up, *lag_vp, *lag_wp, *lag_cs2, *lag_nlm, *lag_nmm;
    int lag_init;
    double lag_c0, lag_theta, lag_mt;
    /* the TKE closure: e, 2 nu_t and the transport tendency (storage
     * arrays), the new e (interior), the coefficients */
    double *tke_e, *tke_k2, *tke_tend, *tke_new;
    double tke_ce0, tke_ce1, tke_cl;
    int tke_exact;
    /* open lateral faces: the plane buffers (x: [f][side][NZ][NY][L], y:
     * [f][side][NZ][L][NX], f = u, v, w, theta), the per-field modes */
    int open_x, open_y, oL;
    double *oxp, *oyp;
    int omode[4];
    double cg_tol;
    int cg_maxit;
    /* radiating outflow (:convective) of the open faces: per side (west, east,
     * south, north) the flag; the raw data planes, the step-start snapshot and
     * the stage-start buffers (the layout of oxp / oyp); the phase speeds and
     * the stage-start interior layers per plane point ([f][side][NZ][NY or NX]);
     * the correction mode (0 uniform, 1 outflow only, 2 none) and its ledger */
    int orad[4], ocorr, omarked;
    double *oxf, *oyf;            /* weights of the normal planes' boundary faces (0 solid) */
    double *oxh, *oyh;            /* :orlanski history: the interior layer at the previous step start */
    int ohist;
    double olast_dt;
    double *oxd, *oyd, *oxs, *oys, *oxv, *oyv;
    double *oxc, *oyc, *ox1, *oy1, *ox2, *oy2;
    double oQ, odelta, oresid;
};

/* the radiating outflow of open faces (defined with oc_set_open) */
static int ob_radiates(const oc_sim* s);
static void ob_prepare(oc_sim* s, double dt);
static void ob_mark(oc_sim* s);
static void ob_update(oc_sim* s, double dt);
static void ob_combine(oc_sim* s, double a, double b);

#define ID(s, i, j, k) ((int64_t)(i) + (int64_t)(s)->NX * ((int64_t)(j) + (int64_t)(s)->NY * (int64_t)(k)))
#define A(f, i, j, k) (f)[ID(s, i, j, k)]

/* ------------------------------------------------------------------------- */
/* Philox4x32-10 (src/Backends.jl:1607-1640) and the uniform fill            */
/* ------------------------------------------------------------------------- */

void oc_philox4x32(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    uint32_t k0 = key[0], k1 = key[1];
    for (int r = 1; r <= 10; ++r) {
        uint64_t p0 = (uint64_t)0xD2511F53u * (uint64_t)c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * (uint64_t)c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ c1 ^ k0, n1 = lo1, n2 = hi0 ^ c3 ^ k1, n3 = lo0;
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
        if (r < 10) { k0 += 0x9E3779B9u; k1 += 0xBB67AE85u; }
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

/* The first 64-bit draw of the counter stream (seed, stream, id)
 * (src/Backends.jl:1707-1739: key = (seed>>32, seed), counter =
 * (block 0, stream, id lo, id hi), draw = x1<<32 | x0) mapped to [0,1) by
 * its top 53 bits, then to [-amp, amp]. */
static double philox_uniform(uint64_t seed, uint32_t stream, uint64_t id) {
    uint32_t key[2] = {(uint32_t)(seed >> 32), (uint32_t)seed};
    uint32_t ctr[4] = {0u, stream, (uint32_t)id, (uint32_t)(id >> 32)};
    uint32_t o[4];
    oc_philox4x32(ctr, key, o);
    uint64_t x = ((uint64_t)o[1] << 32) | (uint64_t)o[0];
    return (double)(x >> 11) * 0x1.0p-53;
}

void oc_uniform_fill(uint64_t seed, uint32_t stream, int64_t n, double amp, double* out) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) out[i] = amp * (2.0 * philox_uniform(seed, stream, (uint64_t)i) - 1.0);
}

void oc_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

/* ------------------------------------------------------------------------- */
/* FFT: own radix-2 (power of two) or direct DFT (other lengths)             */
/* ------------------------------------------------------------------------- */

static void plan_init(fft_plan* pl, int n) {
    pl->n = n;
    pl->pow2 = (n > 0) && ((n & (n - 1)) == 0);
    pl->tw = (cpx*)malloc(sizeof(cpx) * (size_t)(n > 0 ? n : 1));
    for (int k = 0; k < n; ++k) {
        double a = -2.0 * M_PI * (double)k / (double)n;
        pl->tw[k].re = cos(a);
        pl->tw[k].im = sin(a);
    }
    pl->rev = NULL;
    if (pl->pow2) {
        pl->rev = (int*)malloc(sizeof(int) * (size_t)n);
        int lg = 0;
        while ((1 << lg) < n) ++lg;
        for (int i = 0; i < n; ++i) {
            int r = 0;
            for (int b = 0; b < lg; ++b) if (i & (1 << b)) r |= 1 << (lg - 1 - b);
            pl->rev[i] = r;
        }
    }
}

static void plan_free(fft_plan* pl) { free(pl->tw); free(pl->rev); }

/* In-place unnormalised DFT of a (length pl->n); sign -1 forward, +1 inverse.
 * tmp: scratch of length n. */
static void fft_c(const fft_plan* pl, cpx* a, int inverse, cpx* tmp) {
    int n = pl->n;
    if (n <= 1) return;
    if (!pl->pow2) {
        for (int k = 0; k < n; ++k) {
            double sr = 0.0, si = 0.0;
            for (int j = 0; j < n; ++j) {
                int m = (int)(((int64_t)j * k) % n);
                double wr = pl->tw[m].re, wi = inverse ? -pl->tw[m].im : pl->tw[m].im;
                sr += a[j].re * wr - a[j].im * wi;
                si += a[j].re * wi + a[j].im * wr;
            }
            tmp[k].re = sr; tmp[k].im = si;
        }
        memcpy(a, tmp, sizeof(cpx) * (size_t)n);
        return;
    }
    for (int i = 0; i < n; ++i) {
        int r = pl->rev[i];
        if (r > i) { cpx t = a[i]; a[i] = a[r]; a[r] = t; }
    }
    for (int len = 2; len <= n; len <<= 1) {
        int half = len >> 1, step = n / len;
        for (int b = 0; b < n; b += len) {
            for (int j = 0; j < half; ++j) {
                cpx wv = pl->tw[j * step];
                if (inverse) wv.im = -wv.im;
                cpx x = a[b + j], y = a[b + j + half];
                cpx t = {y.re * wv.re - y.im * wv.im, y.re * wv.im + y.im * wv.re};
                a[b + j].re = x.re + t.re; a[b + j].im = x.im + t.im;
                a[b + j + half].re = x.re - t.re; a[b + j + half].im = x.im - t.im;
            }
        }
    }
}

/* Real-to-complex forward DFT of x (length N = 2M) to X[0..M], by the
 * packed length-M complex transform. z: scratch M+1, tmp: scratch M. */
static void rfft_row(const oc_sim* s, const double* x, cpx* X, cpx* z, cpx* tmp) {
    int N = s->p.nx, M = N / 2;
    for (int n = 0; n < M; ++n) { z[n].re = x[2 * n]; z[n].im = x[2 * n + 1]; }
    fft_c(&s->px, z, 0, tmp);
    z[M] = z[0];
    for (int k = 0; k <= M; ++k) {
        cpx a = z[k], b = z[M - k];
        double er = 0.5 * (a.re + b.re), ei = 0.5 * (a.im - b.im);
        double orr = 0.5 * (a.im + b.im), oi = -0.5 * (a.re - b.re);
        cpx w = s->twx[k];
        X[k].re = er + (w.re * orr - w.im * oi);
        X[k].im = ei + (w.re * oi + w.im * orr);
    }
}

/* Unnormalised complex-to-real inverse (FFTW brfft): x[n] = sum over the
 * Hermitian spectrum of X[k] e^{+2 pi i k n / N}. */
static void irfft_row(const oc_sim* s, const cpx* X, double* x, cpx* z, cpx* tmp) {
    int N = s->p.nx, M = N / 2;
    for (int k = 0; k < M; ++k) {
        cpx a = X[k], b = X[M - k];
        double er = a.re + b.re, ei = a.im - b.im;          /* X_k + conj X_{M-k} */
        double dr = a.re - b.re, di = a.im + b.im;          /* X_k - conj X_{M-k} */
        cpx w = s->twx[k];                                  /* multiply by conj(w) */
        double orr = dr * w.re + di * w.im, oi = di * w.re - dr * w.im;
        z[k].re = er - oi;                                  /* E + i O */
        z[k].im = ei + orr;
    }
    fft_c(&s->px, z, 1, tmp);
    for (int n = 0; n < M; ++n) { x[2 * n] = z[n].re; x[2 * n + 1] = z[n].im; }
}

/* ------------------------------------------------------------------------- */
/* Metric accessors (src/FiniteVolume.jl:146-186)                             */
/* ------------------------------------------------------------------------- */

static inline double m_idz(const oc_sim* s, int k) { return s->uniform ? s->idz : s->idzc[k]; }
static inline double m_idzf(const oc_sim* s, int k) { return s->uniform ? s->idz : s->idzf[k]; }
static inline double m_idz_off(const oc_sim* s, int k) { return s->uniform ? s->idz : s->idz_off[k]; }
static inline double m_zface(const oc_sim* s, int k, double lo, double hi) {
    return s->uniform ? 0.5 * (lo + hi) : s->wlo[k] * lo + s->whi[k] * hi;
}
static inline double m_zflux(const oc_sim* s, int k, double lo, double hi) {
    return s->uniform ? 0.5 * (lo + hi) : s->alo[k] * lo + s->ahi[k] * hi;
}
static inline double m_lapz(const oc_sim* s, int loc, int k, double fm, double c, double fp) {
    if (s->uniform) return (fp - 2 * c + fm) * s->idz2;
    if (loc == LOC_FZ) return ((fp - c) * s->idzc[k] - (c - fm) * s->idzc[k - 1]) * s->idzf[k];
    return ((fp - c) * s->idzf[k + 1] - (c - fm) * s->idzf[k]) * s->idzc[k];
}
static inline double m_filter(const oc_sim* s, int k) { return s->uniform ? s->delta_u : s->delta[k]; }

/* ------------------------------------------------------------------------- */
/* Halo fills (src/boundary_conditions/halo_kernels.jl:100-140,               */
/* src/BoundaryConditions.jl:228-258): x, then y, then z.                     */
/* ------------------------------------------------------------------------- */

/* The plane of field d on the open faces (u, v, w, theta with mode 0), or -1:
 * the mirror (_plane_name / _fill_open_face!,
 * src/boundary_conditions/open_boundary.jl:726-772). */
static int open_pid(const oc_sim* s, const double* d) {
    int f = d == s->u ? 0 : d == s->v ? 1 : d == s->w ? 2 : d == s->th ? 3 : -1;
    return f >= 0 && s->omode[f] == 0 ? f : -1;
}

static void fill_halos(oc_sim* s, double* d, int loc) {
    int NX = s->NX, NY = s->NY, NZ = s->NZ;
    int Hx = s->p.hx, Hy = s->p.hy, Hz = s->p.hz, Nx = s->p.nx, Ny = s->p.ny, Nz = s->p.nz;
    int pid = open_pid(s, d), L = s->oL;
    if (s->open_x) {
        /* x: open faces (_fill_x!, :781-785): the plane's slab -- with the
         * boundary face of u on the west (interior 0) -- or the mirror */
        int nw = pid == 0 ? Hx + 1 : Hx;
#pragma omp parallel for collapse(2) schedule(static)
        for (int k = 0; k < NZ; ++k)
            for (int j = 0; j < NY; ++j) {
                if (pid >= 0) {
                    const double* pw = s->oxp + (((int64_t)(pid * 2 + 0) * NZ + k) * NY + j) * L;
                    const double* pe = s->oxp + (((int64_t)(pid * 2 + 1) * NZ + k) * NY + j) * L;
                    for (int l = 0; l < nw; ++l) A(d, l, j, k) = pw[l];
                    for (int l = 0; l < Hx; ++l) A(d, Hx + Nx + l, j, k) = pe[l];
                } else {
                    for (int h = 1; h <= Hx; ++h) {
                        A(d, Hx - h, j, k) = A(d, Hx + h - 1, j, k);
                        A(d, Hx + Nx + h - 1, j, k) = A(d, Hx + Nx - h, j, k);
                    }
                }
            }
    } else {
    /* x: periodic */
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < NZ; ++k)
        for (int j = 0; j < NY; ++j)
            for (int h = 1; h <= Hx; ++h) {
                A(d, h - 1, j, k) = A(d, Nx + h - 1, j, k);
                A(d, Hx + Nx + h - 1, j, k) = A(d, Hx + h - 1, j, k);
            }
    }
    if (s->open_y) {
        int ns = pid == 1 ? Hy + 1 : Hy;
#pragma omp parallel for collapse(2) schedule(static)
        for (int k = 0; k < NZ; ++k)
            for (int i = 0; i < NX; ++i) {
                if (pid >= 0) {
                    for (int l = 0; l < ns; ++l)
                        A(d, i, l, k) = s->oyp[(((int64_t)(pid * 2 + 0) * NZ + k) * L + l) * NX + i];
                    for (int l = 0; l < Hy; ++l)
                        A(d, i, Hy + Ny + l, k) = s->oyp[(((int64_t)(pid * 2 + 1) * NZ + k) * L + l) * NX + i];
                } else {
                    for (int h = 1; h <= Hy; ++h) {
                        A(d, i, Hy - h, k) = A(d, i, Hy + h - 1, k);
                        A(d, i, Hy + Ny + h - 1, k) = A(d, i, Hy + Ny - h, k);
                    }
                }
            }
    } else {
    /* y: periodic */
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < NZ; ++k)
        for (int h = 1; h <= Hy; ++h)
            for (int i = 0; i < NX; ++i) {
                A(d, i, h - 1, k) = A(d, i, Ny + h - 1, k);
                A(d, i, Hy + Ny + h - 1, k) = A(d, i, Hy + h - 1, k);
            }
    }
    /* z */
    if (s->p.bc_z == OC_BC_PERIODIC) {
#pragma omp parallel for schedule(static)
        for (int j = 0; j < NY; ++j)
            for (int h = 1; h <= Hz; ++h)
                for (int i = 0; i < NX; ++i) {
                    A(d, i, j, h - 1) = A(d, i, j, Nz + h - 1);
                    A(d, i, j, Hz + Nz + h - 1) = A(d, i, j, Hz + h - 1);
                }
    } else if (loc != LOC_FZ) {
        /* ImpermeableWall on C / FaceX / FaceY: mirror (NoFlux) */
#pragma omp parallel for schedule(static)
        for (int j = 0; j < NY; ++j)
            for (int h = 1; h <= Hz; ++h)
                for (int i = 0; i < NX; ++i) {
                    A(d, i, j, Hz - h) = A(d, i, j, Hz + h - 1);
                    A(d, i, j, Hz + Nz + h - 1) = A(d, i, j, Hz + Nz - h);
                }
    } else {
        /* ImpermeableWall on FaceZ: wall faces zero, odd extension */
#pragma omp parallel for schedule(static)
        for (int j = 0; j < NY; ++j) {
            for (int i = 0; i < NX; ++i) {
                A(d, i, j, Hz) = 0.0;
                if (Hz + Nz < NZ) A(d, i, j, Hz + Nz) = 0.0;
            }
            for (int h = 1; h <= Hz; ++h)
                for (int i = 0; i < NX; ++i) {
                    A(d, i, j, Hz - h) = -A(d, i, j, Hz + h);
                    int dst = Hz + Nz + h;
                    if (dst < NZ) A(d, i, j, dst) = -A(d, i, j, Hz + Nz - h);
                }
        }
    }
}

void oc_fill_state_halos(oc_sim* s) {
    fill_halos(s, s->u, LOC_FX);
    fill_halos(s, s->v, LOC_FY);
    fill_halos(s, s->w, LOC_FZ);
    fill_halos(s, s->th, LOC_C);
}

/* ------------------------------------------------------------------------- */
/* Point operators                                                            */
/* ------------------------------------------------------------------------- */

/* seven-point Laplacian (src/FiniteVolume.jl:271-280) */
static inline double lap_at(const oc_sim* s, const double* f, int i, int j, int k, int loc) {
    double c = A(f, i, j, k);
    return (A(f, i + 1, j, k) - 2 * c + A(f, i - 1, j, k)) * s->idx2 +
           (A(f, i, j + 1, k) - 2 * c + A(f, i, j - 1, k)) * s->idy2 +
           m_lapz(s, loc, k, A(f, i, j, k - 1), c, A(f, i, j, k + 1));
}

/* centred flux-form momentum advection (src/FiniteVolume.jl:730-797) */
static inline double mom_u_at(const oc_sim* s, const double* u, const double* v, const double* w, int i, int j, int k) {
    double uce = 0.5 * (A(u, i, j, k) + A(u, i + 1, j, k));
    double ucw = 0.5 * (A(u, i - 1, j, k) + A(u, i, j, k));
    double d_uu_dx = (uce * uce - ucw * ucw) * s->idx;
    double vun = 0.5 * (A(v, i - 1, j + 1, k) + A(v, i, j + 1, k));
    double uvn = 0.5 * (A(u, i, j, k) + A(u, i, j + 1, k));
    double vus = 0.5 * (A(v, i - 1, j, k) + A(v, i, j, k));
    double uvs = 0.5 * (A(u, i, j - 1, k) + A(u, i, j, k));
    double d_vu_dy = (vun * uvn - vus * uvs) * s->idy;
    double wut = 0.5 * (A(w, i - 1, j, k + 1) + A(w, i, j, k + 1));
    double uwt = 0.5 * (A(u, i, j, k) + A(u, i, j, k + 1));
    double wub = 0.5 * (A(w, i - 1, j, k) + A(w, i, j, k));
    double uwb = 0.5 * (A(u, i, j, k - 1) + A(u, i, j, k));
    double d_wu_dz = (wut * uwt - wub * uwb) * m_idz(s, k);
    return d_uu_dx + d_vu_dy + d_wu_dz;
}

static inline double mom_v_at(const oc_sim* s, const double* u, const double* v, const double* w, int i, int j, int k) {
    double uve = 0.5 * (A(u, i + 1, j - 1, k) + A(u, i + 1, j, k));
    double vue = 0.5 * (A(v, i, j, k) + A(v, i + 1, j, k));
    double uvw = 0.5 * (A(u, i, j - 1, k) + A(u, i, j, k));
    double vuw = 0.5 * (A(v, i - 1, j, k) + A(v, i, j, k));
    double d_uv_dx = (uve * vue - uvw * vuw) * s->idx;
    double vcn = 0.5 * (A(v, i, j, k) + A(v, i, j + 1, k));
    double vcs = 0.5 * (A(v, i, j - 1, k) + A(v, i, j, k));
    double d_vv_dy = (vcn * vcn - vcs * vcs) * s->idy;
    double wvt = 0.5 * (A(w, i, j - 1, k + 1) + A(w, i, j, k + 1));
    double vwt = 0.5 * (A(v, i, j, k) + A(v, i, j, k + 1));
    double wvb = 0.5 * (A(w, i, j - 1, k) + A(w, i, j, k));
    double vwb = 0.5 * (A(v, i, j, k - 1) + A(v, i, j, k));
    double d_wv_dz = (wvt * vwt - wvb * vwb) * m_idz(s, k);
    return d_uv_dx + d_vv_dy + d_wv_dz;
}

static inline double mom_w_at(const oc_sim* s, const double* u, const double* v, const double* w, int i, int j, int k) {
    double uwe = m_zflux(s, k, A(u, i + 1, j, k - 1), A(u, i + 1, j, k));
    double wue = 0.5 * (A(w, i, j, k) + A(w, i + 1, j, k));
    double uww = m_zflux(s, k, A(u, i, j, k - 1), A(u, i, j, k));
    double wuw = 0.5 * (A(w, i - 1, j, k) + A(w, i, j, k));
    double d_uw_dx = (uwe * wue - uww * wuw) * s->idx;
    double vwn = m_zflux(s, k, A(v, i, j + 1, k - 1), A(v, i, j + 1, k));
    double wvn = 0.5 * (A(w, i, j, k) + A(w, i, j + 1, k));
    double vws = m_zflux(s, k, A(v, i, j, k - 1), A(v, i, j, k));
    double wvs = 0.5 * (A(w, i, j - 1, k) + A(w, i, j, k));
    double d_vw_dy = (vwn * wvn - vws * wvs) * s->idy;
    double wct = 0.5 * (A(w, i, j, k) + A(w, i, j, k + 1));
    double wcb = 0.5 * (A(w, i, j, k - 1) + A(w, i, j, k));
    double d_ww_dz = (wct * wct - wcb * wcb) * m_idzf(s, k);
    return d_uw_dx + d_vw_dy + d_ww_dz;
}

/* centred flux-form scalar advection (src/FiniteVolume.jl:1682-1693) */
static inline double adv_centred_at(const oc_sim* s, const double* u, const double* v, const double* w,
                                    const double* d, int i, int j, int k) {
    double ue = A(u, i + 1, j, k) * 0.5 * (A(d, i, j, k) + A(d, i + 1, j, k));
    double uw = A(u, i, j, k) * 0.5 * (A(d, i - 1, j, k) + A(d, i, j, k));
    double vn = A(v, i, j + 1, k) * 0.5 * (A(d, i, j, k) + A(d, i, j + 1, k));
    double vs = A(v, i, j, k) * 0.5 * (A(d, i, j - 1, k) + A(d, i, j, k));
    double wt = A(w, i, j, k + 1) * 0.5 * (A(d, i, j, k) + A(d, i, j, k + 1));
    double wb = A(w, i, j, k) * 0.5 * (A(d, i, j, k - 1) + A(d, i, j, k));
    return (ue - uw) * s->idx + (vn - vs) * s->idy + (wt - wb) * m_idz(s, k);
}

/* W-weighted centred momentum / scalar advection (src/Anelastic.jl:1193-1306);
 * on a stretched column the vertical metrics and the side-face volume flux of
 * a w control volume (_zflux) replace the uniform ones -- on a uniform grid
 * these are the reference expressions bit for bit. */
static inline double wmom_u(const oc_sim* s, const double* u, const double* v, const double* w, int i, int j, int k) {
    double iwc = 1 / s->wc[k], wfb = s->wf[k], wft = s->wf[k + 1];
    double uce = 0.5 * (A(u, i, j, k) + A(u, i + 1, j, k));
    double ucw = 0.5 * (A(u, i - 1, j, k) + A(u, i, j, k));
    double d_uu_dx = (uce * uce - ucw * ucw) * s->idx;
    double vun = 0.5 * (A(v, i - 1, j + 1, k) + A(v, i, j + 1, k));
    double uvn = 0.5 * (A(u, i, j, k) + A(u, i, j + 1, k));
    double vus = 0.5 * (A(v, i - 1, j, k) + A(v, i, j, k));
    double uvs = 0.5 * (A(u, i, j - 1, k) + A(u, i, j, k));
    double d_vu_dy = (vun * uvn - vus * uvs) * s->idy;
    double wut = 0.5 * (A(w, i - 1, j, k + 1) + A(w, i, j, k + 1));
    double uwt = 0.5 * (A(u, i, j, k) + A(u, i, j, k + 1));
    double wub = 0.5 * (A(w, i - 1, j, k) + A(w, i, j, k));
    double uwb = 0.5 * (A(u, i, j, k - 1) + A(u, i, j, k));
    double d_wu_dz = (wft * wut * uwt - wfb * wub * uwb) * m_idz(s, k) * iwc;
    return d_uu_dx + d_vu_dy + d_wu_dz;
}

static inline double wmom_v(const oc_sim* s, const double* u, const double* v, const double* w, int i, int j, int k) {
    double iwc = 1 / s->wc[k], wfb = s->wf[k], wft = s->wf[k + 1];
    double uve = 0.5 * (A(u, i + 1, j - 1, k) + A(u, i + 1, j, k));
    double vue = 0.5 * (A(v, i, j, k) + A(v, i + 1, j, k));
    double uvw = 0.5 * (A(u, i, j - 1, k) + A(u, i, j, k));
    double vuw = 0.5 * (A(v, i - 1, j, k) + A(v, i, j, k));
    double d_uv_dx = (uve * vue - uvw * vuw) * s->idx;
    double vcn = 0.5 * (A(v, i, j, k) + A(v, i, j + 1, k));
    double vcs = 0.5 * (A(v, i, j - 1, k) + A(v, i, j, k));
    double d_vv_dy = (vcn * vcn - vcs * vcs) * s->idy;
    double wvt = 0.5 * (A(w, i, j - 1, k + 1) + A(w, i, j, k + 1));
    double vwt = 0.5 * (A(v, i, j, k) + A(v, i, j, k + 1));
    double wvb = 0.5 * (A(w, i, j - 1, k) + A(w, i, j, k));
    double vwb = 0.5 * (A(v, i, j, k - 1) + A(v, i, j, k));
    double d_wv_dz = (wft * wvt * vwt - wfb * wvb * vwb) * m_idz(s, k) * iwc;
    return d_uv_dx + d_vv_dy + d_wv_dz;
}

static inline double wmom_w(const oc_sim* s, const double* u, const double* v, const double* w, int i, int j, int k) {
    double iwf = 1 / s->wf[k], wcb = s->wc[k - 1], wct = s->wc[k];
    double uwe = m_zflux(s, k, A(u, i + 1, j, k - 1), A(u, i + 1, j, k));
    double wue = 0.5 * (A(w, i, j, k) + A(w, i + 1, j, k));
    double uww = m_zflux(s, k, A(u, i, j, k - 1), A(u, i, j, k));
    double wuw = 0.5 * (A(w, i - 1, j, k) + A(w, i, j, k));
    double d_uw_dx = (uwe * wue - uww * wuw) * s->idx;
    double vwn = m_zflux(s, k, A(v, i, j + 1, k - 1), A(v, i, j + 1, k));
    double wvn = 0.5 * (A(w, i, j, k) + A(w, i, j + 1, k));
    double vws = m_zflux(s, k, A(v, i, j, k - 1), A(v, i, j, k));
    double wvs = 0.5 * (A(w, i, j - 1, k) + A(w, i, j, k));
    double d_vw_dy = (vwn * wvn - vws * wvs) * s->idy;
    double wtop = 0.5 * (A(w, i, j, k) + A(w, i, j, k + 1));
    double wbot = 0.5 * (A(w, i, j, k - 1) + A(w, i, j, k));
    double d_ww_dz = (wct * wtop * wtop - wcb * wbot * wbot) * m_idzf(s, k) * iwf;
    return d_uw_dx + d_vw_dy + d_ww_dz;
}

static inline double wscal(const oc_sim* s, const double* u, const double* v, const double* w, const double* f,
                           int i, int j, int k) {
    double iwc = 1 / s->wc[k], wfb = s->wf[k], wft = s->wf[k + 1];
    double ue = A(u, i + 1, j, k) * 0.5 * (A(f, i, j, k) + A(f, i + 1, j, k));
    double uw = A(u, i, j, k) * 0.5 * (A(f, i - 1, j, k) + A(f, i, j, k));
    double vn = A(v, i, j + 1, k) * 0.5 * (A(f, i, j, k) + A(f, i, j + 1, k));
    double vs = A(v, i, j, k) * 0.5 * (A(f, i, j - 1, k) + A(f, i, j, k));
    double wt = wft * A(w, i, j, k + 1) * 0.5 * (A(f, i, j, k) + A(f, i, j, k + 1));
    double wb = wfb * A(w, i, j, k) * 0.5 * (A(f, i, j, k - 1) + A(f, i, j, k));
    return (ue - uw) * s->idx + (vn - vs) * s->idy + (wt - wb) * m_idz(s, k) * iwc;
}

/* --- WENO reconstructions (src/AdvectionSchemes.jl:105-120, :240-255,
 *     :319-333) ------------------------------------------------------------ */

static inline double beta3(double a1, double a2) { return a1 * a1 + (13.0 / 3.0) * (a2 * a2); }
static inline double b3_m2(double v1, double v2, double v3) {
    return beta3((v1 - 4 * v2 + 3 * v3) / 2, (v1 - 2 * v2 + v3) / 2);
}
static inline double b3_m1(double v1, double v2, double v3) {
    return beta3((v3 - v1) / 2, (v1 - 2 * v2 + v3) / 2);
}
static inline double b3_p0(double v1, double v2, double v3) {
    return beta3((-3 * v1 + 4 * v2 - v3) / 2, (v1 - 2 * v2 + v3) / 2);
}

static inline double weno_js5_left(double v1, double v2, double v3, double v4, double v5) {
    double q0 = (2 * v1 - 7 * v2 + 11 * v3) / 6;
    double q1 = (-v2 + 5 * v3 + 2 * v4) / 6;
    double q2 = (2 * v3 + 5 * v4 - v5) / 6;
    double b0 = b3_m2(v1, v2, v3), b1 = b3_m1(v2, v3, v4), b2 = b3_p0(v3, v4, v5);
    double e = 1e-6;
    double a0 = (1.0 / 10) / ((b0 + e) * (b0 + e));
    double a1 = (6.0 / 10) / ((b1 + e) * (b1 + e));
    double a2 = (3.0 / 10) / ((b2 + e) * (b2 + e));
    return (a0 * q0 + a1 * q1 + a2 * q2) / (a0 + a1 + a2);
}

static inline double weno_z5_left(double v1, double v2, double v3, double v4, double v5) {
    double q0 = (2 * v1 - 7 * v2 + 11 * v3) / 6;
    double q1 = (-v2 + 5 * v3 + 2 * v4) / 6;
    double q2 = (2 * v3 + 5 * v4 - v5) / 6;
    double b0 = b3_m2(v1, v2, v3), b1 = b3_m1(v2, v3, v4), b2 = b3_p0(v3, v4, v5);
    double eps = DBL_EPSILON * DBL_EPSILON;
    double tau = fabs(b0 - b2);
    double t0 = tau / (b0 + eps), t1 = tau / (b1 + eps), t2 = tau / (b2 + eps);
    double a0 = (1.0 / 10) * (1.0 + t0 * t0);
    double a1 = (6.0 / 10) * (1.0 + t1 * t1);
    double a2 = (3.0 / 10) * (1.0 + t2 * t2);
    return (a0 * q0 + a1 * q1 + a2 * q2) / (a0 + a1 + a2);
}

static inline double recon(int scheme, double v1, double v2, double v3, double v4, double v5) {
    return scheme == OC_ADV_WENO_Z5 ? weno_z5_left(v1, v2, v3, v4, v5) : weno_js5_left(v1, v2, v3, v4, v5);
}

/* upwinded face values between cells c and c+1 along each axis
 * (src/AdvectionSchemes.jl:623-666: mirror-symmetric selection) */
static inline double face_x(const oc_sim* s, int sc, const double* d, int c, int j, int k, double vel) {
    if (vel >= 0) return recon(sc, A(d, c - 2, j, k), A(d, c - 1, j, k), A(d, c, j, k), A(d, c + 1, j, k), A(d, c + 2, j, k));
    return recon(sc, A(d, c + 3, j, k), A(d, c + 2, j, k), A(d, c + 1, j, k), A(d, c, j, k), A(d, c - 1, j, k));
}
static inline double face_y(const oc_sim* s, int sc, const double* d, int i, int c, int k, double vel) {
    if (vel >= 0) return recon(sc, A(d, i, c - 2, k), A(d, i, c - 1, k), A(d, i, c, k), A(d, i, c + 1, k), A(d, i, c + 2, k));
    return recon(sc, A(d, i, c + 3, k), A(d, i, c + 2, k), A(d, i, c + 1, k), A(d, i, c, k), A(d, i, c - 1, k));
}
static inline double face_z(const oc_sim* s, int sc, const double* d, int i, int j, int c, double vel) {
    if (vel >= 0) return recon(sc, A(d, i, j, c - 2), A(d, i, j, c - 1), A(d, i, j, c), A(d, i, j, c + 1), A(d, i, j, c + 2));
    return recon(sc, A(d, i, j, c + 3), A(d, i, j, c + 2), A(d, i, j, c + 1), A(d, i, j, c), A(d, i, j, c - 1));
}

/* flux-form reconstructed scalar advection (src/AdvectionSchemes.jl:685-699) */
static inline double recon_scalar_at(const oc_sim* s, int sc, const double* u, const double* v, const double* w,
                                     const double* f, int i, int j, int k) {
    double uw = A(u, i, j, k), ue = A(u, i + 1, j, k);
    double Fx = (ue * face_x(s, sc, f, i, j, k, ue) - uw * face_x(s, sc, f, i - 1, j, k, uw)) * s->idx;
    double vs = A(v, i, j, k), vn = A(v, i, j + 1, k);
    double Fy = (vn * face_y(s, sc, f, i, j, k, vn) - vs * face_y(s, sc, f, i, j - 1, k, vs)) * s->idy;
    double wb = A(w, i, j, k), wt = A(w, i, j, k + 1);
    double Fz = (wt * face_z(s, sc, f, i, j, k, wt) - wb * face_z(s, sc, f, i, j, k - 1, wb)) * s->idz;
    return Fx + Fy + Fz;
}

/* reconstructed momentum advection (src/AdvectionSchemes.jl:1203-1256) */
static inline double recon_mom_u(const oc_sim* s, int sc, const double* u, const double* v, const double* w, int i, int j, int k) {
    double Ue = (A(u, i, j, k) + A(u, i + 1, j, k)) / 2;
    double Uw = (A(u, i - 1, j, k) + A(u, i, j, k)) / 2;
    double dx = (Ue * face_x(s, sc, u, i, j, k, Ue) - Uw * face_x(s, sc, u, i - 1, j, k, Uw)) * s->idx;
    double Vn = (A(v, i - 1, j + 1, k) + A(v, i, j + 1, k)) / 2;
    double Vs = (A(v, i - 1, j, k) + A(v, i, j, k)) / 2;
    double dy = (Vn * face_y(s, sc, u, i, j, k, Vn) - Vs * face_y(s, sc, u, i, j - 1, k, Vs)) * s->idy;
    double Wt = (A(w, i - 1, j, k + 1) + A(w, i, j, k + 1)) / 2;
    double Wb = (A(w, i - 1, j, k) + A(w, i, j, k)) / 2;
    double dz = (Wt * face_z(s, sc, u, i, j, k, Wt) - Wb * face_z(s, sc, u, i, j, k - 1, Wb)) * s->idz;
    return dx + dy + dz;
}
static inline double recon_mom_v(const oc_sim* s, int sc, const double* u, const double* v, const double* w, int i, int j, int k) {
    double Ue = (A(u, i + 1, j - 1, k) + A(u, i + 1, j, k)) / 2;
    double Uw = (A(u, i, j - 1, k) + A(u, i, j, k)) / 2;
    double dx = (Ue * face_x(s, sc, v, i, j, k, Ue) - Uw * face_x(s, sc, v, i - 1, j, k, Uw)) * s->idx;
    double Vn = (A(v, i, j, k) + A(v, i, j + 1, k)) / 2;
    double Vs = (A(v, i, j - 1, k) + A(v, i, j, k)) / 2;
    double dy = (Vn * face_y(s, sc, v, i, j, k, Vn) - Vs * face_y(s, sc, v, i, j - 1, k, Vs)) * s->idy;
    double Wt = (A(w, i, j - 1, k + 1) + A(w, i, j, k + 1)) / 2;
    double Wb = (A(w, i, j - 1, k) + A(w, i, j, k)) / 2;
    double dz = (Wt * face_z(s, sc, v, i, j, k, Wt) - Wb * face_z(s, sc, v, i, j, k - 1, Wb)) * s->idz;
    return dx + dy + dz;
}
static inline double recon_mom_w(const oc_sim* s, int sc, const double* u, const double* v, const double* w, int i, int j, int k) {
    double Ue = (A(u, i + 1, j, k - 1) + A(u, i + 1, j, k)) / 2;
    double Uw = (A(u, i, j, k - 1) + A(u, i, j, k)) / 2;
    double dx = (Ue * face_x(s, sc, w, i, j, k, Ue) - Uw * face_x(s, sc, w, i - 1, j, k, Uw)) * s->idx;
    double Vn = (A(v, i, j + 1, k - 1) + A(v, i, j + 1, k)) / 2;
    double Vs = (A(v, i, j, k - 1) + A(v, i, j, k)) / 2;
    double dy = (Vn * face_y(s, sc, w, i, j, k, Vn) - Vs * face_y(s, sc, w, i, j - 1, k, Vs)) * s->idy;
    double Wt = (A(w, i, j, k) + A(w, i, j, k + 1)) / 2;
    double Wb = (A(w, i, j, k - 1) + A(w, i, j, k)) / 2;
    double dz = (Wt * face_z(s, sc, w, i, j, k, Wt) - Wb * face_z(s, sc, w, i, j, k - 1, Wb)) * s->idz;
    return dx + dy + dz;
}

/* sigma_operator (src/operators/sigma_closure.jl:130-196): the eigenvalues of
 * g^T g by _sym3_eigvals (:48-97: the trigonometric solution in the
 * deviator; where the smaller gap is under 1 % of the spread, the simple
 * eigenvalue deflated through the largest cross product of two rows of
 * G - lambda I and the close pair from the 2 x 2 compression), s3 from the
 * determinant, D = s3 (s1 - s2)(s2 - s3) / s1^2 clipped at zero. */
static double sigma_op(double g11, double g12, double g13, double g21, double g22, double g23, double g31,
                       double g32, double g33) {
    double G11 = g11 * g11 + g21 * g21 + g31 * g31, G22 = g12 * g12 + g22 * g22 + g32 * g32;
    double G33 = g13 * g13 + g23 * g23 + g33 * g33;
    double G12 = g11 * g12 + g21 * g22 + g31 * g32, G13 = g11 * g13 + g21 * g23 + g31 * g33;
    double G23 = g12 * g13 + g22 * g23 + g32 * g33;
    double m = (G11 + G22 + G33) / 3;
    double a = G11 - m, b = G22 - m, c = G33 - m;
    double off2 = G12 * G12 + G13 * G13 + G23 * G23;
    double al1 = (a * a + b * b + c * c + 2 * off2) / 6;
    double l1 = m, l2 = m;
    if (al1 > 0) {
        double detd = a * (b * c - G23 * G23) - G12 * (G12 * c - G23 * G13) + G13 * (G12 * G23 - b * G13);
        double al2 = detd / 2;
        double r = al2 / (al1 * sqrt(al1));
        r = r < -1 ? -1 : (r > 1 ? 1 : r);
        double ph = acos(r) / 3, sp = sin(ph), cp = cos(ph);
        double sv = 2 * sqrt(al1);
        l1 = m + sv * cp;
        double l3 = m - sv * (cp + sqrt(3.0) * sp) / 2;
        l2 = 3 * m - l1 - l3;
        double gap = (l1 - l2) < (l2 - l3) ? (l1 - l2) : (l2 - l3);
        if (!(gap >= 0.01 * (l1 - l3))) {
            int top = (l1 - l2) >= (l2 - l3);
            double iso = top ? l1 : l3;
            double r1[3] = {G11 - iso, G12, G13}, r2[3] = {G12, G22 - iso, G23}, r3[3] = {G13, G23, G33 - iso};
            double cr[3][3] = {{r1[1] * r2[2] - r1[2] * r2[1], r1[2] * r2[0] - r1[0] * r2[2], r1[0] * r2[1] - r1[1] * r2[0]},
                               {r1[1] * r3[2] - r1[2] * r3[1], r1[2] * r3[0] - r1[0] * r3[2], r1[0] * r3[1] - r1[1] * r3[0]},
                               {r2[1] * r3[2] - r2[2] * r3[1], r2[2] * r3[0] - r2[0] * r3[2], r2[0] * r3[1] - r2[1] * r3[0]}};
            int best = 0;
            double nv = cr[0][0] * cr[0][0] + cr[0][1] * cr[0][1] + cr[0][2] * cr[0][2];
            for (int q = 1; q < 3; ++q) {
                double n = cr[q][0] * cr[q][0] + cr[q][1] * cr[q][1] + cr[q][2] * cr[q][2];
                if (n > nv) { nv = n; best = q; }
            }
            if (nv > 0) {
                double sn = sqrt(nv);
                double v[3] = {cr[best][0] / sn, cr[best][1] / sn, cr[best][2] / sn};
                double ax = fabs(v[0]), ay = fabs(v[1]), az = fabs(v[2]);
                double t[3] = {0, 0, 0};
                if (ax <= ay && ax <= az) t[0] = 1; else if (ay <= az) t[1] = 1; else t[2] = 1;
                double e1[3] = {v[1] * t[2] - v[2] * t[1], v[2] * t[0] - v[0] * t[2], v[0] * t[1] - v[1] * t[0]};
                double ne = sqrt(e1[0] * e1[0] + e1[1] * e1[1] + e1[2] * e1[2]);
                e1[0] /= ne; e1[1] /= ne; e1[2] /= ne;
                double e2[3] = {v[1] * e1[2] - v[2] * e1[1], v[2] * e1[0] - v[0] * e1[2], v[0] * e1[1] - v[1] * e1[0]};
#define SYMMUL(x, o) do { o[0] = G11 * x[0] + G12 * x[1] + G13 * x[2]; \
                          o[1] = G12 * x[0] + G22 * x[1] + G23 * x[2]; \
                          o[2] = G13 * x[0] + G23 * x[1] + G33 * x[2]; } while (0)
                double Gv[3], Ge1[3], Ge2[3];
                SYMMUL(v, Gv); SYMMUL(e1, Ge1); SYMMUL(e2, Ge2);
#undef SYMMUL
                double liso = v[0] * Gv[0] + v[1] * Gv[1] + v[2] * Gv[2];
                double pp = e1[0] * Ge1[0] + e1[1] * Ge1[1] + e1[2] * Ge1[2];
                double qq = e1[0] * Ge2[0] + e1[1] * Ge2[1] + e1[2] * Ge2[2];
                double rr = e2[0] * Ge2[0] + e2[1] * Ge2[1] + e2[2] * Ge2[2];
                double h = sqrt((pp - rr) * (pp - rr) + 4 * qq * qq) / 2;
                double mp = (pp + rr) / 2 + h, mm = (pp + rr) / 2 - h;
                if (top) { l1 = liso > mp ? liso : mp; l2 = mp; }
                else { l1 = mp; l2 = mm; }
            }
        }
    }
    double s1 = sqrt(l1 > 0 ? l1 : 0);
    if (!(s1 > 0)) return 0.0;
    double s2 = sqrt(l2 > 0 ? l2 : 0);
    double detg = g11 * (g22 * g33 - g23 * g32) - g12 * (g21 * g33 - g23 * g31) + g13 * (g21 * g32 - g22 * g31);
    double pr = s1 * s2;
    double s3 = pr > 0 ? fabs(detg) / pr : 0.0;
    double d12 = (l1 - l2 > 0 ? l1 - l2 : 0) / (s1 + s2);
    double D = s3 * d12 * (s2 - s3) / (s1 * s1);
    return D > 0 ? D : 0.0;
}

/* --- AMD: anisotropic minimum dissipation (_amd_point, _amd_scalar_point,
 * _amd_body!, src/operators/sgs_amd_vreman.jl:54-90, :204-212), from the
 * velocity gradient of smag_at (g_ab = du_a/dx_b) and the centred theta
 * gradient (_scalar_gradient_at, :18-25); bg = g/theta0 (0 without
 * buoyancy). nu_t into *nu, theta's own kappa_t into *ka. */
static void amd_at(const oc_sim* s, int i, int j, int k, double* nu, double* ka) {
    const double *u = s->u, *v = s->v, *w = s->w, *t = s->th;
    double idx = s->idx, idy = s->idy, idz = m_idz(s, k), ido = m_idz_off(s, k);
    double g[3][3];
    g[0][0] = (A(u, i + 1, j, k) - A(u, i, j, k)) * idx;
    g[1][1] = (A(v, i, j + 1, k) - A(v, i, j, k)) * idy;
    g[2][2] = (A(w, i, j, k + 1) - A(w, i, j, k)) * idz;
    g[0][1] = ((A(u, i, j + 1, k) + A(u, i + 1, j + 1, k)) - (A(u, i, j - 1, k) + A(u, i + 1, j - 1, k))) * (0.25 * idy);
    g[1][0] = ((A(v, i + 1, j, k) + A(v, i + 1, j + 1, k)) - (A(v, i - 1, j, k) + A(v, i - 1, j + 1, k))) * (0.25 * idx);
    g[0][2] = ((A(u, i, j, k + 1) + A(u, i + 1, j, k + 1)) - (A(u, i, j, k - 1) + A(u, i + 1, j, k - 1))) * (0.25 * ido);
    g[2][0] = ((A(w, i + 1, j, k) + A(w, i + 1, j, k + 1)) - (A(w, i - 1, j, k) + A(w, i - 1, j, k + 1))) * (0.25 * idx);
    g[1][2] = ((A(v, i, j, k + 1) + A(v, i, j + 1, k + 1)) - (A(v, i, j, k - 1) + A(v, i, j + 1, k - 1))) * (0.25 * ido);
    g[2][1] = ((A(w, i, j + 1, k) + A(w, i, j + 1, k + 1)) - (A(w, i, j - 1, k) + A(w, i, j - 1, k + 1))) * (0.25 * idy);
    double gt[3] = {(A(t, i + 1, j, k) - A(t, i - 1, j, k)) * (0.5 * idx),
                    (A(t, i, j + 1, k) - A(t, i, j - 1, k)) * (0.5 * idy),
                    (A(t, i, j, k + 1) - A(t, i, j, k - 1)) * (0.5 * idz)};
    double d2[3] = {s->dx * s->dx, s->dy * s->dy, s->dz * s->dz};
    double bg = s->p.core == OC_CORE_ANELASTIC ? (s->amd_bg ? s->amd_bg[k - s->p.hz] : 0.0)
                                               : (s->p.theta0 != 0 ? s->p.g / s->p.theta0 : 0.0);
#define SDOT(a, b) (d2[0] * (a)[0] * (b)[0] + d2[1] * (a)[1] * (b)[1] + d2[2] * (a)[2] * (b)[2])
    double S12 = 0.5 * (g[0][1] + g[1][0]), S13 = 0.5 * (g[0][2] + g[2][0]), S23 = 0.5 * (g[1][2] + g[2][1]);
    double P = SDOT(g[0], g[0]) * g[0][0] + SDOT(g[1], g[1]) * g[1][1] + SDOT(g[2], g[2]) * g[2][2] +
               2 * (SDOT(g[0], g[1]) * S12 + SDOT(g[0], g[2]) * S13 + SDOT(g[1], g[2]) * S23);
    double B = bg * SDOT(g[2], gt);
    double D = 0;
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) D += g[a][b] * g[a][b];
    double kd = gt[0] * gt[0] + gt[1] * gt[1] + gt[2] * gt[2];
    double N2 = fabs(bg) * sqrt(kd);
    double Bw = D >= N2 ? B : B * (D / N2);           /* B min(1, 1/Ri) */
    double Q = SDOT(g[0], gt) * gt[0] + SDOT(g[1], gt) * gt[1] + SDOT(g[2], gt) * gt[2];
#undef SDOT
    double C = s->p.c_s, nn = -P + Bw;
    *nu = D > 0 ? C * fmax(0.0, nn) / D : 0.0;
    *ka = kd > 0 ? C * fmax(0.0, -Q) / kd : *nu / s->p.pr_t;
}

/* --- dynamic Smagorinsky (compute_dynamic_smagorinsky_nut!, plane
 * averaging, filter ratio 3, clip c_s^2; src/Operators.jl:548-900): pass 1
 * (_germano_pass1_body!) the cell-centred velocity, strain and |S| on the
 * interior + one shell; pass 2 (_germano_pass2_body!, _germano_LM_MM) the
 * 3x3x3 box sums (z outer, x inner) and L^d:M, M:M; the plane sums (j outer,
 * i inner) and the clip (_plane_cs2_body!) into s->cs2. */
static double* dalloc(int64_t n);
static void dyn_coefficients(oc_sim* s) {
    const oc_params* P = &s->p;
    int Hx = P->hx, Hy = P->hy, Hz = P->hz, Nx = P->nx, Ny = P->ny, Nz = P->nz;
    int SX = Nx + 2, SY = Ny + 2, SZ = Nz + 2;
    size_t ns = (size_t)SX * SY * SZ, ni = (size_t)Nx * Ny * Nz;
    if (!s->dyn[0]) {
        for (int f = 0; f < 10; ++f) s->dyn[f] = dalloc((int64_t)ns);
        s->dyn_lm = dalloc((int64_t)ni); s->dyn_mm = dalloc((int64_t)ni); s->cs2 = dalloc(Nz);
    }
    const double *u = s->u, *v = s->v, *w = s->w;
    double idx = s->idx, idy = s->idy, idz = s->idz;
#define SH(li, lj, lk) ((size_t)(li) + (size_t)SX * ((size_t)(lj) + (size_t)SY * (size_t)(lk)))
#pragma omp parallel for collapse(2) schedule(static)
    for (int lk = 0; lk < SZ; ++lk)
        for (int lj = 0; lj < SY; ++lj)
            for (int li = 0; li < SX; ++li) {
                int i = Hx - 1 + li, j = Hy - 1 + lj, k = Hz - 1 + lk;
                size_t e = SH(li, lj, lk);
                s->dyn[0][e] = 0.5 * (A(u, i, j, k) + A(u, i + 1, j, k));
                s->dyn[1][e] = 0.5 * (A(v, i, j, k) + A(v, i, j + 1, k));
                s->dyn[2][e] = 0.5 * (A(w, i, j, k) + A(w, i, j, k + 1));
                double du_dx = (A(u, i + 1, j, k) - A(u, i, j, k)) * idx;
                double dv_dy = (A(v, i, j + 1, k) - A(v, i, j, k)) * idy;
                double dw_dz = (A(w, i, j, k + 1) - A(w, i, j, k)) * idz;
                double du_dy = ((A(u, i, j + 1, k) + A(u, i + 1, j + 1, k)) - (A(u, i, j - 1, k) + A(u, i + 1, j - 1, k))) * (0.25 * idy);
                double dv_dx = ((A(v, i + 1, j, k) + A(v, i + 1, j + 1, k)) - (A(v, i - 1, j, k) + A(v, i - 1, j + 1, k))) * (0.25 * idx);
                double du_dz = ((A(u, i, j, k + 1) + A(u, i + 1, j, k + 1)) - (A(u, i, j, k - 1) + A(u, i + 1, j, k - 1))) * (0.25 * idz);
                double dw_dx = ((A(w, i + 1, j, k) + A(w, i + 1, j, k + 1)) - (A(w, i - 1, j, k) + A(w, i - 1, j, k + 1))) * (0.25 * idx);
                double dv_dz = ((A(v, i, j, k + 1) + A(v, i, j + 1, k + 1)) - (A(v, i, j, k - 1) + A(v, i, j + 1, k - 1))) * (0.25 * idz);
                double dw_dy = ((A(w, i, j + 1, k) + A(w, i, j + 1, k + 1)) - (A(w, i, j - 1, k) + A(w, i, j - 1, k + 1))) * (0.25 * idy);
                double S12 = 0.5 * (du_dy + dv_dx), S13 = 0.5 * (du_dz + dw_dx), S23 = 0.5 * (dv_dz + dw_dy);
                double S2 = 2 * (du_dx * du_dx + dv_dy * dv_dy + dw_dz * dw_dz) + 4 * (S12 * S12 + S13 * S13 + S23 * S23);
                s->dyn[3][e] = du_dx; s->dyn[4][e] = dv_dy; s->dyn[5][e] = dw_dz;
                s->dyn[6][e] = S12; s->dyn[7][e] = S13; s->dyn[8][e] = S23;
                s->dyn[9][e] = sqrt(S2);
            }
    const double d2 = pow(s->dx * s->dy * s->dz, 2.0 / 3.0), a2 = 9.0, inv = 1.0 / 27;
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < Nz; ++k)
        for (int j = 0; j < Ny; ++j)
            for (int i = 0; i < Nx; ++i) {
                double t[21] = {0};
                for (int c = 0; c < 3; ++c)
                    for (int b = 0; b < 3; ++b)
                        for (int a = 0; a < 3; ++a) {
                            size_t e = SH(i + a, j + b, k + c);
                            double uu = s->dyn[0][e], vv = s->dyn[1][e], ww = s->dyn[2][e], ms = s->dyn[9][e];
                            t[0] += uu; t[1] += vv; t[2] += ww;
                            t[3] += uu * uu; t[4] += vv * vv; t[5] += ww * ww;
                            t[6] += uu * vv; t[7] += uu * ww; t[8] += vv * ww;
                            for (int q = 0; q < 6; ++q) { t[9 + q] += s->dyn[3 + q][e]; t[15 + q] += ms * s->dyn[3 + q][e]; }
                        }
                double Ut = t[0] * inv, Vt = t[1] * inv, Wt = t[2] * inv;
                double L11 = t[3] * inv - Ut * Ut, L22 = t[4] * inv - Vt * Vt, L33 = t[5] * inv - Wt * Wt;
                double L12 = t[6] * inv - Ut * Vt, L13 = t[7] * inv - Ut * Wt, L23 = t[8] * inv - Vt * Wt;
                double tr = (L11 + L22 + L33) / 3;
                L11 -= tr; L22 -= tr; L33 -= tr;
                double A11 = t[9] * inv, A22 = t[10] * inv, A33 = t[11] * inv;
                double A12 = t[12] * inv, A13 = t[13] * inv, A23 = t[14] * inv;
                double magSt = sqrt(2 * (A11 * A11 + A22 * A22 + A33 * A33) + 4 * (A12 * A12 + A13 * A13 + A23 * A23));
                double c1 = 2 * d2 * a2 * magSt, c2 = 2 * d2 * inv;
                double M11 = c2 * t[15] - c1 * A11, M22 = c2 * t[16] - c1 * A22, M33 = c2 * t[17] - c1 * A33;
                double M12 = c2 * t[18] - c1 * A12, M13 = c2 * t[19] - c1 * A13, M23 = c2 * t[20] - c1 * A23;
                size_t q = (size_t)i + (size_t)Nx * ((size_t)j + (size_t)Ny * k);
                s->dyn_lm[q] = L11 * M11 + L22 * M22 + L33 * M33 + 2 * (L12 * M12 + L13 * M13 + L23 * M23);
                s->dyn_mm[q] = M11 * M11 + M22 * M22 + M33 * M33 + 2 * (M12 * M12 + M13 * M13 + M23 * M23);
            }
#undef SH
    if (P->sgs_model == OC_SGS_LAGRANGIAN) return;   /* the identity's LM, MM feed the memories */
    double cmax = P->c_s * P->c_s;
    if (P->sgs_model == OC_SGS_DYNAMIC_LOCAL) {   /* _local_cs2_body!: each cell's own ratio, clipped */
        for (size_t q = 0; q < ni; ++q)
            s->dyn_lm[q] = s->dyn_mm[q] > 0 ? fmin(fmax(s->dyn_lm[q] / s->dyn_mm[q], 0.0), cmax) : 0.0;
        return;
    }
    for (int k = 0; k < Nz; ++k) {
        double lm = 0, mm = 0;
        for (int j = 0; j < Ny; ++j)
            for (int i = 0; i < Nx; ++i) {
                size_t q = (size_t)i + (size_t)Nx * ((size_t)j + (size_t)Ny * k);
                lm += s->dyn_lm[q]; mm += s->dyn_mm[q];
            }
        s->cs2[k] = mm > 0 ? fmin(fmax(lm / mm, 0.0), cmax) : 0.0;
    }
}

/* --- Lagrangian dynamic Smagorinsky (LagrangianDynamicSmagorinsky,
 * src/operators/lagrangian_sgs.jl; Meneveau, Lund & Cabot 1996): the
 * scale-invariant model, cadence 1, no mask.  The coefficient of a step is
 * that of the committed memory (sgs_viscosity!, :214-236): min(C0^2,
 * cs_max^2) before the first commit, then _local_cs2_body!(I_LM, I_MM). */
static void lag_coefficient(oc_sim* s) {
    const oc_params* P = &s->p;
    size_t ni = (size_t)P->nx * P->ny * P->nz;
    double cmax = P->c_s * P->c_s;
    for (size_t q = 0; q < ni; ++q) {
        if (!s->lag_init) { s->lag_cs2[q] = fmin(s->lag_c0 * s->lag_c0, cmax); continue; }
        double mm = s->lag_imm[q];
        s->lag_cs2[q] = mm > 0 ? fmin(fmax(s->lag_ilm[q] / mm, 0.0), cmax) : 0.0;
    }
}

static void lag_alloc(oc_sim* s) {
    if (s->lag_ilm) return;
    int64_t ni = (int64_t)s->p.nx * s->p.ny * s->p.nz;
    s->lag_ilm = dalloc(ni); s->lag_imm = dalloc(ni); s->lag_up = dalloc(ni); s->lag_vp = dalloc(ni);
    s->lag_wp = dalloc(ni); s->lag_cs2 = dalloc(ni); s->lag_nlm = dalloc(ni); s->lag_nmm = dalloc(ni);
    s->lag_init = 0;
    if (s->lag_c0 == 0) { s->lag_c0 = 0.16; s->lag_theta = 1.5; s->lag_mt = 0.0; }
    lag_coefficient(s);
}

/* _wrapidx (lagrangian_sgs.jl:392): the 1-based index n wrapped (periodic) or
 * clamped to [1, N]; returned 0-based */
static inline int lag_wrap(int n, int N, int per) {
    if (per) return ((n - 1) % N + N) % N;
    return (n < 1 ? 1 : (n > N ? N : n)) - 1;
}

/* advance_sgs! (lagrangian_sgs.jl:306-355): the Germano identity at the state
 * after the step (velocity halos filled first); the first commit sets I_MM =
 * MM, I_LM = C0^2 MM, later ones relax along the pathlines
 * (_lagrangian_relax! / _relax_body! / _relax_pairs!, :478-568): the
 * departure point x - u^n dt of every cell (1-based fractional cell indices,
 * clamped to [1, N] across a wall, _upstream_n :406-436), the trilinear
 * interpolation of the old memories (dk, dj, di order), the time scale T =
 * theta Delta (max(lm, 1e-8 mm) mm)^(-1/8) (epsilon = 1 where mm = 0, or the
 * fixed memory_time), I_LM clipped at 0; then u^n is the new cell-centred
 * velocity. */
static void lag_commit(oc_sim* s, double dt) {
    const oc_params* P = &s->p;
    int Nx = P->nx, Ny = P->ny, Nz = P->nz;
    int SX = Nx + 2, SY = Ny + 2;
    size_t ni = (size_t)Nx * Ny * Nz;
    lag_alloc(s);
    fill_halos(s, s->u, LOC_FX);
    fill_halos(s, s->v, LOC_FY);
    fill_halos(s, s->w, LOC_FZ);
    dyn_coefficients(s);
    if (!s->lag_init) {
        double c02 = s->lag_c0 * s->lag_c0;
        for (size_t q = 0; q < ni; ++q) { s->lag_imm[q] = s->dyn_mm[q]; s->lag_ilm[q] = c02 * s->dyn_mm[q]; }
        s->lag_init = 1;
    } else {
        double Delta = pow(s->dx * s->dy * s->dz, 1.0 / 3);
        double cx = dt / s->dx, cy = dt / s->dy, cz = dt / s->dz;
        double mt = s->lag_mt, th = s->lag_theta;
        double efix = mt > 0 ? (dt / mt) / (1 + dt / mt) : 0.0;
        int pz = P->bc_z == OC_BC_PERIODIC;
#pragma omp parallel for collapse(2) schedule(static)
        for (int k = 0; k < Nz; ++k)
            for (int j = 0; j < Ny; ++j)
                for (int i = 0; i < Nx; ++i) {
                    size_t q = (size_t)i + (size_t)Nx * ((size_t)j + (size_t)Ny * k);
                    double x = (i + 1) - s->lag_up[q] * cx, y = (j + 1) - s->lag_vp[q] * cy;
                    double z = (k + 1) - s->lag_wp[q] * cz;
                    if (!pz) z = z < 1 ? 1.0 : (z > Nz ? (double)Nz : z);
                    int x0 = (int)floor(x), y0 = (int)floor(y), z0 = (int)floor(z);
                    double fx = x - x0, fy = y - y0, fz = z - z0;
                    double lm = 0.0, mm = 0.0;
                    for (int dk = 0; dk <= 1; ++dk)
                        for (int dj = 0; dj <= 1; ++dj)
                            for (int di = 0; di <= 1; ++di) {
                                int a = lag_wrap(x0 + di, Nx, 1), b = lag_wrap(y0 + dj, Ny, 1), c = lag_wrap(z0 + dk, Nz, pz);
                                double wgt = (di == 0 ? 1 - fx : fx) * (dj == 0 ? 1 - fy : fy) * (dk == 0 ? 1 - fz : fz);
                                size_t r = (size_t)a + (size_t)Nx * ((size_t)b + (size_t)Ny * c);
                                lm += wgt * s->lag_ilm[r];
                                mm += wgt * s->lag_imm[r];
                            }
                    double eps;
                    if (mt > 0) eps = efix;
                    else if (mm > 0) {
                        double Tl = th * Delta * pow(fmax(lm, 1e-8 * mm) * mm, -1.0 / 8);
                        eps = (dt / Tl) / (1 + dt / Tl);
                    } else eps = 1.0;
                    s->lag_nlm[q] = fmax(eps * s->dyn_lm[q] + (1 - eps) * lm, 0.0);
                    s->lag_nmm[q] = eps * s->dyn_mm[q] + (1 - eps) * mm;
                }
        memcpy(s->lag_ilm, s->lag_nlm, ni * sizeof(double));
        memcpy(s->lag_imm, s->lag_nmm, ni * sizeof(double));
    }
    for (int k = 0; k < Nz; ++k)
        for (int j = 0; j < Ny; ++j)
            for (int i = 0; i < Nx; ++i) {
                size_t q = (size_t)i + (size_t)Nx * ((size_t)j + (size_t)Ny * k);
                size_t e = (size_t)(i + 1) + (size_t)SX * ((size_t)(j + 1) + (size_t)SY * (size_t)(k + 1));
                s->lag_up[q] = s->dyn[0][e]; s->lag_vp[q] = s->dyn[1][e]; s->lag_wp[q] = s->dyn[2][e];
            }
    lag_coefficient(s);
}

/* --- Deardorff TKE closure (TKEClosure, src/PrognosticSGS.jl; Deardorff
 * 1980, Moeng 1984): Boussinesq core, uniform grid, no mask / wall cap /
 * first-level factor / surface value, dry N^2. --------------------------- */
static void tke_alloc(oc_sim* s) {
    if (s->tke_e) return;
    s->tke_e = dalloc(s->n); s->tke_k2 = dalloc(s->n); s->tke_tend = dalloc(s->n);
    s->tke_new = dalloc((int64_t)s->p.nx * s->p.ny * s->p.nz);
    s->tke_ce0 = 0.19; s->tke_ce1 = 0.51; s->tke_cl = 0.76; s->tke_exact = 0;
}

/* N^2 of cell (i, j, k): (g/theta0) (theta_face_above - theta_face_below) / dz
 * with the faces the two-cell means (buoyancy_frequency_squared!,
 * src/operators/stratification.jl:124-135; TurbulenceStability.jl:129-130) */
static inline double tke_n2(const oc_sim* s, int i, int j, int k) {
    const oc_params* P = &s->p;
    if (!(P->theta0 > 0 && P->g > 0)) return 0.0;
    const double* th = s->th;
    double below = 0.5 * (A(th, i, j, k - 1) + A(th, i, j, k)), above = 0.5 * (A(th, i, j, k) + A(th, i, j, k + 1));
    return (P->g / P->theta0) * (above - below) * (1 / s->dz);
}

/* tke_length_scale (src/PrognosticSGS.jl:93-110): l and s = sqrt(e) / l */
static inline void tke_length(const oc_sim* s, double e, double N2, double* l, double* sr) {
    double Delta = pow(s->dx * s->dy * s->dz, 1.0 / 3), cl = s->tke_cl;
    double sq = sqrt(fmax(e, 0.0)), lmax = Delta;
    int stable = N2 > 0;
    double N = sqrt(fmax(N2, 0.0));
    *l = stable ? fmin(lmax, cl * sq / N) : lmax;
    *sr = stable ? fmax(sq / lmax, N / cl) : sq / lmax;
}

/* nu_t = c_k l sqrt(e), kappa_t = (1 + 2 l / Delta) nu_t of the committed e and
 * the current N^2 (_coefficients_body! / tke_eddy_coefficients, :432-454, :135-139) */
static void tke_at(const oc_sim* s, int i, int j, int k, double* nu, double* ka) {
    double Delta = pow(s->dx * s->dy * s->dz, 1.0 / 3);
    double e = A(s->tke_e, i, j, k), l, sr;
    tke_length(s, e, tke_n2(s, i, j, k), &l, &sr);
    double v = s->p.c_s * l * sqrt(fmax(e, 0.0));
    *nu = v;
    *ka = (1 + 2 * l / Delta) * v;
}

/* The share of D destined for storage cell (I, J, K) from the velocity points
 * around it (_dual_raw, src/PrognosticSGS.jl:589-632, with the flux shares
 * :541-560 on a RegularGrid): each flux nu dq / h of the momentum operator
 * gives -u_p (+-flux) / h to the cells of its nu.  Points outside the
 * interior box give nothing. */
static double dual_raw(const oc_sim* s, int I, int J, int K) {
    const oc_params* P = &s->p;
    const double *u = s->u, *v = s->v, *w = s->w;
    const double ix2 = 1 / (s->dx * s->dx), iy2 = 1 / (s->dy * s->dy), iz2 = 1 / (s->dz * s->dz);
    int i1 = P->hx, i2 = P->hx + P->nx - 1, j1 = P->hy, j2 = P->hy + P->ny - 1, k1 = P->hz, k2 = P->hz + P->nz - 1;
#define IN(i, j, k) ((i) >= i1 && (i) <= i2 && (j) >= j1 && (j) <= j2 && (k) >= k1 && (k) <= k2)
#define UX_E(i, j, k) (IN(i, j, k) ? -A(u, i, j, k) * (A(u, i + 1, j, k) - A(u, i, j, k)) * ix2 : 0.0)
#define UX_W(i, j, k) (IN(i, j, k) ? A(u, i, j, k) * (A(u, i, j, k) - A(u, i - 1, j, k)) * ix2 : 0.0)
#define UY_N(i, j, k) (IN(i, j, k) ? 0.25 * (-A(u, i, j, k) * (A(u, i, j + 1, k) - A(u, i, j, k)) * iy2) : 0.0)
#define UY_S(i, j, k) (IN(i, j, k) ? 0.25 * (A(u, i, j, k) * (A(u, i, j, k) - A(u, i, j - 1, k)) * iy2) : 0.0)
#define UZ_T(i, j, k) (IN(i, j, k) ? 0.25 * (-A(u, i, j, k) * (A(u, i, j, k + 1) - A(u, i, j, k)) * iz2) : 0.0)
#define UZ_B(i, j, k) (IN(i, j, k) ? 0.25 * (A(u, i, j, k) * (A(u, i, j, k) - A(u, i, j, k - 1)) * iz2) : 0.0)
#define VY_N(i, j, k) (IN(i, j, k) ? -A(v, i, j, k) * (A(v, i, j + 1, k) - A(v, i, j, k)) * iy2 : 0.0)
#define VY_S(i, j, k) (IN(i, j, k) ? A(v, i, j, k) * (A(v, i, j, k) - A(v, i, j - 1, k)) * iy2 : 0.0)
#define VX_E(i, j, k) (IN(i, j, k) ? 0.25 * (-A(v, i, j, k) * (A(v, i + 1, j, k) - A(v, i, j, k)) * ix2) : 0.0)
#define VX_W(i, j, k) (IN(i, j, k) ? 0.25 * (A(v, i, j, k) * (A(v, i, j, k) - A(v, i - 1, j, k)) * ix2) : 0.0)
#define VZ_T(i, j, k) (IN(i, j, k) ? 0.25 * (-A(v, i, j, k) * (A(v, i, j, k + 1) - A(v, i, j, k)) * iz2) : 0.0)
#define VZ_B(i, j, k) (IN(i, j, k) ? 0.25 * (A(v, i, j, k) * (A(v, i, j, k) - A(v, i, j, k - 1)) * iz2) : 0.0)
#define WZ_T(i, j, k) (IN(i, j, k) ? -A(w, i, j, k) * (A(w, i, j, k + 1) - A(w, i, j, k)) * iz2 : 0.0)
#define WZ_B(i, j, k) (IN(i, j, k) ? A(w, i, j, k) * (A(w, i, j, k) - A(w, i, j, k - 1)) * iz2 : 0.0)
#define WX_E(i, j, k) (IN(i, j, k) ? 0.25 * (-A(w, i, j, k) * (A(w, i + 1, j, k) - A(w, i, j, k)) * ix2) : 0.0)
#define WX_W(i, j, k) (IN(i, j, k) ? 0.25 * (A(w, i, j, k) * (A(w, i, j, k) - A(w, i - 1, j, k)) * ix2) : 0.0)
#define WY_N(i, j, k) (IN(i, j, k) ? 0.25 * (-A(w, i, j, k) * (A(w, i, j + 1, k) - A(w, i, j, k)) * iy2) : 0.0)
#define WY_S(i, j, k) (IN(i, j, k) ? 0.25 * (A(w, i, j, k) * (A(w, i, j, k) - A(w, i, j - 1, k)) * iy2) : 0.0)
    double d = UX_E(I, J, K) + UX_W(I + 1, J, K);
    d += (UY_N(I + 1, J, K) + UY_N(I, J, K)) + (UY_N(I + 1, J - 1, K) + UY_N(I, J - 1, K));
    d += (UY_S(I + 1, J + 1, K) + UY_S(I, J + 1, K)) + (UY_S(I + 1, J, K) + UY_S(I, J, K));
    d += (UZ_T(I + 1, J, K) + UZ_T(I, J, K)) + (UZ_T(I + 1, J, K - 1) + UZ_T(I, J, K - 1));
    d += (UZ_B(I + 1, J, K + 1) + UZ_B(I, J, K + 1)) + (UZ_B(I + 1, J, K) + UZ_B(I, J, K));
    d += VY_N(I, J, K) + VY_S(I, J + 1, K);
    d += (VX_E(I, J + 1, K) + VX_E(I - 1, J + 1, K)) + (VX_E(I, J, K) + VX_E(I - 1, J, K));
    d += (VX_W(I + 1, J + 1, K) + VX_W(I, J + 1, K)) + (VX_W(I + 1, J, K) + VX_W(I, J, K));
    d += (VZ_T(I, J + 1, K) + VZ_T(I, J, K)) + (VZ_T(I, J + 1, K - 1) + VZ_T(I, J, K - 1));
    d += (VZ_B(I, J + 1, K + 1) + VZ_B(I, J, K + 1)) + (VZ_B(I, J + 1, K) + VZ_B(I, J, K));
    d += WZ_T(I, J, K) + WZ_B(I, J, K + 1);
    d += (WX_E(I, J, K + 1) + WX_E(I - 1, J, K + 1)) + (WX_E(I, J, K) + WX_E(I - 1, J, K));
    d += (WX_W(I + 1, J, K + 1) + WX_W(I, J, K + 1)) + (WX_W(I + 1, J, K) + WX_W(I, J, K));
    d += (WY_N(I, J, K + 1) + WY_N(I, J - 1, K + 1)) + (WY_N(I, J, K) + WY_N(I, J - 1, K));
    d += (WY_S(I, J + 1, K + 1) + WY_S(I, J, K + 1)) + (WY_S(I, J + 1, K) + WY_S(I, J, K));
#undef IN
#undef UX_E
#undef UX_W
#undef UY_N
#undef UY_S
#undef UZ_T
#undef UZ_B
#undef VY_N
#undef VY_S
#undef VX_E
#undef VX_W
#undef VZ_T
#undef VZ_B
#undef WZ_T
#undef WZ_B
#undef WX_E
#undef WX_W
#undef WY_N
#undef WY_S
    return d;
}

/* _fold_src (src/PrognosticSGS.jl:639-640): source n (1 itself, 2 the low halo
 * layer, 3 the high one) of storage index I along a direction whose low /
 * high halo layers H, H+N+1 are copies of lo / hi; -1 = none */
static inline int fold_src(int I, int H, int N, int lo, int hi, int n) {
    return n == 1 ? I : (n == 2 ? (lo == I ? H - 1 : -1) : (hi == I ? H + N : -1));
}

/* D of interior storage cell (I, J, K) (dual_strain!, _dual_strain_body!,
 * :642-665): the shares of every source the halo fold assigns to it.  The
 * halo images: periodic (H+N-1, H), a wall mirror (H, H+N-1) (0-based). */
static double dual_strain(const oc_sim* s, int I, int J, int K) {
    const oc_params* P = &s->p;
    int Hx = P->hx, Hy = P->hy, Hz = P->hz, Nx = P->nx, Ny = P->ny, Nz = P->nz;
    int lox = Hx + Nx - 1, hix = Hx, loy = Hy + Ny - 1, hiy = Hy;
    int pz = P->bc_z == OC_BC_PERIODIC;
    int loz = pz ? Hz + Nz - 1 : Hz, hiz = pz ? Hz : Hz + Nz - 1;
    double acc = 0.0;
    for (int nz = 1; nz <= 3; ++nz) {
        int sz = fold_src(K, Hz, Nz, loz, hiz, nz);
        if (sz < 0) continue;
        for (int ny = 1; ny <= 3; ++ny) {
            int sy = fold_src(J, Hy, Ny, loy, hiy, ny);
            if (sy < 0) continue;
            for (int nx = 1; nx <= 3; ++nx) {
                int sx = fold_src(I, Hx, Nx, lox, hix, nx);
                if (sx < 0) continue;
                acc += dual_raw(s, sx, sy, sz);
            }
        }
    }
    return acc;
}

/* advance_sgs! of the TKE closure (src/PrognosticSGS.jl:978-1002) over an
 * accepted step: the coefficients of e^n and the new N^2, K = 2 nu_t with
 * filled halos, D, the flux-limited WENO-Z5 transport of e
 * (advect_positive!, accumulate = false) plus div(2 nu_t grad e), then the
 * update of every cell (_tke_update_body, :1077-1145): e* = e + dt (T + P_s
 * + max(P_b, 0)), clipped at 0, and the sinks (dissipation c_eps s e, the
 * buoyant destruction) linearised implicit, or with the exact dissipation
 * step (e*^(-1/2) + c_eps dt / (2 l))^(-2).  A prescribed surface heat flux
 * adds (g/theta0) F / 2 to the first / last level (_surface_buoyancy). */
static void tke_commit(oc_sim* s, double dt) {
    const oc_params* P = &s->p;
    int Hx = P->hx, Hy = P->hy, Hz = P->hz, Nx = P->nx, Ny = P->ny, Nz = P->nz;
    fill_halos(s, s->u, LOC_FX);
    fill_halos(s, s->v, LOC_FY);
    fill_halos(s, s->w, LOC_FZ);
    fill_halos(s, s->th, LOC_C);
    double Delta = pow(s->dx * s->dy * s->dz, 1.0 / 3);
    for (int k = Hz; k < Hz + Nz; ++k)
        for (int j = Hy; j < Hy + Ny; ++j)
            for (int i = Hx; i < Hx + Nx; ++i) {
                double nu, ka;
                tke_at(s, i, j, k, &nu, &ka);
                A(s->tke_k2, i, j, k) = 2 * nu;
            }
    fill_halos(s, s->tke_k2, LOC_C);
    fill_halos(s, s->tke_e, LOC_C);
    oc_advect_positive(s, s->u, s->v, s->w, s->tke_e, s->tke_tend, dt, OC_ADV_WENO_Z5, 0);
    int buoy = P->theta0 > 0 && P->g > 0;
    double pb1 = buoy ? P->g / P->theta0 * P->flux_bot / 2 : 0.0, pb2 = buoy ? P->g / P->theta0 * P->flux_top / 2 : 0.0;
    const double* e0 = s->tke_e;
    const double* K2 = s->tke_k2;
    const double ck = P->c_s, tiny = 2.2250738585072014e-308;
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = Hz; k < Hz + Nz; ++k)
        for (int j = Hy; j < Hy + Ny; ++j)
            for (int i = Hx; i < Hx + Nx; ++i) {
                /* the diffusion of e with K = 2 nu_t (_b_eddy_scalar!, src/FiniteVolume.jl:1280-1300) */
                double nE = 0.5 * (A(K2, i, j, k) + A(K2, i + 1, j, k)), nW = 0.5 * (A(K2, i - 1, j, k) + A(K2, i, j, k));
                double nN = 0.5 * (A(K2, i, j, k) + A(K2, i, j + 1, k)), nS = 0.5 * (A(K2, i, j - 1, k) + A(K2, i, j, k));
                double nT = 0.5 * (A(K2, i, j, k) + A(K2, i, j, k + 1)), nB = 0.5 * (A(K2, i, j, k - 1) + A(K2, i, j, k));
                double fxE = nE * (A(e0, i + 1, j, k) - A(e0, i, j, k)) * s->idx;
                double fxW = nW * (A(e0, i, j, k) - A(e0, i - 1, j, k)) * s->idx;
                double fyN = nN * (A(e0, i, j + 1, k) - A(e0, i, j, k)) * s->idy;
                double fyS = nS * (A(e0, i, j, k) - A(e0, i, j - 1, k)) * s->idy;
                double fzT = nT * (A(e0, i, j, k + 1) - A(e0, i, j, k)) * s->idz;
                double fzB = nB * (A(e0, i, j, k) - A(e0, i, j, k - 1)) * s->idz;
                double tr = A(s->tke_tend, i, j, k) +
                            1.0 * ((fxE - fxW) * s->idx + (fyN - fyS) * s->idy + (fzT - fzB) * s->idz);
                double e = A(e0, i, j, k), N2 = tke_n2(s, i, j, k), l, sr;
                tke_length(s, e, N2, &l, &sr);
                double ce = (s->tke_ce0 + s->tke_ce1 * l / Delta) * 1.0;
                double nu = A(K2, i, j, k) / 2;
                double Ps = nu * dual_strain(s, i, j, k) + 0.0;
                double kv = (1 + 2 * l / Delta) * nu;
                int kk = k - Hz + 1;
                double Psf = (kk == 1 ? pb1 : 0.0) + (kk == Nz ? pb2 : 0.0);
                double src = Ps + (N2 < 0 ? -kv * N2 : 0.0) + fmax(Psf, 0.0);
                double rb = ((N2 > 0) && (sr > 0) ? (1 + 2 * l / Delta) * ck * N2 / sr : 0.0) +
                            (Psf < 0 ? -Psf / fmax(e, tiny) : 0.0);
                double es = e + dt * (tr + src);
                if (es < 0) es = 0.0;
                double R = ce * sr + rb;
                double en = es / (1 + dt * R);
                if (s->tke_exact && l > 0 && es > 0) {
                    double a = 1 / (1 / sqrt(es) + ce * dt / (2 * l));
                    en = (a * a) / (1 + dt * rb);
                }
                s->tke_new[(size_t)(i - Hx) + (size_t)Nx * ((size_t)(j - Hy) + (size_t)Ny * (k - Hz))] = en;
            }
    for (int k = Hz; k < Hz + Nz; ++k)
        for (int j = Hy; j < Hy + Ny; ++j)
            for (int i = Hx; i < Hx + Nx; ++i)
                A(s->tke_e, i, j, k) = s->tke_new[(size_t)(i - Hx) + (size_t)Nx * ((size_t)(j - Hy) + (size_t)Ny * (k - Hz))];
    fill_halos(s, s->tke_e, LOC_C);
}

/* --- Smagorinsky (src/FiniteVolume.jl:936-944, src/Operators.jl:451-496) -- */
static inline double smag_at(const oc_sim* s, int i, int j, int k) {
    const double *u = s->u, *v = s->v, *w = s->w;
    double idx = s->idx, idy = s->idy, idz = m_idz(s, k), ido = m_idz_off(s, k);
    double coef = (s->p.c_s * m_filter(s, k)) * (s->p.c_s * m_filter(s, k));
    double du_dx = (A(u, i + 1, j, k) - A(u, i, j, k)) * idx;
    double dv_dy = (A(v, i, j + 1, k) - A(v, i, j, k)) * idy;
    double dw_dz = (A(w, i, j, k + 1) - A(w, i, j, k)) * idz;
    double du_dy = ((A(u, i, j + 1, k) + A(u, i + 1, j + 1, k)) - (A(u, i, j - 1, k) + A(u, i + 1, j - 1, k))) * (0.25 * idy);
    double dv_dx = ((A(v, i + 1, j, k) + A(v, i + 1, j + 1, k)) - (A(v, i - 1, j, k) + A(v, i - 1, j + 1, k))) * (0.25 * idx);
    double du_dz = ((A(u, i, j, k + 1) + A(u, i + 1, j, k + 1)) - (A(u, i, j, k - 1) + A(u, i + 1, j, k - 1))) * (0.25 * ido);
    double dw_dx = ((A(w, i + 1, j, k) + A(w, i + 1, j, k + 1)) - (A(w, i - 1, j, k) + A(w, i - 1, j, k + 1))) * (0.25 * idx);
    double dv_dz = ((A(v, i, j, k + 1) + A(v, i, j + 1, k + 1)) - (A(v, i, j, k - 1) + A(v, i, j + 1, k - 1))) * (0.25 * ido);
    double dw_dy = ((A(w, i, j + 1, k) + A(w, i, j + 1, k + 1)) - (A(w, i, j - 1, k) + A(w, i, j - 1, k + 1))) * (0.25 * idy);
    if (s->p.sgs_model == OC_SGS_AMD) {
        double nu, ka;
        amd_at(s, i, j, k, &nu, &ka);
        return nu;
    }
    double S11 = du_dx, S22 = dv_dy, S33 = dw_dz;
    double S12 = 0.5 * (du_dy + dv_dx);
    double S13 = 0.5 * (du_dz + dw_dx);
    double S23 = 0.5 * (dv_dz + dw_dy);
    if (s->p.sgs_model == OC_SGS_SIGMA)   /* (C_sigma Delta)^2 D_sigma, compute_sigma_nut! (sigma_closure.jl:208-222) */
        return coef * sigma_op(du_dx, du_dy, du_dz, dv_dx, dv_dy, dv_dz, dw_dx, dw_dy, dw_dz);
    if (s->p.sgs_model == OC_SGS_VREMAN) {
        /* Vreman (2004): c sqrt(B_beta / alpha:alpha), c = 2.5 C_s^2, B_beta in the
         * Cauchy-Binet form over the rows a_m = d_m u (_vreman_point,
         * src/operators/sgs_amd_vreman.jl:93-100; _vreman_body! :293-298) */
        double a1[3] = {du_dx, dv_dx, dw_dx}, a2[3] = {du_dy, dv_dy, dw_dy}, a3[3] = {du_dz, dv_dz, dw_dz};
        double d2x = s->dx * s->dx, d2y = s->dy * s->dy, d2z = s->dz * s->dz;
#define CROSS2(a, b) ((a[1] * b[2] - a[2] * b[1]) * (a[1] * b[2] - a[2] * b[1]) + \
                      (a[2] * b[0] - a[0] * b[2]) * (a[2] * b[0] - a[0] * b[2]) + \
                      (a[0] * b[1] - a[1] * b[0]) * (a[0] * b[1] - a[1] * b[0]))
        double Bb = d2x * d2y * CROSS2(a1, a2) + d2x * d2z * CROSS2(a1, a3) + d2y * d2z * CROSS2(a2, a3);
#undef CROSS2
        double aa = du_dx * du_dx + du_dy * du_dy + du_dz * du_dz + dv_dx * dv_dx + dv_dy * dv_dy + dv_dz * dv_dz +
                    dw_dx * dw_dx + dw_dy * dw_dy + dw_dz * dw_dz;
        double c = 2.5 * s->p.c_s * s->p.c_s;
        return aa > 0 ? c * sqrt(Bb / aa) : 0.0;
    }
    double S2 = 2 * (S11 * S11 + S22 * S22 + S33 * S33) + 4 * (S12 * S12 + S13 * S13 + S23 * S23);
    if (s->p.sgs_model == OC_SGS_DYNAMIC)   /* cs2(k) Delta^2 |S| (_dynamic_nut_body!), dyn_coefficients first */
        return s->cs2[k - s->p.hz] * pow(s->dx * s->dy * s->dz, 2.0 / 3.0) * sqrt(S2);
    if (s->p.sgs_model == OC_SGS_DYNAMIC_LOCAL || s->p.sgs_model == OC_SGS_LAGRANGIAN) {
        /* cs2(i, j, k): the clipped ratios left in dyn_lm, or the committed memory's */
        const oc_params* P = &s->p;
        size_t q = (size_t)(i - P->hx) + (size_t)P->nx * ((size_t)(j - P->hy) + (size_t)P->ny * (size_t)(k - P->hz));
        double c2 = P->sgs_model == OC_SGS_LAGRANGIAN ? s->lag_cs2[q] : s->dyn_lm[q];
        return c2 * pow(s->dx * s->dy * s->dz, 2.0 / 3.0) * sqrt(S2);
    }
    return coef * sqrt(S2);
}

/* eddy viscosity divergence (src/FiniteVolume.jl:969-1042, :1556-1562) */
static inline double eddy_u(const oc_sim* s, int i, int j, int k) {
    const double *u = s->u, *n = s->nut;
    double idx = s->idx, idy = s->idy;
    double fxE = A(n, i, j, k) * (A(u, i + 1, j, k) - A(u, i, j, k)) * idx;
    double fxW = A(n, i - 1, j, k) * (A(u, i, j, k) - A(u, i - 1, j, k)) * idx;
    double eN = 0.25 * (A(n, i - 1, j, k) + A(n, i, j, k) + A(n, i - 1, j + 1, k) + A(n, i, j + 1, k));
    double eS = 0.25 * (A(n, i - 1, j - 1, k) + A(n, i, j - 1, k) + A(n, i - 1, j, k) + A(n, i, j, k));
    double fyN = eN * (A(u, i, j + 1, k) - A(u, i, j, k)) * idy;
    double fyS = eS * (A(u, i, j, k) - A(u, i, j - 1, k)) * idy;
    double eT = 0.25 * (A(n, i - 1, j, k) + A(n, i, j, k) + A(n, i - 1, j, k + 1) + A(n, i, j, k + 1));
    double eB = 0.25 * (A(n, i - 1, j, k - 1) + A(n, i, j, k - 1) + A(n, i - 1, j, k) + A(n, i, j, k));
    double fzT = eT * (A(u, i, j, k + 1) - A(u, i, j, k)) * m_idzf(s, k + 1);
    double fzB = eB * (A(u, i, j, k) - A(u, i, j, k - 1)) * m_idzf(s, k);
    double vert = s->wc ? (s->wf[k + 1] * fzT - s->wf[k] * fzB) * m_idz(s, k) / s->wc[k] : (fzT - fzB) * m_idz(s, k);
    return (fxE - fxW) * idx + (fyN - fyS) * idy + vert;
}

static inline double eddy_v(const oc_sim* s, int i, int j, int k) {
    const double *v = s->v, *n = s->nut;
    double idx = s->idx, idy = s->idy;
    double fyN = A(n, i, j, k) * (A(v, i, j + 1, k) - A(v, i, j, k)) * idy;
    double fyS = A(n, i, j - 1, k) * (A(v, i, j, k) - A(v, i, j - 1, k)) * idy;
    double eE = 0.25 * (A(n, i, j - 1, k) + A(n, i + 1, j - 1, k) + A(n, i, j, k) + A(n, i + 1, j, k));
    double eW = 0.25 * (A(n, i - 1, j - 1, k) + A(n, i, j - 1, k) + A(n, i - 1, j, k) + A(n, i, j, k));
    double fxE = eE * (A(v, i + 1, j, k) - A(v, i, j, k)) * idx;
    double fxW = eW * (A(v, i, j, k) - A(v, i - 1, j, k)) * idx;
    double eT = 0.25 * (A(n, i, j - 1, k) + A(n, i, j, k) + A(n, i, j - 1, k + 1) + A(n, i, j, k + 1));
    double eB = 0.25 * (A(n, i, j - 1, k - 1) + A(n, i, j, k - 1) + A(n, i, j - 1, k) + A(n, i, j, k));
    double fzT = eT * (A(v, i, j, k + 1) - A(v, i, j, k)) * m_idzf(s, k + 1);
    double fzB = eB * (A(v, i, j, k) - A(v, i, j, k - 1)) * m_idzf(s, k);
    double vert = s->wc ? (s->wf[k + 1] * fzT - s->wf[k] * fzB) * m_idz(s, k) / s->wc[k] : (fzT - fzB) * m_idz(s, k);
    return (fxE - fxW) * idx + (fyN - fyS) * idy + vert;
}

static inline double eddy_w(const oc_sim* s, int i, int j, int k) {
    const double *w = s->w, *n = s->nut;
    double idx = s->idx, idy = s->idy;
    double fzT = A(n, i, j, k) * (A(w, i, j, k + 1) - A(w, i, j, k)) * m_idz(s, k);
    double fzB = A(n, i, j, k - 1) * (A(w, i, j, k) - A(w, i, j, k - 1)) * m_idz(s, k - 1);
    double eE = 0.25 * (A(n, i, j, k - 1) + A(n, i + 1, j, k - 1) + A(n, i, j, k) + A(n, i + 1, j, k));
    double eW = 0.25 * (A(n, i - 1, j, k - 1) + A(n, i, j, k - 1) + A(n, i - 1, j, k) + A(n, i, j, k));
    double fxE = eE * (A(w, i + 1, j, k) - A(w, i, j, k)) * idx;
    double fxW = eW * (A(w, i, j, k) - A(w, i - 1, j, k)) * idx;
    double eN = 0.25 * (A(n, i, j, k - 1) + A(n, i, j + 1, k - 1) + A(n, i, j, k) + A(n, i, j + 1, k));
    double eS = 0.25 * (A(n, i, j - 1, k - 1) + A(n, i, j, k - 1) + A(n, i, j - 1, k) + A(n, i, j, k));
    double fyN = eN * (A(w, i, j + 1, k) - A(w, i, j, k)) * idy;
    double fyS = eS * (A(w, i, j, k) - A(w, i, j - 1, k)) * idy;
    double vert = s->wc ? (s->wc[k] * fzT - s->wc[k - 1] * fzB) * m_idzf(s, k) / s->wf[k] : (fzT - fzB) * m_idzf(s, k);
    return (fxE - fxW) * idx + (fyN - fyS) * idy + vert;
}

/* scalar eddy diffusion: Boussinesq s*(div K grad) with K = nut, s = 1/Prt
 * (src/FiniteVolume.jl:1280-1300); sound-proof W-weighted form with
 * K = nut/Prt (src/FiniteVolume.jl:1473-1492). */
static inline double eddy_scalar(const oc_sim* s, const double* d, int i, int j, int k) {
    double idx = s->idx, idy = s->idy;
    if (!s->wc) {
        /* the AMD closure: its own kappa_t, unscaled (AMDClosure,
         * src/operators/sgs_amd_vreman.jl:325-354) */
        const int amd = s->p.sgs_model == OC_SGS_AMD || s->p.sgs_model == OC_SGS_TKE;
        const double* H = amd ? s->kt : s->nut;
        double sc = amd ? 1.0 : 1 / s->p.pr_t;
        double nE = 0.5 * (A(H, i, j, k) + A(H, i + 1, j, k));
        double nW = 0.5 * (A(H, i - 1, j, k) + A(H, i, j, k));
        double nN = 0.5 * (A(H, i, j, k) + A(H, i, j + 1, k));
        double nS = 0.5 * (A(H, i, j - 1, k) + A(H, i, j, k));
        double nT = 0.5 * (A(H, i, j, k) + A(H, i, j, k + 1));
        double nB = 0.5 * (A(H, i, j, k - 1) + A(H, i, j, k));
        double fxE = nE * (A(d, i + 1, j, k) - A(d, i, j, k)) * idx;
        double fxW = nW * (A(d, i, j, k) - A(d, i - 1, j, k)) * idx;
        double fyN = nN * (A(d, i, j + 1, k) - A(d, i, j, k)) * idy;
        double fyS = nS * (A(d, i, j, k) - A(d, i, j - 1, k)) * idy;
        double fzT = nT * (A(d, i, j, k + 1) - A(d, i, j, k)) * m_idzf(s, k + 1);
        double fzB = nB * (A(d, i, j, k) - A(d, i, j, k - 1)) * m_idzf(s, k);
        return sc * ((fxE - fxW) * idx + (fyN - fyS) * idy + (fzT - fzB) * m_idz(s, k));
    }
    const double* K = s->kt;
    double fxE = 0.5 * (A(K, i, j, k) + A(K, i + 1, j, k)) * (A(d, i + 1, j, k) - A(d, i, j, k)) * idx;
    double fxW = 0.5 * (A(K, i - 1, j, k) + A(K, i, j, k)) * (A(d, i, j, k) - A(d, i - 1, j, k)) * idx;
    double fyN = 0.5 * (A(K, i, j, k) + A(K, i, j + 1, k)) * (A(d, i, j + 1, k) - A(d, i, j, k)) * idy;
    double fyS = 0.5 * (A(K, i, j - 1, k) + A(K, i, j, k)) * (A(d, i, j, k) - A(d, i, j - 1, k)) * idy;
    double fzT = 0.5 * (A(K, i, j, k) + A(K, i, j, k + 1)) * (A(d, i, j, k + 1) - A(d, i, j, k)) * m_idzf(s, k + 1);
    double fzB = 0.5 * (A(K, i, j, k - 1) + A(K, i, j, k)) * (A(d, i, j, k) - A(d, i, j, k - 1)) * m_idzf(s, k);
    double vert = (s->wf[k + 1] * fzT - s->wf[k] * fzB) * m_idz(s, k) / s->wc[k];
    return (fxE - fxW) * idx + (fyN - fyS) * idy + vert;
}

/* Rayleigh sponge rate (src/FiniteVolume.jl:578-592, :664-702) */
static inline double sponge_rate(const oc_sim* s, double z) {
    double zs = s->p.sponge_zstart, ztop = s->p.z0 + s->p.lz;
    if (!(z >= zs)) return 0.0;
    double inv = 1 / (ztop - zs);
    double sn = sin(0.5 * M_PI * (z - zs) * inv);
    return s->p.sponge_alpha * sn * sn;
}

/* ------------------------------------------------------------------------- */
/* Tendencies of one substage (src/Simulations.jl:548-620,                    */
/* src/Anelastic.jl:1809-1849)                                                */
/* ------------------------------------------------------------------------- */

static void compute_tendencies(oc_sim* s) {
    const oc_params* P = &s->p;
    int Hx = P->hx, Hy = P->hy, Hz = P->hz, Nx = P->nx, Ny = P->ny, Nz = P->nz;
    int anel = (P->core == OC_CORE_ANELASTIC);
    int sc = P->advection;
    int has_visc = P->nu != 0, has_sgs = P->c_s != 0;
    int has_buoy = anel ? (P->g != 0) : (P->theta0 != 0);
    const double *u = s->u, *v = s->v, *w = s->w, *th = s->th;

    /* 4a. Smagorinsky coefficients, then their halos (velocity BCs) */
    if (has_sgs && (P->sgs_model == OC_SGS_DYNAMIC || P->sgs_model == OC_SGS_DYNAMIC_LOCAL)) dyn_coefficients(s);
    if (has_sgs) {
#pragma omp parallel for collapse(2) schedule(static)
        for (int k = Hz; k < Hz + Nz; ++k)
            for (int j = Hy; j < Hy + Ny; ++j)
                for (int i = Hx; i < Hx + Nx; ++i) {
                    if (P->sgs_model == OC_SGS_AMD) amd_at(s, i, j, k, &A(s->nut, i, j, k), &A(s->kt, i, j, k));
                    else if (P->sgs_model == OC_SGS_TKE) tke_at(s, i, j, k, &A(s->nut, i, j, k), &A(s->kt, i, j, k));
                    else A(s->nut, i, j, k) = smag_at(s, i, j, k);
                }
        fill_halos(s, s->nut, LOC_C);
        if (P->sgs_model == OC_SGS_AMD || P->sgs_model == OC_SGS_TKE) fill_halos(s, s->kt, LOC_C);
        if (anel && P->sgs_model != OC_SGS_AMD && P->sgs_model != OC_SGS_TKE)   /* AMD and TKE keep their own kappa_t */
            for (int64_t q = 0; q < s->n; ++q) s->kt[q] = s->nut[q] / P->pr_t;
    }

#pragma omp parallel for collapse(2) schedule(static)
    for (int k = Hz; k < Hz + Nz; ++k)
        for (int j = Hy; j < Hy + Ny; ++j)
            for (int i = Hx; i < Hx + Nx; ++i) {
                double tu, tv, tw, tt;
                /* 2. advection (the tendencies start from zero) */
                if (anel) {
                    tu = 0.0 - wmom_u(s, u, v, w, i, j, k);
                    tv = 0.0 - wmom_v(s, u, v, w, i, j, k);
                    tw = 0.0 - wmom_w(s, u, v, w, i, j, k);
                    tt = 0.0 - wscal(s, u, v, w, th, i, j, k);
                } else if (sc == OC_ADV_CENTRED) {
                    tu = 0.0 - mom_u_at(s, u, v, w, i, j, k);
                    tv = 0.0 - mom_v_at(s, u, v, w, i, j, k);
                    tw = 0.0 - mom_w_at(s, u, v, w, i, j, k);
                    tt = 0.0 - adv_centred_at(s, u, v, w, th, i, j, k);
                } else {
                    tu = 0.0 - recon_mom_u(s, sc, u, v, w, i, j, k);
                    tv = 0.0 - recon_mom_v(s, sc, u, v, w, i, j, k);
                    tw = 0.0 - recon_mom_w(s, sc, u, v, w, i, j, k);
                    tt = 0.0 - recon_scalar_at(s, sc, u, v, w, th, i, j, k);
                }
                /* 3. molecular viscosity / diffusion */
                if (has_visc) {
                    tu = tu + P->nu * lap_at(s, u, i, j, k, LOC_FX);
                    tv = tv + P->nu * lap_at(s, v, i, j, k, LOC_FY);
                    tw = tw + P->nu * lap_at(s, w, i, j, k, LOC_FZ);
                    tt = tt + P->nu * lap_at(s, th, i, j, k, LOC_C);
                }
                /* 4b. SGS tendencies */
                if (has_sgs) {
                    tu += eddy_u(s, i, j, k);
                    tv += eddy_v(s, i, j, k);
                    tw += eddy_w(s, i, j, k);
                    tt += eddy_scalar(s, th, i, j, k);
                }
                /* 5. buoyancy on the z faces */
                if (has_buoy) {
                    if (anel) {
                        double tb = s->thf[k];
                        double coef = P->g / tb;
                        double thface = m_zface(s, k, A(th, i, j, k - 1), A(th, i, j, k));
                        tw += coef * (thface - tb);
                    } else {
                        double thface = m_zface(s, k, A(th, i, j, k - 1), A(th, i, j, k));
                        tw += (P->g / P->theta0) * (thface - P->theta0);
                    }
                }
                /* 6. Coriolis */
                if (P->f_coriolis != 0) {
                    double v_at_u = 0.25 * (A(v, i - 1, j, k) + A(v, i, j, k) + A(v, i - 1, j + 1, k) + A(v, i, j + 1, k));
                    tu += P->f_coriolis * v_at_u;
                    double u_at_v = 0.25 * (A(u, i, j - 1, k) + A(u, i + 1, j - 1, k) + A(u, i, j, k) + A(u, i + 1, j, k));
                    tv -= P->f_coriolis * u_at_v;
                }
                /* 6a. prescribed wall fluxes of theta */
                if (k == Hz) tt += P->flux_bot * m_idz(s, Hz);
                if (k == Hz + Nz - 1) tt -= P->flux_top * m_idz(s, Hz + Nz - 1);
                /* 6b. Rayleigh sponge toward rest */
                if (P->sponge_alpha != 0) {
                    double zcen = s->zc[k], zface = s->zf[k];
                    double rc = sponge_rate(s, zcen), rf = sponge_rate(s, zface);
                    if (zcen >= P->sponge_zstart) { tu -= rc * (A(u, i, j, k) - 0.0); tv -= rc * (A(v, i, j, k) - 0.0); }
                    if (zface >= P->sponge_zstart) tw -= rf * (A(w, i, j, k) - 0.0);
                }
                A(s->tu, i, j, k) = tu;
                A(s->tv, i, j, k) = tv;
                A(s->tw, i, j, k) = tw;
                A(s->tt, i, j, k) = tt;
            }
}

int oc_tendencies(oc_sim* s, double* tu, double* tv, double* tw, double* tt) {
    oc_fill_state_halos(s);
    compute_tendencies(s);
    size_t b = sizeof(double) * (size_t)s->n;
    if (tu) memcpy(tu, s->tu, b);
    if (tv) memcpy(tv, s->tv, b);
    if (tw) memcpy(tw, s->tw, b);
    if (tt) memcpy(tt, s->tt, b);
    return 0;
}

/* ------------------------------------------------------------------------- */
/* Divergence (src/FiniteVolume.jl:312-316, :1869-1888;                       */
/* src/Anelastic.jl:1110-1120)                                                */
/* ------------------------------------------------------------------------- */

static inline double div_at(const oc_sim* s, const double* u, const double* v, const double* w, int i, int j, int k) {
    return (A(u, i + 1, j, k) - A(u, i, j, k)) * s->idx + (A(v, i, j + 1, k) - A(v, i, j, k)) * s->idy +
           (A(w, i, j, k + 1) - A(w, i, j, k)) * m_idz(s, k);
}
static inline double wdiv_at(const oc_sim* s, const double* u, const double* v, const double* w, int i, int j, int k) {
    double wc = s->wc[k], wfb = s->wf[k], wft = s->wf[k + 1];
    return wc * ((A(u, i + 1, j, k) - A(u, i, j, k)) * s->idx + (A(v, i, j + 1, k) - A(v, i, j, k)) * s->idy) +
           (wft * A(w, i, j, k + 1) - wfb * A(w, i, j, k)) * m_idz(s, k);
}

/* ------------------------------------------------------------------------- */
/* Pressure solvers                                                           */
/* ------------------------------------------------------------------------- */

/* Forward x-y transform of s->src into s->hat (rfft in x, DFT in y). */
static void xy_forward(oc_sim* s) {
    int Nx = s->p.nx, Ny = s->p.ny, Nz = s->p.nz, Mh = Nx / 2 + 1;
#pragma omp parallel
    {
        int nmax = (Nx > Ny ? Nx : Ny) + 2;
        cpx* z = (cpx*)malloc(sizeof(cpx) * (size_t)nmax);
        cpx* tmp = (cpx*)malloc(sizeof(cpx) * (size_t)nmax);
        cpx* col = (cpx*)malloc(sizeof(cpx) * (size_t)nmax);
#pragma omp for collapse(2) schedule(static)
        for (int k = 0; k < Nz; ++k)
            for (int j = 0; j < Ny; ++j)
                rfft_row(s, s->src + (int64_t)Nx * (j + (int64_t)Ny * k), s->hat + (int64_t)Mh * (j + (int64_t)Ny * k), z, tmp);
#pragma omp for collapse(2) schedule(static)
        for (int k = 0; k < Nz; ++k)
            for (int p = 0; p < Mh; ++p) {
                for (int j = 0; j < Ny; ++j) col[j] = s->hat[p + (int64_t)Mh * (j + (int64_t)Ny * k)];
                fft_c(&s->py, col, 0, tmp);
                for (int j = 0; j < Ny; ++j) s->hat[p + (int64_t)Mh * (j + (int64_t)Ny * k)] = col[j];
            }
        free(z); free(tmp); free(col);
    }
}

static void xy_inverse(oc_sim* s) {
    int Nx = s->p.nx, Ny = s->p.ny, Nz = s->p.nz, Mh = Nx / 2 + 1;
#pragma omp parallel
    {
        int nmax = (Nx > Ny ? Nx : Ny) + 2;
        cpx* z = (cpx*)malloc(sizeof(cpx) * (size_t)nmax);
        cpx* tmp = (cpx*)malloc(sizeof(cpx) * (size_t)nmax);
        cpx* col = (cpx*)malloc(sizeof(cpx) * (size_t)nmax);
#pragma omp for collapse(2) schedule(static)
        for (int k = 0; k < Nz; ++k)
            for (int p = 0; p < Mh; ++p) {
                for (int j = 0; j < Ny; ++j) col[j] = s->hat[p + (int64_t)Mh * (j + (int64_t)Ny * k)];
                fft_c(&s->py, col, 1, tmp);
                for (int j = 0; j < Ny; ++j) s->hat[p + (int64_t)Mh * (j + (int64_t)Ny * k)] = col[j];
            }
#pragma omp for collapse(2) schedule(static)
        for (int k = 0; k < Nz; ++k)
            for (int j = 0; j < Ny; ++j)
                irfft_row(s, s->hat + (int64_t)Mh * (j + (int64_t)Ny * k), s->src + (int64_t)Nx * (j + (int64_t)Ny * k), z, tmp);
        free(z); free(tmp); free(col);
    }
}

/* FFTPoissonSolver (src/PressureSolvers.jl:103-174): forward x-y then z,
 * scale by nrm/lambda (zero for the mean mode), inverse z then x-y. */
static void solve_fft(oc_sim* s) {
    int Nx = s->p.nx, Ny = s->p.ny, Nz = s->p.nz, Mh = Nx / 2 + 1;
    double nrm = 1 / (double)((int64_t)Nx * Ny * Nz);
    xy_forward(s);
#pragma omp parallel
    {
        cpx* tmp = (cpx*)malloc(sizeof(cpx) * (size_t)(Nz + 1));
        cpx* col = (cpx*)malloc(sizeof(cpx) * (size_t)(Nz + 1));
#pragma omp for collapse(2) schedule(static)
        for (int j = 0; j < Ny; ++j)
            for (int p = 0; p < Mh; ++p) {
                for (int k = 0; k < Nz; ++k) col[k] = s->hat[p + (int64_t)Mh * (j + (int64_t)Ny * k)];
                fft_c(&s->pz, col, 0, tmp);
                for (int k = 0; k < Nz; ++k) {
                    double lam = -(s->kx2[p] + s->ky2[j] + s->kz2[k]);
                    double il = lam == 0 ? 0.0 : nrm / lam;
                    col[k].re = col[k].re * il;
                    col[k].im = col[k].im * il;
                }
                fft_c(&s->pz, col, 1, tmp);
                for (int k = 0; k < Nz; ++k) s->hat[p + (int64_t)Mh * (j + (int64_t)Ny * k)] = col[k];
            }
        free(tmp); free(col);
    }
    xy_inverse(s);
}

/* ColumnTridiagonalSolver (src/PressureSolvers.jl:591-805): x-y transform,
 * Thomas per horizontal wavenumber with the factorisation of :650-661,
 * the mean mode integrated (_mean_mode!, :780-805), inverse, x norm. */
static void solve_column(oc_sim* s) {
    int Nx = s->p.nx, Ny = s->p.ny, Nz = s->p.nz, Mh = Nx / 2 + 1;
    double norm = 1.0 / (double)(1 * Nx * 1 * Ny);
    xy_forward(s);
    const double *lo = s->lower, *up = s->upper, *hw = s->hw;
#pragma omp parallel
    {
        double* cp = (double*)malloc(sizeof(double) * (size_t)Nz);
        double* id = (double*)malloc(sizeof(double) * (size_t)Nz);
#pragma omp for collapse(2) schedule(static)
        for (int q = 0; q < Ny; ++q)
            for (int p = 0; p < Mh; ++p) {
                if (p == 0 && q == 0) continue;
                double lam = s->kx2[p] + s->ky2[q];
                double cprev = 0.0;
                for (int k = 0; k < Nz; ++k) {
                    double b = -(lo[k] + up[k]) - lam * hw[k];
                    double den = b - lo[k] * cprev;
                    id[k] = 1 / den;
                    cprev = up[k] / den;
                    cp[k] = cprev;
                }
                cpx* c0 = s->hat + p + (int64_t)Mh * q;
                int64_t st = (int64_t)Mh * Ny;
                c0[0].re *= id[0];
                c0[0].im *= id[0];
                for (int k = 1; k < Nz; ++k) {
                    double a = lo[k];
                    c0[k * st].re = (c0[k * st].re - a * c0[(k - 1) * st].re) * id[k];
                    c0[k * st].im = (c0[k * st].im - a * c0[(k - 1) * st].im) * id[k];
                }
                for (int k = Nz - 2; k >= 0; --k) {
                    c0[k * st].re -= cp[k] * c0[(k + 1) * st].re;
                    c0[k * st].im -= cp[k] * c0[(k + 1) * st].im;
                }
            }
        free(cp); free(id);
    }
    /* the mean mode (real) */
    {
        int64_t st = (int64_t)Mh * Ny;
        double* col = (double*)malloc(sizeof(double) * (size_t)Nz);
        for (int k = 0; k < Nz; ++k) col[k] = s->hat[k * st].re;
        double mb = 0.0;
        for (int k = 0; k < Nz; ++k) mb += col[k] * s->meas[k];
        mb /= s->meas_sum;
        double F = 0.0, ph = 0.0, prev = col[0] - mb;
        col[0] = 0.0;
        for (int k = 1; k < Nz; ++k) {
            F += prev * s->meas[k - 1];
            ph += F * s->iota[k];
            prev = col[k] - mb;
            col[k] = ph;
        }
        double mp = 0.0;
        for (int k = 0; k < Nz; ++k) mp += col[k] * s->gauge[k];
        double sh = mp / s->gauge_sum;
        for (int k = 0; k < Nz; ++k) { s->hat[k * st].re = col[k] - sh; s->hat[k * st].im = 0.0; }
        free(col);
    }
    xy_inverse(s);
    int64_t nin = (int64_t)Nx * Ny * Nz;
    for (int64_t q = 0; q < nin; ++q) s->src[q] *= norm;
}

static void solve_src(oc_sim* s) {
    if (s->p.solver == OC_SOLVER_FFT) solve_fft(s);
    else solve_column(s);
}

int oc_pressure_solve(oc_sim* s, const double* src, double* phi) {
    int64_t nin = (int64_t)s->p.nx * s->p.ny * s->p.nz;
    memcpy(s->src, src, sizeof(double) * (size_t)nin);
    solve_src(s);
    memcpy(phi, s->src, sizeof(double) * (size_t)nin);
    return 0;
}

/* The operator each solver inverts, on interior-sized arrays (periodic x, y;
 * z periodic 7-point or the column coefficients with zero end fluxes). */
int oc_apply_poisson_operator(oc_sim* s, const double* phi, double* out) {
    int Nx = s->p.nx, Ny = s->p.ny, Nz = s->p.nz;
#define PI3(i, j, k) phi[(int64_t)(i) + (int64_t)Nx * ((int64_t)(j) + (int64_t)Ny * (int64_t)(k))]
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < Nz; ++k)
        for (int j = 0; j < Ny; ++j)
            for (int i = 0; i < Nx; ++i) {
                int ip = (i + 1) % Nx, im = (i + Nx - 1) % Nx, jp = (j + 1) % Ny, jm = (j + Ny - 1) % Ny;
                double c = PI3(i, j, k);
                double h = (PI3(ip, j, k) - 2 * c + PI3(im, j, k)) * s->idx2 + (PI3(i, jp, k) - 2 * c + PI3(i, jm, k)) * s->idy2;
                double r;
                if (s->p.solver == OC_SOLVER_FFT) {
                    int kp = (k + 1) % Nz, km = (k + Nz - 1) % Nz;
                    r = h + (PI3(i, j, kp) - 2 * c + PI3(i, j, km)) * s->idz2;
                } else {
                    r = s->hw[k] * h;
                    if (k > 0) r += s->lower[k] * (PI3(i, j, k - 1) - c);
                    if (k < Nz - 1) r += s->upper[k] * (PI3(i, j, k + 1) - c);
                }
                out[(int64_t)i + (int64_t)Nx * (j + (int64_t)Ny * k)] = r;
            }
#undef PI3
    return 0;
}

/* ------------------------------------------------------------------------- */
/* One projected substage (src/Simulations.jl:531-650, :711-744)              */
/* ------------------------------------------------------------------------- */

/* stage: 0 plain Euler; otherwise c(x, snap) = ca*snap + cb*x */
/* The cut-cell projection (solver = PCG; src/CutCell.jl:602-700, 852-880):
 * b = sum over the faces of (+-) a u* / h (u* in the storage arrays, halos
 * filled), phi = A^-1 b by MGPreconditionedCG with the a^2 face coefficients
 * (src/Multigrid.jl:893-967) into cgx.  On the sound-proof core the flux
 * carries the density weights of DensityWeightedPoissonSolver
 * (src/Anelastic.jl:734-793: W_c on x and y faces, W_f on z faces), and on a
 * stretched column the z-difference is over dz_c; the equation of cell k is
 * taken times dz_c[k] / h_z (the symmetric form of the operator built in
 * oc_set_apertures), h_z = L_z / N_z. */
static void cc_solve(oc_sim* s) {
    const oc_params* P = &s->p;
    int Hx = P->hx, Hy = P->hy, Hz = P->hz, Nx = P->nx, Ny = P->ny, Nz = P->nz;
    int64_t pl = (int64_t)Nx * Ny;
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < Nz; ++k)
        for (int j = 0; j < Ny; ++j)
            for (int i = 0; i < Nx; ++i) {
                int64_t qi = i + (int64_t)Nx * (j + (int64_t)Ny * k);
                int64_t xr = (int64_t)(Nx + 1) * (j + (int64_t)Ny * k), yr = (int64_t)Nx * (j + (int64_t)(Ny + 1) * k);
                int I = i + Hx, J = j + Hy, K = k + Hz;
                double aw = s->apx[xr + i], ae = s->apx[xr + i + 1];
                double as = s->apy[yr + i], an = s->apy[yr + Nx + i];
                double ab = s->apz[qi], at = s->apz[qi + pl];
                if (P->core != OC_CORE_ANELASTIC && s->uniform) {
                    s->src[qi] = (ae * A(s->u, I + 1, J, K) - aw * A(s->u, I, J, K)) * s->idx +
                                 (an * A(s->v, I, J + 1, K) - as * A(s->v, I, J, K)) * s->idy +
                                 (at * A(s->w, I, J, K + 1) - ab * A(s->w, I, J, K)) * s->idz;
                } else {
                    double wcc = P->core == OC_CORE_ANELASTIC ? s->wc[K] : 1.0;
                    double wfb = P->core == OC_CORE_ANELASTIC ? s->wf[K] : 1.0;
                    double wft = P->core == OC_CORE_ANELASTIC ? s->wf[K + 1] : 1.0;
                    double sc = s->uniform ? 1.0 : s->dzc[K] / s->dz;
                    s->src[qi] = wcc * sc * ((ae * A(s->u, I + 1, J, K) - aw * A(s->u, I, J, K)) * s->idx +
                                             (an * A(s->v, I, J + 1, K) - as * A(s->v, I, J, K)) * s->idy) +
                                 (wft * (at * A(s->w, I, J, K + 1)) - wfb * (ab * A(s->w, I, J, K))) / s->dz;
                }
            }
    ocg_solve(s->cg, s->src, s->cgx, &s->cg_st);
}

/* u = c(u* - a d(phi), u^n) on every face (0 on a blocked one), theta =
 * c(theta + dt t_theta, theta^n) (with_theta), p = phi/dt; c(x, s) = ca s + cb x
 * in stages 2 and 3. */
static void cc_correct(oc_sim* s, double dt, int stage, double ca, double cb, int with_theta) {
    const oc_params* P = &s->p;
    int Hx = P->hx, Hy = P->hy, Hz = P->hz, Nx = P->nx, Ny = P->ny, Nz = P->nz;
    int64_t pl = (int64_t)Nx * Ny;
    const double* phi = s->cgx;
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < Nz; ++k)
        for (int j = 0; j < Ny; ++j)
            for (int i = 0; i < Nx; ++i) {
                int64_t qi = i + (int64_t)Nx * (j + (int64_t)Ny * k);
                int64_t q = ID(s, i + Hx, j + Hy, k + Hz);
                double pc = phi[qi];
                /* phi's halo is the mirror on an open face (d phi / dn = 0) */
                double pw = i > 0 ? phi[qi - 1] : (s->open_x ? pc : phi[qi + Nx - 1]);
                double ps = j > 0 ? phi[qi - Nx] : (s->open_y ? pc : phi[qi + (int64_t)(Ny - 1) * Nx]);
                double pb = phi[k > 0 ? qi - pl : (P->bc_z == OC_BC_PERIODIC ? qi + (int64_t)(Nz - 1) * pl : qi)];
                double aw = s->apx[(int64_t)(Nx + 1) * (j + (int64_t)Ny * k) + i];
                double as = s->apy[(int64_t)Nx * (j + (int64_t)(Ny + 1) * k) + i];
                double ab = s->apz[qi];
                double un = aw > 0 ? s->u[q] - aw * ((pc - pw) * s->idx) : 0.0;
                double vn = as > 0 ? s->v[q] - as * ((pc - ps) * s->idy) : 0.0;
                double wn = ab > 0 ? s->w[q] - ab * ((pc - pb) * m_idzf(s, k + Hz)) : 0.0;
                double tn = with_theta ? s->th[q] + dt * s->tt[q] : s->th[q];
                if (stage) {
                    un = ca * s->u0[q] + cb * un;
                    vn = ca * s->v0[q] + cb * vn;
                    wn = ca * s->w0[q] + cb * wn;
                    tn = ca * s->th0[q] + cb * tn;
                }
                s->u[q] = un; s->v[q] = vn; s->w[q] = wn; s->th[q] = tn;
                s->pr[q] = pc / dt;
            }
}

/* implicit_ibm_correction! (src/IBM.jl:295-300) as the post-predictor hook
 * (src/Simulations.jl:624-628): every face of a solid interior cell scaled by
 * 1/(1 + dt/tau) (0 for tau = 0), once per solid cell it touches.  The halo
 * fill that follows replaces the faces beyond the interior with periodic
 * images, so an interior face counts the solid cell on its high side and, for
 * all but the first face of a row, the one on its low side. */
static void ibm_correct(oc_sim* s, double dt) {
    const oc_params* P = &s->p;
    int Hx = P->hx, Hy = P->hy, Hz = P->hz, Nx = P->nx, Ny = P->ny, Nz = P->nz;
    const double f = s->ibm_tau > 0 ? 1 / (1 + dt / s->ibm_tau) : 0.0;
    const unsigned char* m = s->ibm;
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < Nz; ++k)
        for (int j = 0; j < Ny; ++j)
            for (int i = 0; i < Nx; ++i) {
                int64_t c = i + (int64_t)Nx * (j + (int64_t)Ny * k);
                int64_t q = ID(s, i + Hx, j + Hy, k + Hz);
                int nu = m[c] + (i > 0 ? m[c - 1] : 0);
                int nv = m[c] + (j > 0 ? m[c - Nx] : 0);
                int nw = m[c] + (k > 0 ? m[c - (int64_t)Nx * Ny] : 0);
                for (int r = 0; r < nu; ++r) s->u[q] *= f;
                for (int r = 0; r < nv; ++r) s->v[q] *= f;
                for (int r = 0; r < nw; ++r) s->w[q] *= f;
            }
}

int oc_set_ibm(oc_sim* s, const unsigned char* mask, double tau) {
    const oc_params* P = &s->p;
    if (!(tau >= 0) || P->solver == OC_SOLVER_PCG) return -1;
    free(s->ibm);
    s->ibm = NULL;
    if (!mask) return 0;
    int64_t nin = (int64_t)P->nx * P->ny * P->nz;
    s->ibm = (unsigned char*)malloc((size_t)nin);
    for (int k = 0; k < P->nz; ++k)
        for (int j = 0; j < P->ny; ++j)
            for (int i = 0; i < P->nx; ++i)
                s->ibm[i + (int64_t)P->nx * (j + (int64_t)P->ny * k)] =
                    mask[ID(s, i + P->hx, j + P->hy, k + P->hz)] ? 1 : 0;
    s->ibm_tau = tau;
    return 0;
}

static void substage(oc_sim* s, double dt, int stage, double ca, double cb) {
    const oc_params* P = &s->p;
    int Hx = P->hx, Hy = P->hy, Hz = P->hz, Nx = P->nx, Ny = P->ny, Nz = P->nz;
    int anel = P->core == OC_CORE_ANELASTIC;
    oc_fill_state_halos(s);
    if (ob_radiates(s)) ob_mark(s);          /* the stage-start layers, after the fill (src/Simulations.jl:537-538) */
    compute_tendencies(s);
    /* 7. predictor */
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = Hz; k < Hz + Nz; ++k)
        for (int j = Hy; j < Hy + Ny; ++j)
            for (int i = Hx; i < Hx + Nx; ++i) {
                int64_t q = ID(s, i, j, k);
                s->u[q] = s->u[q] + dt * s->tu[q];
                s->v[q] = s->v[q] + dt * s->tv[q];
                s->w[q] = s->w[q] + dt * s->tw[q];
            }
    if (s->ibm) ibm_correct(s, dt);
    ob_update(s, dt);                        /* 7c. open boundaries (src/Simulations.jl:630-633) */
    /* 8. divergence into the solver's buffer */
    fill_halos(s, s->u, LOC_FX);
    fill_halos(s, s->v, LOC_FY);
    fill_halos(s, s->w, LOC_FZ);
    if (P->solver == OC_SOLVER_PCG) {
        cc_solve(s);
        cc_correct(s, dt, stage, ca, cb, 1);
        return;
    }
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < Nz; ++k)
        for (int j = 0; j < Ny; ++j)
            for (int i = 0; i < Nx; ++i)
                s->src[(int64_t)i + (int64_t)Nx * (j + (int64_t)Ny * k)] =
                    anel ? wdiv_at(s, s->u, s->v, s->w, i + Hx, j + Hy, k + Hz)
                         : div_at(s, s->u, s->v, s->w, i + Hx, j + Hy, k + Hz);
    /* 9. Poisson solve */
    solve_src(s);
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < Nz; ++k)
        for (int j = 0; j < Ny; ++j)
            for (int i = 0; i < Nx; ++i)
                A(s->phi, i + Hx, j + Hy, k + Hz) = s->src[(int64_t)i + (int64_t)Nx * (j + (int64_t)Ny * k)];
    fill_halos(s, s->phi, LOC_C);
    /* 10. correction, p = phi/dt, RK combination; 11. theta */
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = Hz; k < Hz + Nz; ++k)
        for (int j = Hy; j < Hy + Ny; ++j)
            for (int i = Hx; i < Hx + Nx; ++i) {
                int64_t q = ID(s, i, j, k);
                double pc = s->phi[q];
                double un = s->u[q] - (pc - A(s->phi, i - 1, j, k)) * s->idx;
                double vn = s->v[q] - (pc - A(s->phi, i, j - 1, k)) * s->idy;
                double wn = s->w[q] - (pc - A(s->phi, i, j, k - 1)) * m_idzf(s, k);
                double tn = s->th[q] + dt * s->tt[q];
                if (stage) {
                    un = ca * s->u0[q] + cb * un;
                    vn = ca * s->v0[q] + cb * vn;
                    wn = ca * s->w0[q] + cb * wn;
                    tn = ca * s->th0[q] + cb * tn;
                }
                s->u[q] = un; s->v[q] = vn; s->w[q] = wn; s->th[q] = tn;
                s->pr[q] = pc / dt;
            }
}

/* The Chorin projection of the current velocity with dt = 1 (the config
 * driver's `_project!(sim, 1.0)` of a noisy initial field,
 * src/config/simulation_driver.jl:1316; steps 8-10 of src/Simulations.jl:711-744). */
int oc_project(oc_sim* s) {
    const oc_params* P = &s->p;
    int Hx = P->hx, Hy = P->hy, Hz = P->hz, Nx = P->nx, Ny = P->ny, Nz = P->nz;
    int anel = P->core == OC_CORE_ANELASTIC;
    fill_halos(s, s->u, LOC_FX);
    fill_halos(s, s->v, LOC_FY);
    fill_halos(s, s->w, LOC_FZ);
    if (P->solver == OC_SOLVER_PCG) {
        cc_solve(s);
        cc_correct(s, 1.0, 0, 0.0, 0.0, 0);
        return 0;
    }
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < Nz; ++k)
        for (int j = 0; j < Ny; ++j)
            for (int i = 0; i < Nx; ++i)
                s->src[(int64_t)i + (int64_t)Nx * (j + (int64_t)Ny * k)] =
                    anel ? wdiv_at(s, s->u, s->v, s->w, i + Hx, j + Hy, k + Hz)
                         : div_at(s, s->u, s->v, s->w, i + Hx, j + Hy, k + Hz);
    solve_src(s);
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < Nz; ++k)
        for (int j = 0; j < Ny; ++j)
            for (int i = 0; i < Nx; ++i)
                A(s->phi, i + Hx, j + Hy, k + Hz) = s->src[(int64_t)i + (int64_t)Nx * (j + (int64_t)Ny * k)];
    fill_halos(s, s->phi, LOC_C);
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = Hz; k < Hz + Nz; ++k)
        for (int j = Hy; j < Hy + Ny; ++j)
            for (int i = Hx; i < Hx + Nx; ++i) {
                int64_t q = ID(s, i, j, k);
                double pc = s->phi[q];
                s->u[q] = s->u[q] - (pc - A(s->phi, i - 1, j, k)) * s->idx;
                s->v[q] = s->v[q] - (pc - A(s->phi, i, j - 1, k)) * s->idy;
                s->w[q] = s->w[q] - (pc - A(s->phi, i, j, k - 1)) * m_idzf(s, k);
                s->pr[q] = pc;
            }
    return 0;
}

int oc_step_euler(oc_sim* s, double dt, int nsteps) {
    for (int n = 0; n < nsteps; ++n) {
        if (ob_radiates(s)) ob_prepare(s, dt);
        substage(s, dt, 0, 0.0, 0.0);
        if (s->p.c_s != 0 && s->p.sgs_model == OC_SGS_LAGRANGIAN) lag_commit(s, dt);   /* once per step */
        if (s->p.c_s != 0 && s->p.sgs_model == OC_SGS_TKE) tke_commit(s, dt);
    }
    return 0;
}

/* cfl_diagnostics + adaptive_dt (src/TimeIntegration.jl:164-185, :209-226,
 * :291-365, :436-454): the advective rate max_cell sum |u_i|/dx_i, the
 * diffusive (molecular + Smagorinsky) and SGS limits over the harmonic
 * spacing of the thinnest cell, the Brunt-Vaisala limit of the plane-mean
 * theta profile, the Coriolis limit; then the growth limit and the clamp.
 * limiter: 0 adv, 1 diff, 2 buoy, 3 cor, 4 sgs, 5 growth, 6 dt_min, 7 dt_max. */
double oc_adaptive_dt(oc_sim* s, const oc_cfl* c, double dt_prev, int* limiter) {
    const oc_params* P = &s->p;
    int Hx = P->hx, Hy = P->hy, Hz = P->hz, Nx = P->nx, Ny = P->ny, Nz = P->nz;
    int anel = P->core == OC_CORE_ANELASTIC;
    fill_halos(s, s->u, LOC_FX);
    fill_halos(s, s->v, LOC_FY);
    fill_halos(s, s->w, LOC_FZ);
    if (P->c_s != 0 && (P->sgs_model == OC_SGS_DYNAMIC || P->sgs_model == OC_SGS_DYNAMIC_LOCAL)) dyn_coefficients(s);
    if (P->c_s != 0 && P->sgs_model == OC_SGS_TKE) fill_halos(s, s->th, LOC_C);
    double rate = 0.0, nutm = 0.0, ktm = 0.0;
    int nanr = 0;
    double* mean = (double*)calloc((size_t)Nz, sizeof(double));
    for (int k = Hz; k < Hz + Nz; ++k) {
        double acc = 0.0;
        for (int j = Hy; j < Hy + Ny; ++j)
            for (int i = Hx; i < Hx + Nx; ++i) {
                double au = fmax(fabs(A(s->u, i, j, k)), fabs(A(s->u, i + 1, j, k)));
                double av = fmax(fabs(A(s->v, i, j, k)), fabs(A(s->v, i, j + 1, k)));
                double aw = fmax(fabs(A(s->w, i, j, k)), fabs(A(s->w, i, j, k + 1)));
                double r = au * s->idx + av * s->idy + aw * m_idz(s, k);
                if (isnan(r)) nanr = 1;
                else if (r > rate) rate = r;
                if (P->c_s != 0) {
                    double n, kk = 0.0;
                    if (P->sgs_model == OC_SGS_AMD) amd_at(s, i, j, k, &n, &kk);
                    else if (P->sgs_model == OC_SGS_TKE) tke_at(s, i, j, k, &n, &kk);
                    else n = smag_at(s, i, j, k);
                    if (n > nutm) nutm = n;
                    if (kk > ktm) ktm = kk;
                }
                acc += A(s->th, i, j, k);
            }
        mean[k - Hz] = acc / ((double)Nx * Ny);
    }
    const double INF = 1.0 / 0.0;
    if (nanr) rate = NAN;
    double dt_adv = isnan(rate) ? NAN : (rate > 0 ? c->c_adv / rate : INF);
    double dzmin = INF;
    for (int k = Hz; k < Hz + Nz; ++k) dzmin = fmin(dzmin, s->dzc[k]);
    double harm = 1.0 / (1 / (s->dx * s->dx) + 1 / (s->dy * s->dy) + 1 / (dzmin * dzmin));
    double nu_total = P->nu + nutm;
    double dt_diff = nu_total > 0 ? c->c_diff * harm / nu_total : INF;
    /* max(nu_t, kappa_t), kappa_t the AMD closure's own (src/TimeIntegration.jl:322-335) */
    double ksgs = fmax(nutm, P->c_s != 0 ? ((P->sgs_model == OC_SGS_AMD || P->sgs_model == OC_SGS_TKE) ? ktm : nutm / P->pr_t)
                                         : 0.0);
    double dt_sgs = ksgs > 0 ? c->c_diff * harm / ksgs : INF;
    int buoy = anel ? (P->g != 0) : (P->theta0 != 0);
    double n2max = 0.0;
    if (buoy)
        for (int k = 1; k < Nz; ++k) {
            double dzf = s->dzf[Hz + k];
            double n2 = anel ? P->g * (log(mean[k]) - log(mean[k - 1])) / dzf
                             : (P->g / P->theta0) * (mean[k] - mean[k - 1]) * (1 / dzf);
            n2max = fmax(n2max, n2);
        }
    free(mean);
    double N = sqrt(fmax(n2max, 0.0));
    double dt_buoy = N > 0 ? c->c_buoy / N : INF;
    double f = fabs(P->f_coriolis);
    double dt_cor = f > 0 ? c->c_cor / f : INF;
    double dt = dt_adv;
    int lim = 0;
    if (dt_diff < dt) { dt = dt_diff; lim = 1; }
    if (dt_buoy < dt) { dt = dt_buoy; lim = 2; }
    if (dt_cor < dt) { dt = dt_cor; lim = 3; }
    if (dt_sgs < dt) { dt = dt_sgs; lim = 4; }
    if (isnan(dt)) {
        dt = c->dt_min;
        lim = 6;
    } else {
        if (dt_prev > 0 && c->growth * dt_prev < dt) { dt = c->growth * dt_prev; lim = 5; }
        if (dt < c->dt_min) lim = 6;
        if (dt > c->dt_max) lim = 7;
        dt = fmin(fmax(dt, c->dt_min), c->dt_max);
    }
    if (limiter) *limiter = lim;
    return dt;
}

/* SSP-RK3 of three projected substages (src/Simulations.jl:854-912) */
int oc_step_rk3(oc_sim* s, double dt, int nsteps) {
    size_t b = sizeof(double) * (size_t)s->n;
    double inv3 = 1.0 / 3, two3 = 2 * inv3;
    for (int n = 0; n < nsteps; ++n) {
        if (ob_radiates(s)) ob_prepare(s, dt);
        memcpy(s->u0, s->u, b); memcpy(s->v0, s->v, b); memcpy(s->w0, s->w, b); memcpy(s->th0, s->th, b);
        substage(s, dt, 0, 0.0, 0.0);
        substage(s, dt, 1, 0.75, 0.25);
        ob_combine(s, 0.75, 0.25);
        substage(s, dt, 1, inv3, two3);
        ob_combine(s, inv3, two3);
        if (s->p.c_s != 0 && s->p.sgs_model == OC_SGS_LAGRANGIAN) lag_commit(s, dt);   /* once per step */
        if (s->p.c_s != 0 && s->p.sgs_model == OC_SGS_TKE) tke_commit(s, dt);
    }
    return 0;
}

/* nsteps of step_adaptive! without failures: the adaptive_dt pick, then
 * step_rk3!.  dts (nsteps entries, may be NULL) receives the dt sequence;
 * *dt_prev carries the growth limit in and the last dt out. */
int oc_step_adaptive(oc_sim* s, const oc_cfl* c, int nsteps, double* dt_prev, double* dts) {
    double dp = dt_prev ? *dt_prev : 0.0;
    for (int n = 0; n < nsteps; ++n) {
        double dt = oc_adaptive_dt(s, c, dp, NULL);
        oc_step_rk3(s, dt, 1);
        if (dts) dts[n] = dt;
        dp = dt;
    }
    if (dt_prev) *dt_prev = dp;
    return 0;
}

/* ------------------------------------------------------------------------- */
/* Diagnostics (src/Simulations.jl:992-1050)                                  */
/* ------------------------------------------------------------------------- */

/* ------------------------------------------------------------------------- */
/* Positivity-preserving scalar advection (advect_positive!,                   */
/* src/AdvectionSchemes.jl:1100-1160, the limiter :1015-1098)                  */
/* ------------------------------------------------------------------------- */

/* Adds (accumulate) or writes -div(u phi) to tend (storage arrays of the
 * domain's layout, halos of u, v, w and phi filled, halo >= 3): the
 * reconstructed face fluxes F = vel * face value (WENO-JS5 / WENO-Z5,
 * _reconstructed_fluxes! :868-892), the first-order upwind fluxes L
 * (_upwind_fluxes! :899-909), the antidiffusive outflow ratio of every cell
 * (_b_limit_ratio! :1015-1043), its one-layer periodic wrap
 * (_wrap_one_layer! :951-958, the default without boundary conditions), the
 * limited fluxes L + c (F - L) with c the donor's ratio (_b_limit_x/y/z!
 * :1045-1071) and their divergence (_b_flux_div! :911-926).  Uniform grids. */
int oc_advect_positive(oc_sim* s, const double* u, const double* v, const double* w, const double* phi,
                       double* tend, double dt, int scheme, int accumulate) {
    const oc_params* P = &s->p;
    if (!s->uniform || (scheme != OC_ADV_WENO_JS5 && scheme != OC_ADV_WENO_Z5)) return -1;
    if (P->hx < 3 || P->hy < 3 || P->hz < 3) return -1;
    int Hx = P->hx, Hy = P->hy, Hz = P->hz, Nx = P->nx, Ny = P->ny, Nz = P->nz;
    int64_t n = s->n;
    double *Fx = (double*)calloc((size_t)n, sizeof(double)), *Fy = (double*)calloc((size_t)n, sizeof(double));
    double *Fz = (double*)calloc((size_t)n, sizeof(double)), *Lx = (double*)calloc((size_t)n, sizeof(double));
    double *Ly = (double*)calloc((size_t)n, sizeof(double)), *Lz = (double*)calloc((size_t)n, sizeof(double));
    double* R = (double*)calloc((size_t)n, sizeof(double));
    /* face fluxes over the interior faces plus the closing face of each axis */
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = Hz; k <= Hz + Nz; ++k)
        for (int j = Hy; j <= Hy + Ny; ++j)
            for (int i = Hx; i <= Hx + Nx; ++i) {
                int64_t q = ID(s, i, j, k);
                if (j < Hy + Ny && k < Hz + Nz) {
                    double vel = u[q];
                    Fx[q] = vel * face_x(s, scheme, phi, i - 1, j, k, vel);
                    Lx[q] = vel * (vel >= 0 ? A(phi, i - 1, j, k) : phi[q]);
                }
                if (i < Hx + Nx && k < Hz + Nz) {
                    double vel = v[q];
                    Fy[q] = vel * face_y(s, scheme, phi, i, j - 1, k, vel);
                    Ly[q] = vel * (vel >= 0 ? A(phi, i, j - 1, k) : phi[q]);
                }
                if (i < Hx + Nx && j < Hy + Ny) {
                    double vel = w[q];
                    Fz[q] = vel * face_z(s, scheme, phi, i, j, k - 1, vel);
                    Lz[q] = vel * (vel >= 0 ? A(phi, i, j, k - 1) : phi[q]);
                }
            }
    const double z = 0.0, idx = s->idx, idy = s->idy, idz = s->idz;
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = Hz; k < Hz + Nz; ++k)
        for (int j = Hy; j < Hy + Ny; ++j)
            for (int i = Hx; i < Hx + Nx; ++i) {
                double lxe = A(Lx, i + 1, j, k), lxw = A(Lx, i, j, k);
                double lyn = A(Ly, i, j + 1, k), lys = A(Ly, i, j, k);
                double lzt = A(Lz, i, j, k + 1), lzb = A(Lz, i, j, k);
                double axe = A(Fx, i + 1, j, k) - lxe, axw = A(Fx, i, j, k) - lxw;
                double ayn = A(Fy, i, j + 1, k) - lyn, ays = A(Fy, i, j, k) - lys;
                double azt = A(Fz, i, j, k + 1) - lzt, azb = A(Fz, i, j, k) - lzb;
                double Pm = dt * ((fmax(axe, z) + fmax(-axw, z)) * idx + (fmax(ayn, z) + fmax(-ays, z)) * idy +
                                  (fmax(azt, z) + fmax(-azb, z)) * idz);
                double div_lo = (lxe - lxw) * idx + (lyn - lys) * idy + (lzt - lzb) * idz;
                double Q = fmax(A(phi, i, j, k) - dt * div_lo, z);
                A(R, i, j, k) = Pm > z ? fmin(1.0, Q / Pm) : 1.0;
            }
    /* one-layer periodic wrap of the ratio, x then y then z */
    for (int k = Hz; k < Hz + Nz; ++k)
        for (int j = Hy; j < Hy + Ny; ++j) {
            A(R, Hx - 1, j, k) = A(R, Hx + Nx - 1, j, k);
            A(R, Hx + Nx, j, k) = A(R, Hx, j, k);
        }
    for (int k = Hz; k < Hz + Nz; ++k)
        for (int i = Hx; i < Hx + Nx; ++i) {
            A(R, i, Hy - 1, k) = A(R, i, Hy + Ny - 1, k);
            A(R, i, Hy + Ny, k) = A(R, i, Hy, k);
        }
    for (int j = Hy; j < Hy + Ny; ++j)
        for (int i = Hx; i < Hx + Nx; ++i) {
            A(R, i, j, Hz - 1) = A(R, i, j, Hz + Nz - 1);
            A(R, i, j, Hz + Nz) = A(R, i, j, Hz);
        }
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = Hz; k <= Hz + Nz; ++k)
        for (int j = Hy; j <= Hy + Ny; ++j)
            for (int i = Hx; i <= Hx + Nx; ++i) {
                int64_t q = ID(s, i, j, k);
                if (j < Hy + Ny && k < Hz + Nz) {
                    double a = Fx[q] - Lx[q], c = a >= z ? A(R, i - 1, j, k) : R[q];
                    Fx[q] = Lx[q] + c * a;
                }
                if (i < Hx + Nx && k < Hz + Nz) {
                    double a = Fy[q] - Ly[q], c = a >= z ? A(R, i, j - 1, k) : R[q];
                    Fy[q] = Ly[q] + c * a;
                }
                if (i < Hx + Nx && j < Hy + Ny) {
                    double a = Fz[q] - Lz[q], c = a >= z ? A(R, i, j, k - 1) : R[q];
                    Fz[q] = Lz[q] + c * a;
                }
            }
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = Hz; k < Hz + Nz; ++k)
        for (int j = Hy; j < Hy + Ny; ++j)
            for (int i = Hx; i < Hx + Nx; ++i) {
                int64_t q = ID(s, i, j, k);
                double d = (A(Fx, i + 1, j, k) - Fx[q]) * idx + (A(Fy, i, j + 1, k) - Fy[q]) * idy +
                           (A(Fz, i, j, k + 1) - Fz[q]) * idz;
                tend[q] = accumulate ? tend[q] - d : -d;
            }
    free(Fx); free(Fy); free(Fz); free(Lx); free(Ly); free(Lz); free(R);
    return 0;
}

double oc_kinetic_energy(oc_sim* s) {
    const oc_params* P = &s->p;
    int Hx = P->hx, Hy = P->hy, Hz = P->hz, Nx = P->nx, Ny = P->ny, Nz = P->nz;
    double* part = (double*)calloc((size_t)Nz, sizeof(double));
#pragma omp parallel for schedule(static)
    for (int k = Hz; k < Hz + Nz; ++k) {
        double acc = 0.0;
        for (int j = Hy; j < Hy + Ny; ++j)
            for (int i = Hx; i < Hx + Nx; ++i) {
                double uu = A(s->u, i, j, k), vv = A(s->v, i, j, k), ww = A(s->w, i, j, k);
                if (s->uniform) acc += uu * uu + vv * vv + ww * ww;
                else acc += (uu * uu + vv * vv) * s->dzc[k] + ww * ww * s->dzf[k];
            }
        part[k - Hz] = acc;
    }
    double tot = 0.0;
    for (int k = 0; k < Nz; ++k) tot += part[k];
    free(part);
    if (s->uniform) return 0.5 * tot * (s->dx * s->dy * s->dz);
    return 0.5 * tot * s->dx * s->dy;
}

double oc_max_divergence(oc_sim* s) {
    const oc_params* P = &s->p;
    int Hx = P->hx, Hy = P->hy, Hz = P->hz, Nx = P->nx, Ny = P->ny, Nz = P->nz;
    fill_halos(s, s->u, LOC_FX);
    fill_halos(s, s->v, LOC_FY);
    fill_halos(s, s->w, LOC_FZ);
    double m = 0.0;
#pragma omp parallel for collapse(2) reduction(max : m) schedule(static)
    for (int k = Hz; k < Hz + Nz; ++k)
        for (int j = Hy; j < Hy + Ny; ++j)
            for (int i = Hx; i < Hx + Nx; ++i) {
                double d;
                if (P->solver == OC_SOLVER_PCG) {
                    int64_t qi = (i - Hx) + (int64_t)Nx * ((j - Hy) + (int64_t)Ny * (k - Hz));
                    int64_t xr = (int64_t)(Nx + 1) * ((j - Hy) + (int64_t)Ny * (k - Hz));
                    int64_t yr = (int64_t)Nx * ((j - Hy) + (int64_t)(Ny + 1) * (k - Hz));
                    double dw;
                    if (P->core == OC_CORE_ANELASTIC)
                        dw = (s->wf[k + 1] * (s->apz[qi + (int64_t)Nx * Ny] * A(s->w, i, j, k + 1)) -
                              s->wf[k] * (s->apz[qi] * A(s->w, i, j, k))) * m_idz(s, k) / s->wc[k];
                    else
                        dw = (s->apz[qi + (int64_t)Nx * Ny] * A(s->w, i, j, k + 1) - s->apz[qi] * A(s->w, i, j, k)) * m_idz(s, k);
                    d = (s->apx[xr + i - Hx + 1] * A(s->u, i + 1, j, k) - s->apx[xr + i - Hx] * A(s->u, i, j, k)) * s->idx +
                        (s->apy[yr + Nx + i - Hx] * A(s->v, i, j + 1, k) - s->apy[yr + i - Hx] * A(s->v, i, j, k)) * s->idy + dw;
                } else {
                    d = s->wc ? wdiv_at(s, s->u, s->v, s->w, i, j, k) / s->wc[k] : div_at(s, s->u, s->v, s->w, i, j, k);
                }
                d = fabs(d);
                if (d > m) m = d;
            }
    return m;
}

/* ------------------------------------------------------------------------- */
/* Construction                                                               */
/* ------------------------------------------------------------------------- */

static double* dalloc(int64_t n) { return (double*)calloc((size_t)(n > 0 ? n : 1), sizeof(double)); }

oc_sim* oc_create(const oc_params* p, const double* zfi, const double* wc, const double* wf, const double* thf) {
    if (p->bc_x != OC_BC_PERIODIC || p->bc_y != OC_BC_PERIODIC) return NULL;
    if (p->nx % 2 != 0) return NULL;
    int H = p->hx;
    if (p->advection != OC_ADV_CENTRED && (H < 3 || p->hy < 3 || p->hz < 3)) return NULL;
    if (p->advection != OC_ADV_CENTRED && (p->stretched || p->core == OC_CORE_ANELASTIC)) return NULL;
    if (p->core == OC_CORE_ANELASTIC && (!wc || !wf || p->bc_z != OC_BC_WALL)) return NULL;
    if (p->solver == OC_SOLVER_FFT && p->bc_z != OC_BC_PERIODIC) return NULL;
    if (p->solver == OC_SOLVER_COLUMN && p->bc_z != OC_BC_WALL) return NULL;
    if (p->stretched && (!zfi || p->bc_z != OC_BC_WALL)) return NULL;
    if ((p->sgs_model == OC_SGS_VREMAN || p->sgs_model == OC_SGS_SIGMA || p->sgs_model == OC_SGS_AMD ||
         p->sgs_model == OC_SGS_DYNAMIC || p->sgs_model == OC_SGS_DYNAMIC_LOCAL || p->sgs_model == OC_SGS_LAGRANGIAN ||
         p->sgs_model == OC_SGS_TKE) &&
        p->stretched)
        return NULL;
    /* the TKE closure: the Boussinesq core (theta0 its buoyancy reference), WENO-Z5 transport of e (halos >= 3) */
    if (p->c_s != 0 && p->sgs_model == OC_SGS_TKE && (p->core != OC_CORE_BOUSSINESQ || p->hx < 3 || p->hy < 3 || p->hz < 3))
        return NULL;
    oc_sim* s = (oc_sim*)calloc(1, sizeof(oc_sim));
    s->p = *p;
    s->NX = p->nx + 2 * p->hx; s->NY = p->ny + 2 * p->hy; s->NZ = p->nz + 2 * p->hz;
    s->n = (int64_t)s->NX * s->NY * s->NZ;
    int NZ = s->NZ, Nz = p->nz, Hz = p->hz;
    s->uniform = !p->stretched;
    s->dx = p->lx / p->nx; s->dy = p->ly / p->ny; s->dz = p->lz / p->nz;
    s->idx = 1 / s->dx; s->idy = 1 / s->dy; s->idx2 = 1 / (s->dx * s->dx); s->idy2 = 1 / (s->dy * s->dy);
    s->idz = 1 / s->dz; s->idz2 = 1 / (s->dz * s->dz);
    s->delta_u = pow(s->dx * s->dy * s->dz, 1.0 / 3);
    /* vertical storage metrics (src/StretchedGrids.jl:345-400, :570-590) */
    s->zf = dalloc(NZ + 1); s->zc = dalloc(NZ); s->dzc = dalloc(NZ); s->dzf = dalloc(NZ + 1);
    s->idzc = dalloc(NZ); s->idzf = dalloc(NZ + 1); s->idz_off = dalloc(NZ);
    s->wlo = dalloc(NZ); s->whi = dalloc(NZ); s->alo = dalloc(NZ); s->ahi = dalloc(NZ); s->delta = dalloc(NZ);
    if (s->uniform) {
        for (int k = 0; k < NZ + 1; ++k) s->zf[k] = p->z0 + (double)(k - Hz) * s->dz;
        for (int k = 0; k < NZ; ++k) s->zc[k] = p->z0 + ((double)(k - Hz) + 0.5) * s->dz;
        for (int k = 0; k < NZ; ++k) s->dzc[k] = s->dz;
        for (int k = 0; k < NZ + 1; ++k) s->dzf[k] = s->dz;
    } else {
        for (int k = 0; k <= Nz; ++k) s->zf[Hz + k] = zfi[k];
        for (int k = Hz - 1; k >= 0; --k) s->zf[k] = 2 * s->zf[k + 1] - s->zf[k + 2];
        for (int k = Hz + Nz + 1; k <= NZ; ++k) s->zf[k] = 2 * s->zf[k - 1] - s->zf[k - 2];
        for (int k = 0; k < NZ; ++k) s->dzc[k] = s->zf[k + 1] - s->zf[k];
        for (int k = 0; k < NZ; ++k) s->zc[k] = (s->zf[k] + s->zf[k + 1]) / 2;
        s->dzf[0] = s->dzc[0];
        for (int k = 1; k < NZ; ++k) s->dzf[k] = s->zc[k] - s->zc[k - 1];
        s->dzf[NZ] = s->dzc[NZ - 1];
    }
    for (int k = 0; k < NZ; ++k) s->idzc[k] = 1 / s->dzc[k];
    for (int k = 0; k < NZ + 1; ++k) s->idzf[k] = 1 / s->dzf[k];
    for (int k = 0; k < NZ; ++k) s->idz_off[k] = 2 / (s->dzf[k] + s->dzf[k + 1]);
    for (int k = 1; k < NZ; ++k) {
        s->wlo[k] = s->dzc[k] / (s->dzc[k - 1] + s->dzc[k]);
        s->whi[k] = s->dzc[k - 1] / (s->dzc[k - 1] + s->dzc[k]);
        double sm = s->dzc[k - 1] + s->dzc[k];
        s->alo[k] = s->dzc[k - 1] / sm;
        s->ahi[k] = s->dzc[k] / sm;
    }
    for (int k = 0; k < NZ; ++k) s->delta[k] = pow(s->dx * s->dy * s->dzc[k], 1.0 / 3);
    if (p->core == OC_CORE_ANELASTIC) {
        s->wc = dalloc(NZ); s->wf = dalloc(NZ + 1); s->thf = dalloc(NZ + 1);
        memcpy(s->wc, wc, sizeof(double) * (size_t)NZ);
        memcpy(s->wf, wf, sizeof(double) * (size_t)(NZ + 1));
        if (thf) memcpy(s->thf, thf, sizeof(double) * (size_t)(NZ + 1));
    }
    int64_t n = s->n;
    s->u = dalloc(n); s->v = dalloc(n); s->w = dalloc(n); s->th = dalloc(n); s->pr = dalloc(n);
    s->nut = dalloc(n); s->kt = dalloc(n); s->phi = dalloc(n);
    s->tu = dalloc(n); s->tv = dalloc(n); s->tw = dalloc(n); s->tt = dalloc(n);
    s->u0 = dalloc(n); s->v0 = dalloc(n); s->w0 = dalloc(n); s->th0 = dalloc(n);
    int Nx = p->nx, Ny = p->ny, Mh = Nx / 2 + 1;
    s->src = dalloc((int64_t)Nx * Ny * Nz);
    s->hat = (cpx*)calloc((size_t)Mh * Ny * Nz, sizeof(cpx));
    plan_init(&s->px, Nx / 2);
    plan_init(&s->py, Ny);
    plan_init(&s->pz, Nz);
    s->twx = (cpx*)malloc(sizeof(cpx) * (size_t)Mh);
    for (int k = 0; k < Mh; ++k) {
        double a = -2.0 * M_PI * (double)k / (double)Nx;
        s->twx[k].re = cos(a); s->twx[k].im = sin(a);
    }
    /* eigenvalue pieces */
    s->kx2 = dalloc(Mh); s->ky2 = dalloc(Ny); s->kz2 = dalloc(Nz);
    if (p->solver == OC_SOLVER_FFT) {
        /* src/PressureSolvers.jl:128-130 */
        for (int m = 0; m < Mh; ++m) { double sn = sin(M_PI * m / Nx); s->kx2[m] = 4 / (s->dx * s->dx) * (sn * sn); }
        for (int m = 0; m < Ny; ++m) { double sn = sin(M_PI * m / Ny); s->ky2[m] = 4 / (s->dy * s->dy) * (sn * sn); }
        for (int m = 0; m < Nz; ++m) { double sn = sin(M_PI * m / Nz); s->kz2[m] = 4 / (s->dz * s->dz) * (sn * sn); }
    } else {
        /* _r2r_eigen, src/PressureSolvers.jl:618-624 */
        for (int m = 0; m < Mh; ++m) { int mm = m < Nx - m ? m : Nx - m; double sn = sin(M_PI * mm / Nx); s->kx2[m] = 4 / (s->dx * s->dx) * (sn * sn); }
        for (int m = 0; m < Ny; ++m) { int mm = m < Ny - m ? m : Ny - m; double sn = sin(M_PI * mm / Ny); s->ky2[m] = 4 / (s->dy * s->dy) * (sn * sn); }
        /* column coefficients */
        s->lower = dalloc(Nz); s->upper = dalloc(Nz); s->hw = dalloc(Nz);
        s->meas = dalloc(Nz); s->iota = dalloc(Nz + 1); s->gauge = dalloc(Nz);
        for (int k = 0; k < Nz; ++k) {
            int K = Hz + k;                      /* storage level of cell k */
            if (p->core == OC_CORE_ANELASTIC) {
                if (s->uniform) {
                    /* DirectWeightedPoissonSolver, src/Anelastic.jl:1013-1019 */
                    double idz2 = 1 / (s->dz * s->dz);
                    s->lower[k] = k > 0 ? s->wf[K] * idz2 : 0.0;
                    s->upper[k] = k < Nz - 1 ? s->wf[K + 1] * idz2 : 0.0;
                    s->hw[k] = s->wc[K];
                    s->meas[k] = s->dz * s->dz;
                    s->gauge[k] = 1.0;
                } else {
                    /* weighted operator on the stretched column */
                    s->lower[k] = k > 0 ? s->wf[K] / (s->dzc[K] * s->dzf[K]) : 0.0;
                    s->upper[k] = k < Nz - 1 ? s->wf[K + 1] / (s->dzc[K] * s->dzf[K + 1]) : 0.0;
                    s->hw[k] = s->wc[K];
                    s->meas[k] = s->dzc[K];
                    s->gauge[k] = s->dzc[K];
                }
            } else {
                /* ColumnTridiagonalSolver(dzc, dzf), src/PressureSolvers.jl:686-700 */
                s->lower[k] = k > 0 ? 1 / (s->dzc[K] * s->dzf[K]) : 0.0;
                s->upper[k] = k < Nz - 1 ? 1 / (s->dzc[K] * s->dzf[K + 1]) : 0.0;
                s->hw[k] = 1.0;
                s->meas[k] = s->dzc[K];
                s->gauge[k] = s->dzc[K];
            }
        }
        for (int k = 0; k <= Nz; ++k) {
            int K = Hz + k;
            if (p->core == OC_CORE_ANELASTIC)
                s->iota[k] = s->uniform ? 1 / s->wf[K] : s->dzf[K] / s->wf[K];
            else
                s->iota[k] = s->dzf[K];
        }
        s->meas_sum = 0.0; s->gauge_sum = 0.0;
        for (int k = 0; k < Nz; ++k) { s->meas_sum += s->meas[k]; s->gauge_sum += s->gauge[k]; }
    }
    if (p->c_s != 0 && p->sgs_model == OC_SGS_LAGRANGIAN) lag_alloc(s);
    if (p->c_s != 0 && p->sgs_model == OC_SGS_TKE) tke_alloc(s);
    if (p->solver == OC_SOLVER_PCG) {
        s->cgx = dalloc((int64_t)Nx * Ny * Nz);
        if (oc_set_apertures(s, NULL, NULL, NULL, 1e-8, 200)) {
            oc_destroy(s);
            return NULL;
        }
    }
    return s;
}

int oc_set_lagrangian(oc_sim* s, double c0, double theta, double memory_time) {
    if (s->p.sgs_model != OC_SGS_LAGRANGIAN || !(c0 > 0) || !(theta > 0)) return -1;
    lag_alloc(s);
    s->lag_c0 = c0; s->lag_theta = theta; s->lag_mt = memory_time > 0 ? memory_time : 0.0;
    lag_coefficient(s);
    return 0;
}

int oc_set_tke(oc_sim* s, double c_eps0, double c_eps1, double c_l, int exact) {
    if (s->p.sgs_model != OC_SGS_TKE || s->p.c_s == 0 || !(c_eps0 >= 0) || !(c_eps1 >= 0) || !(c_l > 0)) return -1;
    tke_alloc(s);
    s->tke_ce0 = c_eps0; s->tke_ce1 = c_eps1; s->tke_cl = c_l; s->tke_exact = exact != 0;
    return 0;
}

int oc_get_sgs_state(const oc_sim* s, double* out) {
    size_t ni = (size_t)s->p.nx * s->p.ny * s->p.nz;
    if (s->p.sgs_model == OC_SGS_TKE && s->tke_e && out) {
        const oc_params* P = &s->p;
        for (int k = 0; k < P->nz; ++k)
            for (int j = 0; j < P->ny; ++j)
                for (int i = 0; i < P->nx; ++i)
                    out[(size_t)i + (size_t)P->nx * ((size_t)j + (size_t)P->ny * k)] = A(s->tke_e, i + P->hx, j + P->hy, k + P->hz);
        return 0;
    }
    if (s->p.sgs_model != OC_SGS_LAGRANGIAN || !out) return -1;
    const double* a[5] = {s->lag_ilm, s->lag_imm, s->lag_up, s->lag_vp, s->lag_wp};
    for (int f = 0; f < 5; ++f)
        for (size_t q = 0; q < ni; ++q) out[f * ni + q] = a[f] ? a[f][q] : 0.0;
    out[5 * ni] = s->lag_init;
    return 0;
}

int oc_set_sgs_state(oc_sim* s, const double* in) {
    if (s->p.sgs_model == OC_SGS_TKE && s->tke_e && in) {
        const oc_params* P = &s->p;
        for (int k = 0; k < P->nz; ++k)
            for (int j = 0; j < P->ny; ++j)
                for (int i = 0; i < P->nx; ++i)
                    A(s->tke_e, i + P->hx, j + P->hy, k + P->hz) = in[(size_t)i + (size_t)P->nx * ((size_t)j + (size_t)P->ny * k)];
        fill_halos(s, s->tke_e, LOC_C);
        return 0;
    }
    if (s->p.sgs_model != OC_SGS_LAGRANGIAN || !in) return -1;
    lag_alloc(s);
    size_t ni = (size_t)s->p.nx * s->p.ny * s->p.nz;
    double* a[5] = {s->lag_ilm, s->lag_imm, s->lag_up, s->lag_vp, s->lag_wp};
    for (int f = 0; f < 5; ++f) memcpy(a[f], in + f * ni, ni * sizeof(double));
    s->lag_init = in[5 * ni] != 0;
    lag_coefficient(s);
    return 0;
}

int oc_set_sgs_buoyancy(oc_sim* s, const double* bg) {
    if (!bg) return -1;
    if (!s->amd_bg) s->amd_bg = dalloc(s->p.nz);
    for (int k = 0; k < s->p.nz; ++k) s->amd_bg[k] = bg[k];
    return 0;
}

int oc_set_apertures(oc_sim* s, const double* ax, const double* ay, const double* az, double tol, int maxit) {
    const oc_params* P = &s->p;
    if (P->solver != OC_SOLVER_PCG || !(tol > 0) || maxit < 1) return -1;
    if ((ax == NULL) != (ay == NULL) || (ax == NULL) != (az == NULL)) return -1;
    int Nx = P->nx, Ny = P->ny, Nz = P->nz;
    int64_t n[3] = {(int64_t)(Nx + 1) * Ny * Nz, (int64_t)Nx * (Ny + 1) * Nz, (int64_t)Nx * Ny * (Nz + 1)};
    const double* in[3] = {ax, ay, az};
    double* a[3];
    double* c2[3];
    for (int d = 0; d < 3; ++d) {
        a[d] = dalloc(n[d]);
        c2[d] = dalloc(n[d]);
        for (int64_t q = 0; q < n[d]; ++q) a[d][q] = in[d] ? in[d][q] : 1.0;
    }
    int bad = 0;
    for (int d = 0; d < 3; ++d)
        for (int64_t q = 0; q < n[d]; ++q)
            if (!(a[d][q] >= 0.0 && a[d][q] <= 1.0)) bad = 1;
    if (P->bc_z == OC_BC_WALL)
        for (int64_t q = 0; q < (int64_t)Nx * Ny; ++q) {
            a[2][q] = 0.0;
            a[2][(int64_t)Nz * Nx * Ny + q] = 0.0;
        }
    for (int d = 0; d < 3; ++d)
        for (int64_t q = 0; q < n[d]; ++q) c2[d][q] = a[d][q] * a[d][q];
    /* open faces: no coupling across (the Neumann condition of phi) */
    if (s->open_x)
        for (int64_t r = 0; r < (int64_t)Ny * Nz; ++r) c2[0][r * (Nx + 1)] = c2[0][r * (Nx + 1) + Nx] = 0.0;
    if (s->open_y)
        for (int k = 0; k < Nz; ++k)
            for (int i = 0; i < Nx; ++i)
                c2[1][(int64_t)k * (Ny + 1) * Nx + i] = c2[1][((int64_t)k * (Ny + 1) + Ny) * Nx + i] = 0.0;
    if (P->core == OC_CORE_ANELASTIC || !s->uniform) {
        /* the symmetric form of the density-weighted operator on the column:
         * W_c a^2 dz_c / h_z on x and y faces, W_f a^2 h_z / dz_f on z faces */
        int Hz = P->hz, anel = P->core == OC_CORE_ANELASTIC;
        for (int d = 0; d < 2; ++d) {
            int64_t row = d == 0 ? (int64_t)(Nx + 1) * Ny : (int64_t)Nx * (Ny + 1);
            for (int64_t q = 0; q < n[d]; ++q) {
                int K = Hz + (int)(q / row);
                c2[d][q] *= (anel ? s->wc[K] : 1.0) * (s->dzc[K] / s->dz);
            }
        }
        for (int64_t q = 0; q < n[2]; ++q) {
            int K = Hz + (int)(q / ((int64_t)Nx * Ny));
            c2[2][q] *= (anel ? s->wf[K] : 1.0) * (s->dz / s->dzf[K]);
        }
    }
    ocg* cg = NULL;
    if (!bad) {
        ocg_params prm = {Nx, Ny, Nz, s->dx, s->dy, s->dz, s->open_x ? OCG_BC_NEUMANN : OCG_BC_PERIODIC,
                          s->open_y ? OCG_BC_NEUMANN : OCG_BC_PERIODIC,
                          P->bc_z == OC_BC_WALL ? OCG_BC_NEUMANN : OCG_BC_PERIODIC, tol, maxit,
                          2, 2, 50, 4, 1, OCG_PC_VCYCLE};
        cg = ocg_create(&prm, c2[0], c2[1], c2[2]);
    }
    for (int d = 0; d < 3; ++d) free(c2[d]);
    if (!cg) {
        for (int d = 0; d < 3; ++d) free(a[d]);
        return -1;
    }
    free(s->apx); free(s->apy); free(s->apz);
    if (s->cg) ocg_destroy(s->cg);
    s->apx = a[0]; s->apy = a[1]; s->apz = a[2];
    s->cg = cg;
    s->cg_tol = tol;
    s->cg_maxit = maxit;
    memset(&s->cg_st, 0, sizeof(s->cg_st));
    return 0;
}

/* ---- radiating outflow (src/boundary_conditions/outflow.jl) ------------- */

static int ob_radiates(const oc_sim* s) { return s->orad[0] || s->orad[1] || s->orad[2] || s->orad[3]; }

/* element (layer l, tangential a, b) of plane (f, side) of axis 0 (x faces:
 * a = storage j, b = storage k) or 1 (y faces: a = storage i, b = storage k) */
static inline int64_t ob_pi(const oc_sim* s, int axis, int f, int side, int l, int a, int b) {
    if (axis == 0) return (((int64_t)(f * 2 + side) * s->NZ + b) * s->NY + a) * s->oL + l;
    return (((int64_t)(f * 2 + side) * s->NZ + b) * s->oL + l) * s->NX + a;
}
static inline int64_t ob_ti(const oc_sim* s, int axis, int f, int side, int a, int b) {
    return ((int64_t)(f * 2 + side) * s->NZ + b) * (axis == 0 ? s->NY : s->NX) + a;
}
static inline double* ob_field(oc_sim* s, int f) { return f == 0 ? s->u : f == 1 ? s->v : f == 2 ? s->w : s->th; }
static inline double ob_at(const oc_sim* s, const double* d, int axis, int li, int a, int b) {
    return axis == 0 ? A(d, li, a, b) : A(d, a, li, b);
}
/* storage index of the boundary layer (the normal velocity's face, the first
 * halo cell of the rest), the local layer of it, the outward step
 * (_boundary_storage, _boundary_local, _outward, outflow.jl:104-106) */
static inline void ob_geom(const oc_sim* s, int axis, int f, int side, int* sb, int* lb, int* o, int* nl) {
    int H = axis == 0 ? s->p.hx : s->p.hy, N = axis == 0 ? s->p.nx : s->p.ny;
    if (side) { *sb = H + N; *lb = 0; *o = 1; *nl = H; }
    else { *sb = f == axis ? H : H - 1; *lb = *sb; *o = -1; *nl = *sb + 1; }
}

/* prepare_open_boundaries! (open_boundary.jl:1189-1200): the step-start
 * snapshot of every buffer, and per radiating plane point the phase speed
 * c = the outward normal velocity of the boundary face when positive, else
 * NaN (an inflow point keeps its data) (_outward_un, _phase_speed_body!,
 * outflow.jl:113-182; :convective) */
static void ob_prepare(oc_sim* s, double dt) {
    int64_t nxp = (int64_t)8 * s->NZ * s->NY * s->oL, nyp = (int64_t)8 * s->NZ * s->oL * s->NX;
    memcpy(s->oxs, s->oxp, sizeof(double) * nxp);
    memcpy(s->oys, s->oyp, sizeof(double) * nyp);
    for (int axis = 0; axis < 2; ++axis)
        for (int side = 0; side < 2; ++side) {
            if (!s->orad[axis * 2 + side]) continue;
            const double* P = axis == 0 ? s->oxp : s->oyp;
            double* C = axis == 0 ? s->oxc : s->oyc;
            int NA = axis == 0 ? s->NY : s->NX;
            int H = axis == 0 ? s->p.hx : s->p.hy;
            int fl = side ? 0 : H;                       /* the normal plane's boundary face */
            double sg = side ? 1.0 : -1.0;
            int mode = s->orad[axis * 2 + side];
            double* Hs = axis == 0 ? s->oxh : s->oyh;
            double dn = axis == 0 ? s->dx : s->dy;
            for (int f = 0; f < 4; ++f)
                for (int b = 0; b < s->NZ; ++b)
                    for (int a = 0; a < NA; ++a) {
                        double un, phi1 = 0, phi2 = 0;
                        if (mode == 2) {
                            int sb, lb, o, nl;
                            ob_geom(s, axis, f, side, &sb, &lb, &o, &nl);
                            phi1 = ob_at(s, ob_field(s, f), axis, sb - o, a, b);
                            phi2 = ob_at(s, ob_field(s, f), axis, sb - 2 * o, a, b);
                        }
                        /* staggered along a tangential direction: the mean of the two faces */
                        int st1 = (axis == 0 && f == 1) || (axis == 1 && f == 0), st2 = f == 2;
                        if (st1) {
                            int am = a > 0 ? a - 1 : 0;
                            un = sg * (P[ob_pi(s, axis, axis, side, fl, am, b)] + P[ob_pi(s, axis, axis, side, fl, a, b)]) / 2;
                        } else if (st2) {
                            int bm = b > 0 ? b - 1 : 0;
                            un = sg * (P[ob_pi(s, axis, axis, side, fl, a, bm)] + P[ob_pi(s, axis, axis, side, fl, a, b)]) / 2;
                        } else {
                            un = sg * P[ob_pi(s, axis, axis, side, fl, a, b)];
                        }
                        int64_t ti = ob_ti(s, axis, f, side, a, b);
                        if (!(s->omode[f] == 0 && un > 0)) {
                            C[ti] = NAN;
                        } else if (mode == 2 && f != axis && s->ohist) {
                            /* Orlanski (1976), clipped to [0, dn/dtau] (Miller & Thorpe 1981) */
                            double num = -(phi1 - Hs[ti]) / s->olast_dt, den = (phi1 - phi2) / dn;
                            double c = num / den, cmax = dn / s->olast_dt;
                            C[ti] = isnan(c) ? 0.0 : (c < 0 ? 0.0 : (c > cmax ? cmax : c));
                        } else {
                            C[ti] = un;
                        }
                        if (mode == 2) Hs[ti] = phi1;
                    }
        }
    s->ohist = 1;
    s->olast_dt = dt;
}

/* mark_open_boundary_stage! (outflow.jl:198-237): the two interior layers
 * next to every radiating face at the start of a (sub)stage */
static void ob_mark(oc_sim* s) {
    for (int axis = 0; axis < 2; ++axis)
        for (int side = 0; side < 2; ++side) {
            if (!s->orad[axis * 2 + side]) continue;
            int NA = axis == 0 ? s->NY : s->NX;
            double* S1 = axis == 0 ? s->ox1 : s->oy1;
            double* S2 = axis == 0 ? s->ox2 : s->oy2;
            for (int f = 0; f < 4; ++f) {
                int sb, lb, o, nl;
                ob_geom(s, axis, f, side, &sb, &lb, &o, &nl);
                const double* d = ob_field(s, f);
                for (int b = 0; b < s->NZ; ++b)
                    for (int a = 0; a < NA; ++a) {
                        S1[ob_ti(s, axis, f, side, a, b)] = ob_at(s, d, axis, sb - o, a, b);
                        S2[ob_ti(s, axis, f, side, a, b)] = ob_at(s, d, axis, sb - 2 * o, a, b);
                    }
            }
        }
    s->omarked = 1;
}

/* correct_boundary_mass_flux! (open_boundary.jl:1024-1083) on the buffers */
static void ob_correct(oc_sim* s) {
    const oc_params* P = &s->p;
    double Q = 0, Aout = 0, Aall = 0;
    for (int pass = 0; pass < 2; ++pass) {
        double delta = 0;
        int only_out = 0;
        if (pass == 1) {
            if (s->ocorr == 2 || Q == 0) break;
            only_out = s->ocorr == 1;
            double Ar = only_out ? Aout : Aall;
            if (Ar == 0) { only_out = 0; Ar = Aall; }
            delta = Q / Ar;
            s->odelta = delta;
        }
        for (int axis = 0; axis < 2; ++axis) {
            if (!(axis == 0 ? s->open_x : s->open_y)) continue;
            double* Pl = axis == 0 ? s->oxp : s->oyp;
            int H = axis == 0 ? P->hx : P->hy, Ht = axis == 0 ? P->hy : P->hx, Nt = axis == 0 ? P->ny : P->nx;
            double area = (axis == 0 ? s->dy : s->dx) * s->dz;
            for (int side = 0; side < 2; ++side) {
                int fl = side ? 0 : H;
                double sg = side ? 1.0 : -1.0;
                for (int b = P->hz; b < P->hz + P->nz; ++b)
                    for (int a = Ht; a < Ht + Nt; ++a) {
                        const double* F = axis == 0 ? s->oxf : s->oyf;
                        const double wt = F ? F[((int64_t)side * P->nz + (b - P->hz)) * Nt + (a - Ht)] : 1.0;
                        if (!(wt > 0)) continue;
                        double* v = &Pl[ob_pi(s, axis, axis, side, fl, a, b)];
                        double out = sg * *v;
                        if (pass == 0) {
                            Q += out * area * wt;
                            if (out > 0) Aout += area * wt;
                            Aall += area * wt;
                        } else if (!only_out || out > 0) {
                            *v -= sg * delta;
                        }
                    }
            }
        }
    }
    s->oQ = Q;
    if (s->ocorr == 2 || Q == 0) s->odelta = 0;
    double R = 0;
    for (int axis = 0; axis < 2; ++axis) {
        if (!(axis == 0 ? s->open_x : s->open_y)) continue;
        double* Pl = axis == 0 ? s->oxp : s->oyp;
        int H = axis == 0 ? P->hx : P->hy, Ht = axis == 0 ? P->hy : P->hx, Nt = axis == 0 ? P->ny : P->nx;
        double area = (axis == 0 ? s->dy : s->dx) * s->dz;
        const double* F = axis == 0 ? s->oxf : s->oyf;
        for (int side = 0; side < 2; ++side)
            for (int b = P->hz; b < P->hz + P->nz; ++b)
                for (int a = Ht; a < Ht + Nt; ++a) {
                    const double wt = F ? F[((int64_t)side * P->nz + (b - P->hz)) * Nt + (a - Ht)] : 1.0;
                    if (wt > 0) R += (side ? 1.0 : -1.0) * Pl[ob_pi(s, axis, axis, side, side ? 0 : H, a, b)] * area * wt;
                }
    }
    s->oresid = R;
}

/* update_open_boundaries! (open_boundary.jl:1137-1152) with a radiating face:
 * the buffers from the data, the outflow points advanced by the explicit
 * second-order upstream radiation update from the stage-start values
 * (_radiate_body!, outflow.jl:240-285), then the mass-flux correction */
static void ob_update(oc_sim* s, double dt) {
    if (!ob_radiates(s)) return;
    int64_t nxp = (int64_t)8 * s->NZ * s->NY * s->oL, nyp = (int64_t)8 * s->NZ * s->oL * s->NX;
    memcpy(s->oxv, s->oxp, sizeof(double) * nxp);
    memcpy(s->oyv, s->oyp, sizeof(double) * nyp);
    memcpy(s->oxp, s->oxd, sizeof(double) * nxp);
    memcpy(s->oyp, s->oyd, sizeof(double) * nyp);
    for (int axis = 0; axis < 2; ++axis)
        for (int side = 0; side < 2; ++side) {
            if (!s->orad[axis * 2 + side]) continue;
            int NA = axis == 0 ? s->NY : s->NX;
            double dn = axis == 0 ? s->dx : s->dy;
            double* Pl = axis == 0 ? s->oxp : s->oyp;
            const double* P0 = axis == 0 ? s->oxv : s->oyv;
            const double* C = axis == 0 ? s->oxc : s->oyc;
            const double* S1 = axis == 0 ? s->ox1 : s->oy1;
            const double* S2 = axis == 0 ? s->ox2 : s->oy2;
            for (int f = 0; f < 4; ++f) {
                int sb, lb, o, nl;
                ob_geom(s, axis, f, side, &sb, &lb, &o, &nl);
                const double* d = ob_field(s, f);
                for (int b = 0; b < s->NZ; ++b)
                    for (int a = 0; a < NA; ++a) {
                        double c = C[ob_ti(s, axis, f, side, a, b)];
                        if (isnan(c)) continue;
                        double r = fmin(c * dt / dn, 1.0);
                        double i1 = s->omarked ? S1[ob_ti(s, axis, f, side, a, b)] : ob_at(s, d, axis, sb - o, a, b);
                        double i2 = s->omarked ? S2[ob_ti(s, axis, f, side, a, b)] : ob_at(s, d, axis, sb - 2 * o, a, b);
                        for (int q = 0, l = lb; q < nl; ++q, l += o) {
                            double p0 = P0[ob_pi(s, axis, f, side, l, a, b)];
                            Pl[ob_pi(s, axis, f, side, l, a, b)] = p0 - r * (3 * p0 - 4 * i1 + i2) / 2;
                            i2 = i1;
                            i1 = p0;
                        }
                    }
            }
        }
    s->omarked = 0;
    ob_correct(s);
}

/* combine_open_boundaries! (open_boundary.jl:1262-1280): buffer = a snapshot + b buffer */
static void ob_combine(oc_sim* s, double a, double b) {
    if (!ob_radiates(s)) return;
    int64_t nxp = (int64_t)8 * s->NZ * s->NY * s->oL, nyp = (int64_t)8 * s->NZ * s->oL * s->NX;
    for (int64_t q = 0; q < nxp; ++q) s->oxp[q] = a * s->oxs[q] + b * s->oxp[q];
    for (int64_t q = 0; q < nyp; ++q) s->oyp[q] = a * s->oys[q] + b * s->oyp[q];
}

/* Open lateral faces (open_boundary_conditions and the halo fills of
 * src/boundary_conditions/open_boundary.jl:532-807): copies of the planes
 * (the layout of aeo_set_open), the modes; the CG rebuilt on the domain's
 * apertures with the Neumann condition on the open axes.  open_x = open_y = 0
 * closes them. */
int oc_set_open(oc_sim* s, int open_x, int open_y, const double* xp, const double* yp, const int* modes) {
    const oc_params* P = &s->p;
    if (P->solver != OC_SOLVER_PCG || P->core == OC_CORE_ANELASTIC || !s->uniform || P->bc_z != OC_BC_WALL ||
        (P->c_s != 0.0 && (P->sgs_model == OC_SGS_DYNAMIC || P->sgs_model == OC_SGS_DYNAMIC_LOCAL ||
                           P->sgs_model == OC_SGS_LAGRANGIAN || P->sgs_model == OC_SGS_TKE)))
        return -1;
    if ((open_x && !xp) || (open_y && !yp) || ((open_x || open_y) && !modes)) return -1;
    int L = (P->hx > P->hy ? P->hx : P->hy) + 1;
    int64_t nxp = (int64_t)8 * s->NZ * s->NY * L, nyp = (int64_t)8 * s->NZ * L * s->NX;
    free(s->oxp); free(s->oyp);
    s->oxp = dalloc(nxp);
    s->oyp = dalloc(nyp);
    if (open_x) memcpy(s->oxp, xp, sizeof(double) * nxp);
    if (open_y) memcpy(s->oyp, yp, sizeof(double) * nyp);
    for (int f = 0; f < 4; ++f) s->omode[f] = (open_x || open_y) ? modes[f] : 0;
    s->oL = L;
    s->open_x = open_x != 0;
    s->open_y = open_y != 0;
    for (int q = 0; q < 4; ++q) s->orad[q] = 0;   /* Dirichlet until oc_set_open_outflow */
    /* the operator on the current apertures (the wall faces already closed) */
    int64_t n[3] = {(int64_t)(P->nx + 1) * P->ny * P->nz, (int64_t)P->nx * (P->ny + 1) * P->nz,
                    (int64_t)P->nx * P->ny * (P->nz + 1)};
    double* a[3];
    for (int d = 0; d < 3; ++d) {
        const double* src = d == 0 ? s->apx : d == 1 ? s->apy : s->apz;
        a[d] = dalloc(n[d]);
        for (int64_t q = 0; q < n[d]; ++q) a[d][q] = src ? src[q] : 1.0;
    }
    int r = oc_set_apertures(s, a[0], a[1], a[2], s->cg ? s->cg_tol : 1e-8, s->cg ? s->cg_maxit : 200);
    for (int d = 0; d < 3; ++d) free(a[d]);
    if (r) return r;
    oc_fill_state_halos(s);
    return 0;
}

/* The radiating outflow of open faces already set (oc_set_open): rad[4]
 * (west, east, south, north) 1 = :convective, the correction mode (0 uniform,
 * 1 outflow only, 2 none) and the raw data planes (before the correction) in
 * the layout of the buffers.  All zero: Dirichlet outflow everywhere. */
void oc_get_open_planes(const oc_sim* s, double* xp, double* yp) {
    int64_t nxp = (int64_t)8 * s->NZ * s->NY * s->oL, nyp = (int64_t)8 * s->NZ * s->oL * s->NX;
    if (xp && s->oxp) memcpy(xp, s->oxp, sizeof(double) * nxp);
    if (yp && s->oyp) memcpy(yp, s->oyp, sizeof(double) * nyp);
}

/* A checkpoint's planes back into the buffers (restore_open_boundary_checkpoint!,
 * open_boundary.jl:1307-1350), the state's halos refilled from them */
int oc_set_open_planes(oc_sim* s, const double* xp, const double* yp) {
    if (!(s->open_x || s->open_y) || !xp || !yp) return -1;
    int64_t nxp = (int64_t)8 * s->NZ * s->NY * s->oL, nyp = (int64_t)8 * s->NZ * s->oL * s->NX;
    memcpy(s->oxp, xp, sizeof(double) * nxp);
    memcpy(s->oyp, yp, sizeof(double) * nyp);
    oc_fill_state_halos(s);
    return 0;
}

/* The :orlanski history of a radiating set ([f][side][NZ][NY or NX]) and
 * sc = (history set, the last step's length): read (set 0) or written */
int oc_open_history(oc_sim* s, double* xh, double* yh, double* sc, int set) {
    if (!ob_radiates(s) || !xh || !yh || !sc) return -1;
    int64_t ntx = (int64_t)8 * s->NZ * s->NY, nty = (int64_t)8 * s->NZ * s->NX;
    if (set) {
        memcpy(s->oxh, xh, sizeof(double) * ntx);
        memcpy(s->oyh, yh, sizeof(double) * nty);
        s->ohist = sc[0] != 0.0;
        s->olast_dt = sc[1];
    } else {
        memcpy(xh, s->oxh, sizeof(double) * ntx);
        memcpy(yh, s->oyh, sizeof(double) * nty);
        sc[0] = s->ohist;
        sc[1] = s->olast_dt;
    }
    return 0;
}

void oc_open_ledger(const oc_sim* s, double* out) { out[0] = s->oQ; out[1] = s->oresid; out[2] = s->odelta; }

int oc_set_open_outflow(oc_sim* s, const int* rad, int corr, const double* xd, const double* yd,
                        const double* xf, const double* yf) {
    if (!(s->open_x || s->open_y) || !rad || corr < 0 || corr > 2) return -1;
    for (int q = 0; q < 4; ++q) {
        if (rad[q] < 0 || rad[q] > 2 || (rad[q] && !(q < 2 ? s->open_x : s->open_y))) return -1;
        s->orad[q] = rad[q];
    }
    s->ohist = 0;
    s->ocorr = corr;
    int64_t nxp = (int64_t)8 * s->NZ * s->NY * s->oL, nyp = (int64_t)8 * s->NZ * s->oL * s->NX;
    int64_t ntx = (int64_t)8 * s->NZ * s->NY, nty = (int64_t)8 * s->NZ * s->NX;
    double** bufs[6] = {&s->oxd, &s->oyd, &s->oxs, &s->oys, &s->oxv, &s->oyv};
    for (int q = 0; q < 6; ++q) { free(*bufs[q]); *bufs[q] = dalloc(q % 2 ? nyp : nxp); }
    double** tb[8] = {&s->oxc, &s->oyc, &s->ox1, &s->oy1, &s->ox2, &s->oy2, &s->oxh, &s->oyh};
    for (int q = 0; q < 8; ++q) { free(*tb[q]); *tb[q] = dalloc(q % 2 ? nty : ntx); }
    free(s->oxf); free(s->oyf);
    s->oxf = dalloc((int64_t)2 * s->p.nz * s->p.ny);
    s->oyf = dalloc((int64_t)2 * s->p.nz * s->p.nx);
    for (int64_t q = 0; q < (int64_t)2 * s->p.nz * s->p.ny; ++q) s->oxf[q] = xf ? xf[q] : 1.0;
    for (int64_t q = 0; q < (int64_t)2 * s->p.nz * s->p.nx; ++q) s->oyf[q] = yf ? yf[q] : 1.0;
    if (ob_radiates(s)) {
        if ((s->open_x && !xd) || (s->open_y && !yd)) return -1;
        if (s->open_x) memcpy(s->oxd, xd, sizeof(double) * nxp);
        if (s->open_y) memcpy(s->oyd, yd, sizeof(double) * nyp);
    }
    s->omarked = 0;
    return 0;
}

int oc_pcg_stats(const oc_sim* s, int* iterations, int* status, double* residual, double* bnorm) {
    if (s->p.solver != OC_SOLVER_PCG) return -1;
    if (iterations) *iterations = s->cg_st.iterations;
    if (status) *status = s->cg_st.status;
    if (residual) *residual = s->cg_st.residual;
    if (bnorm) *bnorm = s->cg_st.bnorm;
    return 0;
}

void oc_destroy(oc_sim* s) {
    if (!s) return;
    double* ptrs[] = {s->zf, s->zc, s->dzc, s->dzf, s->idzc, s->idzf, s->idz_off, s->wlo, s->whi, s->alo, s->ahi,
                      s->delta, s->wc, s->wf, s->thf, s->u, s->v, s->w, s->th, s->pr, s->nut, s->kt, s->phi,
                      s->tu, s->tv, s->tw, s->tt, s->u0, s->v0, s->w0, s->th0, s->src, s->kx2, s->ky2, s->kz2,
                      s->lower, s->upper, s->hw, s->meas, s->iota, s->gauge};
    for (size_t q = 0; q < sizeof(ptrs) / sizeof(ptrs[0]); ++q) free(ptrs[q]);
    free(s->hat); free(s->twx);
    free(s->apx); free(s->apy); free(s->apz); free(s->cgx); free(s->ibm); free(s->oxp); free(s->oyp);
    free(s->oxd); free(s->oyd); free(s->oxs); free(s->oys); free(s->oxv); free(s->oyv);
    free(s->oxc); free(s->oyc); free(s->ox1); free(s->oy1); free(s->ox2); free(s->oy2);
    free(s->oxf); free(s->oyf); free(s->oxh); free(s->oyh);
    for (int f = 0; f < 10; ++f) free(s->dyn[f]);
    free(s->dyn_lm); free(s->dyn_mm); free(s->cs2); free(s->amd_bg);
    free(s->lag_ilm); free(s->lag_imm); free(s->lag_up); free(s->lag_vp); free(s->lag_wp);
    free(s->lag_cs2); free(s->lag_nlm); free(s->lag_nmm);
    free(s->tke_e); free(s->tke_k2); free(s->tke_tend); free(s->tke_new);
    if (s->cg) ocg_destroy(s->cg);
    plan_free(&s->px); plan_free(&s->py); plan_free(&s->pz);
    free(s);
}

int64_t oc_storage_size(const oc_sim* s) { return s->n; }

static double* field_ptr(const oc_sim* s, int id) {
    switch (id) {
        case OC_U: return s->u;
        case OC_V: return s->v;
        case OC_W: return s->w;
        case OC_THETA: return s->th;
        case OC_P: return s->pr;
        case OC_NUT: return s->nut;
        case OC_KT: return s->kt;
        case OC_PHI: return s->phi;
        default: return NULL;
    }
}

int oc_set_field(oc_sim* s, int id, const double* src) {
    double* d = field_ptr(s, id);
    if (!d) return -1;
    memcpy(d, src, sizeof(double) * (size_t)s->n);
    return 0;
}

int oc_get_field(const oc_sim* s, int id, double* dst) {
    const double* d = field_ptr(s, id);
    if (!d) return -1;
    memcpy(dst, d, sizeof(double) * (size_t)s->n);
    return 0;
}
