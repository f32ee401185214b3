// aeo_cutcell.cuh -- the projection of the stepping engine with the
// multigrid-preconditioned CG pressure solver (solver = AEO_SOLVER_PCG) on
// cut-cell face apertures.
//
// With apertures a in [0, 1] on every face (a = 0: blocked), the projection
// solves A phi = b with
//   b        = sum over the cell's faces of (+-) a u* / h   (the aperture-weighted divergence),
//   A phi    = sum over the cell's faces of a^2 (phi_nbr - phi) / h^2,
// the a^2-weighted Laplacian of the MG-PCG handle, and corrects
//   u = u* - a (phi+ - phi-) / h    on every face,
// so that the aperture-weighted divergence of u is A phi - b = 0 to the
// solve's tolerance, and the velocity of a blocked face is zero after every
// projection (apply_cutcell_velocity_bc!, src/CutCell.jl:852-880).  b is
// cutcell_divergence! times vol_eff (the symmetric right-hand side) and the
// correction is cutcell_gradient_x/y/z! (src/CutCell.jl:602-700); with every
// aperture 1 this is the projection of MGPreconditionedCG as the Boussinesq
// pressure solver (the urban :mg_cg slot, src/components/urban/pressure_solver.jl:126).
//
// On the sound-proof core and on a stretched column the same projection
// carries the density weights W_c, W_f (DensityWeightedPoissonSolver,
// src/Anelastic.jl:734-793: W_c on x and y faces, W_f on z faces) and the
// column metrics, in the symmetric form the multigrid hierarchy takes (one
// spacing h_z = L_z / N_z per axis): every equation is multiplied by
// dz_c[k] / h_z, so
//   b     = dz_c/h_z (W_c (a u)_x + W_c (a v)_y) + (W_f a w)_z / h_z   (differences over the cell),
//   A phi = sum of c (phi_nbr - phi) / h^2,  c = W_c a^2 dz_c / h_z (x, y faces), W_f a^2 h_z / dz_f (z faces),
//   w     = w* - a (phi_k - phi_k-1) / dz_f   (u, v as before),
// and after the projection the aperture- and density-weighted divergence
// D(W a u) vanishes to the solve's tolerance (the a = 1 case is the direct
// weighted solve's constraint, src/Anelastic.jl:987-1021).
//
// Apertures live in the face layout of aeolus_b200_mgpcg.h: ax (nx+1) per
// row, ay (ny+1) rows per level, az (nz+1) levels; face index i is the west
// (south, bottom) face of cell i.
#pragma once

#include "aeo_common.cuh"

// b = the aperture-weighted divergence of (u*, v*, w*) (interior arrays), in
// FP64; ANEL: density-weighted, !UNI: on the stretched column (symmetric form)
template <typename R, bool ANEL = false, bool UNI = true>
__global__ void __launch_bounds__(256) cc_div_kernel(Geo g, const R* __restrict__ us, const R* __restrict__ vs,
                                                     const R* __restrict__ ws, const R* __restrict__ ax,
                                                     const R* __restrict__ ay, const R* __restrict__ az,
                                                     double* __restrict__ b, const R* __restrict__ bw = nullptr,
                                                     const R* __restrict__ be = nullptr,
                                                     const R* __restrict__ bs = nullptr,
                                                     const R* __restrict__ bn = nullptr) {
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= g.nin) return;
    const int lnx = __ffs(g.nx) - 1, lny = __ffs(g.ny) - 1;
    const int i = (int)(q & (g.nx - 1)), j = (int)((q >> lnx) & (g.ny - 1)), k = (int)(q >> (lnx + lny));
    const long long pl = (long long)g.nx * g.ny;
    const long long xr = (long long)(g.nx + 1) * (j + (long long)g.ny * k);
    const long long yr = (long long)g.nx * (j + (long long)(g.ny + 1) * k);
    const R aw = ax[xr + i], ae = ax[xr + i + 1];
    const R as = ay[yr + i], an = ay[yr + g.nx + i];
    const R ab = az[q], at = az[q + pl];
    R uw = us[q], ue = us[i + 1 < g.nx ? q + 1 : q + 1 - g.nx];
    R vsv = vs[q], vn = vs[j + 1 < g.ny ? q + g.nx : q - (long long)(g.ny - 1) * g.nx];
    // open faces: the boundary faces carry the planes' (mass-corrected) normal
    // velocities, which the fill writes into u* before the projection
    if (bw) {
        if (i == 0) uw = bw[(long long)k * g.ny + j];
        if (i == g.nx - 1) ue = be[(long long)k * g.ny + j];
    }
    if (bs) {
        if (j == 0) vsv = bs[(long long)k * g.nx + i];
        if (j == g.ny - 1) vn = bn[(long long)k * g.nx + i];
    }
    const R wb = ws[q];
    const R wt = k + 1 < g.nz ? ws[q + pl] : (g.bc_z == 0 ? ws[q - (long long)(g.nz - 1) * pl] : R(0));
    // in FP64 whatever R is: a fluid region the obstacles seal off from the rest
    // adds a null space whose right-hand side sums to zero only to the
    // rounding of this sum, and CG drifts along it unless that rounding is FP64's
    if constexpr (!ANEL && UNI) {
        b[q] = ((double)ae * ue - (double)aw * uw) * g.idx + ((double)an * vn - (double)as * vsv) * g.idy +
               ((double)at * wt - (double)ab * wb) * g.idz;
    } else {
        const double wc = ANEL ? lvl(g.wc, k) : 1.0;
        const double wfb = ANEL ? lvl(g.wf, k) : 1.0, wft = ANEL ? lvl(g.wf, k + 1) : 1.0;
        const double sc = UNI ? 1.0 : g.idz / lvl(g.idzc, k);   // dz_c / h_z
        b[q] = wc * sc * (((double)ae * ue - (double)aw * uw) * g.idx + ((double)an * vn - (double)as * vsv) * g.idy) +
               (wft * ((double)at * wt) - wfb * ((double)ab * wb)) * g.idz;
    }
}

// u = c(u* - a d(phi), u^n) on every face (0 on a blocked one), p = phi/dt;
// c(x, s) = ca*s + cb*x in RK3 stages 2 and 3 (as correct_kernel)
template <typename R, bool UNI = true>
__global__ void __launch_bounds__(256) cc_correct_kernel(Geo g, const R* __restrict__ us, const R* __restrict__ vs,
                                                         const R* __restrict__ ws, const double* __restrict__ phi,
                                                         const R* __restrict__ ax, const R* __restrict__ ay,
                                                         const R* __restrict__ az, const R* u0, const R* v0,
                                                         const R* w0, R* uo, R* vo, R* wo, R* __restrict__ p,
                                                         const double* __restrict__ dtp, R ca, R cb, int stage,
                                                         const R* __restrict__ bw = nullptr,
                                                         const R* __restrict__ bs = nullptr) {
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= g.nin) return;
    const int lnx = __ffs(g.nx) - 1, lny = __ffs(g.ny) - 1;
    const int i = (int)(q & (g.nx - 1)), j = (int)((q >> lnx) & (g.ny - 1)), k = (int)(q >> (lnx + lny));
    const long long pl = (long long)g.nx * g.ny;
    const double pc = phi[q];
    // a west / south open face: phi's mirror halo (d phi / dn = 0) leaves the
    // prescribed boundary-face velocity as the fill wrote it
    const bool ow = bw && i == 0, os = bs && j == 0;
    const double pw = ow ? pc : phi[i > 0 ? q - 1 : q + g.nx - 1];
    const double ps = os ? pc : phi[j > 0 ? q - g.nx : q + (long long)(g.ny - 1) * g.nx];
    // k - 1 = -1: periodic wrap, or the wall mirror (the bottom face is blocked there)
    const double pb = phi[k > 0 ? q - pl : (g.bc_z == 0 ? q + (long long)(g.nz - 1) * pl : q)];
    const R aw = ax[(long long)(g.nx + 1) * (j + (long long)g.ny * k) + i];
    const R as = ay[(long long)g.nx * (j + (long long)(g.ny + 1) * k) + i];
    const R ab = az[q];
    const R ustar = ow ? bw[(long long)k * g.ny + j] : us[q], vstar = os ? bs[(long long)k * g.nx + i] : vs[q];
    R un = aw > R(0) ? ustar - aw * R((pc - pw) * g.idx) : R(0);
    R vn = as > R(0) ? vstar - as * R((pc - ps) * g.idy) : R(0);
    R wn = ab > R(0) ? ws[q] - ab * R((pc - pb) * (UNI ? g.idz : lvl(g.idzf, k))) : R(0);
    const long long qp = pidx(g, i, j, k);
    if (stage) {
        un = rk_combine(ca, cb, u0[qp], un);
        vn = rk_combine(ca, cb, v0[qp], vn);
        wn = rk_combine(ca, cb, w0[qp], wn);
    }
    uo[qp] = un;
    vo[qp] = vn;
    wo[qp] = wn;
    p[q] = R(pc / __ldg(dtp));   // p = phi/dt (_DivBy, src/Simulations.jl:1207-1211)
}

// y[i] = x[i] in FP64 (the seam-2 source into the solver's right-hand side)
template <typename R>
__global__ void to_f64_kernel(long long n, const R* __restrict__ x, double* __restrict__ y) {
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q < n) y[q] = (double)x[q];
}
template <typename R>
__global__ void from_f64_kernel(long long n, const double* __restrict__ x, R* __restrict__ y) {
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q < n) y[q] = R(x[q]);
}

// per level: max |aperture-weighted divergence| of the padded state (halos
// filled); ANEL: (1/W_c) D(W a u), the weighted constraint
template <typename R, bool ANEL = false, bool UNI = true>
__global__ void __launch_bounds__(256) cc_maxdiv_levels_kernel(Geo g, const R* __restrict__ u,
                                                               const R* __restrict__ v, const R* __restrict__ w,
                                                               const R* __restrict__ ax, const R* __restrict__ ay,
                                                               const R* __restrict__ az, double* __restrict__ part) {
    __shared__ double red[256];
    const int k = blockIdx.x;
    double acc = 0.0;
    for (int e = threadIdx.x; e < g.nx * g.ny; e += blockDim.x) {
        const int i = e % g.nx, j = e / g.nx;
        const long long q = pidx(g, i, j, k), qi = iidx(g, i, j, k);
        const long long xr = (long long)(g.nx + 1) * (j + (long long)g.ny * k);
        const long long yr = (long long)g.nx * (j + (long long)(g.ny + 1) * k);
        const double du = ((double)ax[xr + i + 1] * (double)u[q + 1] - (double)ax[xr + i] * (double)u[q]) * g.idx;
        const double dv = ((double)ay[yr + g.nx + i] * (double)v[q + g.sy] - (double)ay[yr + i] * (double)v[q]) * g.idy;
        const double idz = UNI ? g.idz : lvl(g.idzc, k);
        double dw;
        if (ANEL)
            dw = (lvl(g.wf, k + 1) * ((double)az[qi + (long long)g.nx * g.ny] * (double)w[q + g.sz]) -
                  lvl(g.wf, k) * ((double)az[qi] * (double)w[q])) * idz / lvl(g.wc, k);
        else
            dw = ((double)az[qi + (long long)g.nx * g.ny] * (double)w[q + g.sz] - (double)az[qi] * (double)w[q]) * idz;
        acc = fmax(acc, fabs(du + dv + dw));
    }
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + s]);
        __syncthreads();
    }
    if (threadIdx.x == 0) part[k] = red[0];
}

// implicit_ibm_correction! (src/IBM.jl:295-300) as the post-predictor term
// (src/Simulations.jl:624-628) on the interior predictor faces: a face is
// scaled by 1/(1 + dt/tau) (0 for tau = 0) once per solid cell it touches --
// the cell above it along its axis and, but for the first face of a row
// (whose low neighbour lies beyond the interior, where the halo fill that
// follows the hook replaces the scaled copy), the cell below.
template <typename R>
__global__ void __launch_bounds__(256) ibm_kernel(Geo g, R* __restrict__ us, R* __restrict__ vs, R* __restrict__ ws,
                                                  const unsigned char* __restrict__ mask,
                                                  const double* __restrict__ dtp, double tau) {
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= g.nin) return;
    const int lnx = __ffs(g.nx) - 1, lny = __ffs(g.ny) - 1;
    const int i = (int)(q & (g.nx - 1)), j = (int)((q >> lnx) & (g.ny - 1)), k = (int)(q >> (lnx + lny));
    const long long pl = (long long)g.nx * g.ny;
    const int mc = mask[q];
    const int nu = mc + (i > 0 ? mask[q - 1] : 0);
    const int nv = mc + (j > 0 ? mask[q - g.nx] : 0);
    const int nw = mc + (k > 0 ? mask[q - pl] : 0);
    if ((nu | nv | nw) == 0) return;
    const R f = tau > 0 ? R(1.0 / (1.0 + *dtp / tau)) : R(0);
    if (nu) {
        R v = us[q] * f;
        if (nu > 1) v = v * f;
        us[q] = v;
    }
    if (nv) {
        R v = vs[q] * f;
        if (nv > 1) v = v * f;
        vs[q] = v;
    }
    if (nw) {
        R v = ws[q] * f;
        if (nw > 1) v = v * f;
        ws[q] = v;
    }
}
