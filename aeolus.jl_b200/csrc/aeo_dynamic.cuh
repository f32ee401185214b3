// aeo_dynamic.cuh -- the dynamic Smagorinsky coefficient: the Germano
// identity in Lilly's least-squares form, plane-averaged per level and
// clipped to [0, cs_max^2] (compute_dynamic_smagorinsky_nut! and its passes
// _germano_pass1! / _germano_pass2! / _germano_LM_MM / _plane_cs2_body! /
// _dynamic_nut!, src/Operators.jl:488-496, :548-900).
//
// Pass 1 writes the cell-centred velocity, the strain tensor and |S| of the
// interior plus one shell of halo cells into ten workspace arrays (the 3 x 3 x
// 3 test filter of an interior cell reaches one cell into the halo); pass 2
// sums the 21 test-filtered quantities over each interior cell's box (z
// outer, x inner), forms L^d_ij M_ij and M_ij M_ij and reduces them per level
// chunk; the level pass adds the chunks and clips LM / MM. The sweep then
// evaluates nu_t = cs2(k) Delta^2 |S| in its coefficient pass.  With the
// :local averaging pass 2 writes each cell's clipped LM / MM instead (a
// padded field with filled halos) and nu_t = cs2(i, j, k) Delta^2 |S|; the
// Lagrangian closure runs passes 1 and 2 once per step, after it, to
// commit its memories, whose clipped ratio is the next step's cs2(i, j, k).
#pragma once

#include "aeo_sweep.cuh"

enum { DYN_UC = 0, DYN_VC, DYN_WC, DYN_S11, DYN_S22, DYN_S33, DYN_S12, DYN_S13, DYN_S23, DYN_MS, DYN_N };

template <typename R>
struct DynWs {
    R* f[DYN_N];      // (nx+2) x (ny+2) x (nz+2), x fastest; shell index l = interior index + 1
    int sx, sy;       // nx + 2, ny + 2
};

// Pass 1 over the interior plus one shell (_germano_pass1_body!).
template <typename R>
__global__ void __launch_bounds__(256) germano_pass1_kernel(Geo g, const R* __restrict__ u, const R* __restrict__ v,
                                                            const R* __restrict__ w, DynWs<R> ws) {
    const long long n = (long long)ws.sx * ws.sy * (g.nz + 2);
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
         e += (long long)gridDim.x * blockDim.x) {
        const int li = (int)(e % ws.sx);
        const long long r = e / ws.sx;
        const int lj = (int)(r % ws.sy), lk = (int)(r / ws.sy);
        const int i = li - 1, j = lj - 1, k = lk - 1;
        const long long q = pidx(g, i, j, k);
        Nb<R> U{u + q, g.sy, g.sz}, V{v + q, g.sy, g.sz}, W{w + q, g.sy, g.sz};
        ws.f[DYN_UC][e] = R(0.5) * (U(0, 0, 0) + U(1, 0, 0));
        ws.f[DYN_VC][e] = R(0.5) * (V(0, 0, 0) + V(0, 1, 0));
        ws.f[DYN_WC][e] = R(0.5) * (W(0, 0, 0) + W(0, 0, 1));
        R S6[6];
        const R ms = strain_at<R, true>(Met<R, true>(g), g, k, U, V, W, S6);
#pragma unroll
        for (int c = 0; c < 6; ++c) ws.f[DYN_S11 + c][e] = S6[c];
        ws.f[DYN_MS][e] = ms;
    }
}

// The Lagrangian averaging (LagrangianDynamicSmagorinsky,
// src/operators/lagrangian_sgs.jl): two sets of five interior arrays (x
// fastest) -- I_LM, I_MM and the cell-centred velocity u^n the memory was
// committed with -- one committed, the other written by the next commit.
// state[0] is the committed set, state[1] is 1 once the memory is
// initialised; both change only in lag_flip_kernel, after the commit.
template <typename R>
struct LagArgs {
    R* mem[2][5];
    int* state;
    const double* dtp;     // the step's dt
    double idx, idy, idz;  // 1 / dx, 1 / dy, 1 / dz
    double theta_delta;    // theta (dx dy dz)^(1/3)
    double memory_time;    // > 0: the fixed relaxation time, else MLC96's T
    double c02;            // C0^2
    double cs2max;
};

// _wrapidx (lagrangian_sgs.jl:392): the 1-based index n wrapped (periodic)
// or clamped to [1, N], returned 0-based
__device__ __forceinline__ int lag_wrap(int n, int N, bool per) {
    if (per) { const int r = (n - 1) % N; return r < 0 ? r + N : r; }
    return min(max(n, 1), N) - 1;
}

// One cell's commit (advance_sgs! :306-355 with _upstream_n :406-436 and
// _relax_pairs! :545-568): the first commit sets I_MM = MM, I_LM = C0^2 MM;
// later ones interpolate the committed memories trilinearly at the departure
// point x - u^n dt (1-based fractional indices as the reference, clamped to
// [1, N] across a wall) and relax toward this step's identity with epsilon =
// (dt/T) / (1 + dt/T), T = theta Delta (max(lm, 1e-8 mm) mm)^(-1/8) (1 where
// the upstream mm is 0; the fixed memory_time if given), I_LM clipped at 0.
// u^n becomes this state's cell-centred velocity; cs2f (padded) gets the new
// memory's clipped ratio (_local_cs2_body!).
template <typename R>
__device__ __forceinline__ void lag_commit_cell(const Geo& g, const DynWs<R>& ws, const LagArgs<R>& L, R* cs2f,
                                                int i, int j, int k, double lmc, double mmc) {
    const int cs = L.state[0];
    R* const* old = L.mem[cs];
    R* const* nw = L.mem[cs ^ 1];
    const long long q = iidx(g, i, j, k);
    double nlm, nmm;
    if (!L.state[1]) {
        nmm = mmc;
        nlm = L.c02 * mmc;
    } else {
        const double dt = *L.dtp;
        const double x = (double)(i + 1) - (double)old[2][q] * (dt * L.idx);
        const double y = (double)(j + 1) - (double)old[3][q] * (dt * L.idy);
        double z = (double)(k + 1) - (double)old[4][q] * (dt * L.idz);
        const bool pz = g.bc_z == 0;
        if (!pz) z = fmin(fmax(z, 1.0), (double)g.nz);
        const double fx0 = floor(x), fy0 = floor(y), fz0 = floor(z);
        const int x0 = (int)fx0, y0 = (int)fy0, z0 = (int)fz0;
        const double fx = x - fx0, fy = y - fy0, fz = z - fz0;
        double lm = 0.0, mm = 0.0;
#pragma unroll
        for (int dk = 0; dk <= 1; ++dk) {
            const int c = lag_wrap(z0 + dk, g.nz, pz);
#pragma unroll
            for (int dj = 0; dj <= 1; ++dj) {
                const int b = lag_wrap(y0 + dj, g.ny, true);
#pragma unroll
                for (int di = 0; di <= 1; ++di) {
                    const int a = lag_wrap(x0 + di, g.nx, true);
                    const double wgt = (di == 0 ? 1 - fx : fx) * (dj == 0 ? 1 - fy : fy) * (dk == 0 ? 1 - fz : fz);
                    const long long r = iidx(g, a, b, c);
                    lm += wgt * (double)old[0][r];
                    mm += wgt * (double)old[1][r];
                }
            }
        }
        double eps;
        if (L.memory_time > 0) {
            eps = (dt / L.memory_time) / (1 + dt / L.memory_time);
        } else if (mm > 0) {
            const double Tl = L.theta_delta * pow(fmax(lm, 1e-8 * mm) * mm, -0.125);
            eps = (dt / Tl) / (1 + dt / Tl);
        } else {
            eps = 1.0;
        }
        nlm = fmax(eps * lmc + (1 - eps) * lm, 0.0);
        nmm = eps * mmc + (1 - eps) * mm;
    }
    const R slm = R(nlm), smm = R(nmm);
    nw[0][q] = slm;
    nw[1][q] = smm;
    const long long sh = (long long)(i + 1) + (long long)ws.sx * ((j + 1) + (long long)ws.sy * (k + 1));
    nw[2][q] = ws.f[DYN_UC][sh];
    nw[3][q] = ws.f[DYN_VC][sh];
    nw[4][q] = ws.f[DYN_WC][sh];
    cs2f[pidx(g, i, j, k)] = R(smm > R(0) ? fmin(fmax((double)slm / (double)smm, 0.0), L.cs2max) : 0.0);
}

// After a commit: the written set becomes the committed one.
__global__ void lag_flip_kernel(int* state) {
    state[0] ^= 1;
    state[1] = 1;
}

// The coefficient of the committed memory into the padded field cs2f (its
// halos filled afterwards): min(C0^2, cs_max^2) before the first commit.
template <typename R>
__global__ void __launch_bounds__(256) lag_coefficient_kernel(Geo g, LagArgs<R> L, R* __restrict__ cs2f) {
    const R* lm = L.mem[L.state[0]][0];
    const R* mm = L.mem[L.state[0]][1];
    const bool init = L.state[1] != 0;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < g.nin;
         e += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(e % g.nx);
        const long long r = e / g.nx;
        const int j = (int)(r % g.ny), k = (int)(r / g.ny);
        double c;
        if (!init) c = fmin(L.c02, L.cs2max);
        else c = mm[e] > R(0) ? fmin(fmax((double)lm[e] / (double)mm[e], 0.0), L.cs2max) : 0.0;
        cs2f[pidx(g, i, j, k)] = R(c);
    }
}

// Pass 2 (_germano_pass2_body! / _germano_LM_MM): blocks of 256 cells of one
// level (grid.y = level); per block the sums of LM and MM into part.
// MODE 1 (averaging = :local, _local_cs2_body!): every interior cell's own
// clipped ratio goes to the padded field cs2f (its halos filled afterwards
// like a cell-centred field's) and no partials are written.  MODE 2 (the
// Lagrangian commit): every cell's LM and MM enter its memory update
// (lag_commit_cell), which writes cs2f.
template <typename R, int MODE = 0>
__global__ void __launch_bounds__(256) germano_pass2_kernel(Geo g, DynWs<R> ws, R inv27, R d2, R a2,
                                                            double* __restrict__ part, R* __restrict__ cs2f = nullptr,
                                                            double cs2max = 0.0, LagArgs<R> lag = {}) {
    __shared__ double slm[256], smm[256];
    const int k = blockIdx.y;
    const int e = blockIdx.x * 256 + threadIdx.x;
    double lmv = 0.0, mmv = 0.0;
    if (e < g.nx * g.ny) {
        const int i = e % g.nx, j = e / g.nx;
        R t[21];
#pragma unroll
        for (int c = 0; c < 21; ++c) t[c] = R(0);
        for (int dk = -1; dk <= 1; ++dk)
            for (int dj = -1; dj <= 1; ++dj)
                for (int di = -1; di <= 1; ++di) {
                    const long long s = (long long)(i + 1 + di) + (long long)ws.sx * ((j + 1 + dj) + (long long)ws.sy * (k + 1 + dk));
                    const R uu = ws.f[DYN_UC][s], vv = ws.f[DYN_VC][s], wv = ws.f[DYN_WC][s];
                    const R s11 = ws.f[DYN_S11][s], s22 = ws.f[DYN_S22][s], s33 = ws.f[DYN_S33][s];
                    const R s12 = ws.f[DYN_S12][s], s13 = ws.f[DYN_S13][s], s23 = ws.f[DYN_S23][s];
                    const R ms = ws.f[DYN_MS][s];
                    t[0] += uu; t[1] += vv; t[2] += wv;
                    t[3] += uu * uu; t[4] += vv * vv; t[5] += wv * wv;
                    t[6] += uu * vv; t[7] += uu * wv; t[8] += vv * wv;
                    t[9] += s11; t[10] += s22; t[11] += s33; t[12] += s12; t[13] += s13; t[14] += s23;
                    t[15] += ms * s11; t[16] += ms * s22; t[17] += ms * s33;
                    t[18] += ms * s12; t[19] += ms * s13; t[20] += ms * s23;
                }
        const R inv = inv27;
        const R Ut = t[0] * inv, Vt = t[1] * inv, Wt = t[2] * inv;
        R L11 = t[3] * inv - Ut * Ut, L22 = t[4] * inv - Vt * Vt, L33 = t[5] * inv - Wt * Wt;
        const R L12 = t[6] * inv - Ut * Vt, L13 = t[7] * inv - Ut * Wt, L23 = t[8] * inv - Vt * Wt;
        const R tr = (L11 + L22 + L33) / R(3);
        L11 -= tr; L22 -= tr; L33 -= tr;
        const R A11 = t[9] * inv, A22 = t[10] * inv, A33 = t[11] * inv;
        const R A12 = t[12] * inv, A13 = t[13] * inv, A23 = t[14] * inv;
        const R magSt = sqrt(R(2) * (A11 * A11 + A22 * A22 + A33 * A33) + R(4) * (A12 * A12 + A13 * A13 + A23 * A23));
        const R c1 = R(2) * d2 * a2 * magSt, c2 = R(2) * d2 * inv;
        const R M11 = c2 * t[15] - c1 * A11, M22 = c2 * t[16] - c1 * A22, M33 = c2 * t[17] - c1 * A33;
        const R M12 = c2 * t[18] - c1 * A12, M13 = c2 * t[19] - c1 * A13, M23 = c2 * t[20] - c1 * A23;
        lmv = L11 * M11 + L22 * M22 + L33 * M33 + R(2) * (L12 * M12 + L13 * M13 + L23 * M23);
        mmv = M11 * M11 + M22 * M22 + M33 * M33 + R(2) * (M12 * M12 + M13 * M13 + M23 * M23);
        if (MODE == 1) cs2f[pidx(g, i, j, k)] = R(mmv > 0 ? fmin(fmax(lmv / mmv, 0.0), cs2max) : 0.0);
        if (MODE == 2) lag_commit_cell<R>(g, ws, lag, cs2f, i, j, k, lmv, mmv);
    }
    if (MODE != 0) return;
    slm[threadIdx.x] = lmv;
    smm[threadIdx.x] = mmv;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            slm[threadIdx.x] += slm[threadIdx.x + s];
            smm[threadIdx.x] += smm[threadIdx.x + s];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        part[2 * ((long long)k * gridDim.x + blockIdx.x)] = slm[0];
        part[2 * ((long long)k * gridDim.x + blockIdx.x) + 1] = smm[0];
    }
}

// The plane average and the clip (_plane_cs2_body!): one thread per level.
__global__ void germano_level_kernel(int nz, int nb, const double* __restrict__ part, double cs2max,
                                     double* __restrict__ cs2) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nz) return;
    double lm = 0.0, mm = 0.0;
    for (int b = 0; b < nb; ++b) {
        lm += part[2 * ((long long)k * nb + b)];
        mm += part[2 * ((long long)k * nb + b) + 1];
    }
    cs2[k] = mm > 0 ? fmin(fmax(lm / mm, 0.0), cs2max) : 0.0;
}

// the coefficient of level k (a halo level of a periodic z wraps)
__device__ __forceinline__ double dyn_cs2_at(const Geo& g, const double* cs2, int k) {
    return cs2[k < 0 ? k + g.nz : (k >= g.nz ? k - g.nz : k)];
}
// the coefficient of cell (i, j, k): the padded per-cell field of the :local
// averaging (halos filled), else the level's
template <typename R>
__device__ __forceinline__ double dyn_cs2_cell(const Geo& g, const double* cs2, const R* cs2f, int i, int j, int k) {
    return cs2f ? (double)cs2f[pidx(g, i, j, k)] : dyn_cs2_at(g, cs2, k);
}
