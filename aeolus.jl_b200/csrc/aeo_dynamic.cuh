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
// padded field with filled halos) and nu_t = cs2(i, j, k) Delta^2 |S|.
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

// Pass 2 (_germano_pass2_body! / _germano_LM_MM): blocks of 256 cells of one
// level (grid.y = level); per block the sums of LM and MM into part.
// LOCAL (averaging = :local, _local_cs2_body!): every interior cell's own
// clipped ratio goes to the padded field cs2f (its halos filled afterwards
// like a cell-centred field's) and no partials are written.
template <typename R, bool LOCAL = false>
__global__ void __launch_bounds__(256) germano_pass2_kernel(Geo g, DynWs<R> ws, R inv27, R d2, R a2,
                                                            double* __restrict__ part, R* __restrict__ cs2f = nullptr,
                                                            double cs2max = 0.0) {
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
        if (LOCAL) cs2f[pidx(g, i, j, k)] = R(mmv > 0 ? fmin(fmax(lmv / mmv, 0.0), cs2max) : 0.0);
    }
    if (LOCAL) return;
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
