// aeo_init.cuh -- the spectral isotropic initial field on the device.
//
// isotropic_turbulence_field! (src/operators/spectra.jl:312-343): every
// mode's complex normal triple comes from a SplitMix64 hash of (seed, mode)
// (_splitmix, _mode_key, _mode_normals, :257-275), projected solenoidally,
// scaled by sqrt(E(k) dV / (4 pi k^2)) with the Passot-Pouquet spectrum
// (:248-253) and phase-shifted to each component's first staggered node.
// iso_modes_kernel writes the half spectrum (kx in [0, nx/2]) of one
// component; the library's own inverse transforms (z, y, then c2r along x)
// turn it into the field.
#pragma once

#include "aeo_fft.cuh"

__device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
    x += 0x9e3779b97f4a7c15ULL;
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ULL;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebULL;
    return x ^ (x >> 31);
}
__device__ __forceinline__ double unit53(uint64_t h) { return (double)((h >> 11) + 1) * 0x1.0p-53; }

struct IsoParams {
    double u_rms, k_peak, kmax, lx, ly, lz;
    double x1, y1, z1;   // the component's first node
    unsigned long long seed;
    int comp;            // 0 u, 1 v, 2 w
};

__device__ __forceinline__ int fftfreq_i(int a, int n) { return a < (n + 1) / 2 ? a : a - n; }

template <typename R>
__global__ void iso_modes_kernel(Geo g, cplx<R>* __restrict__ S, IsoParams p) {
    const int Mh = g.nx / 2 + 1;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long total = (long long)Mh * g.ny * g.nz;
    if (t >= total) return;
    const int a = (int)(t % Mh), b = (int)((t / Mh) % g.ny), c = (int)(t / ((long long)Mh * g.ny));
    const int m1 = a, m2 = fftfreq_i(b, g.ny), m3 = fftfreq_i(c, g.nz);
    cplx<R> out = cmk<R>(R(0), R(0));
    const bool keep = 2 * abs(m1) < g.nx && 2 * abs(m2) < g.ny && 2 * abs(m3) < g.nz && !(m1 == 0 && m2 == 0 && m3 == 0);
    if (keep) {
        const double c1 = 2 * M_PI / p.lx, c2 = 2 * M_PI / p.ly, c3 = 2 * M_PI / p.lz;
        const double dV = c1 * c2 * c3;
        const double k1 = c1 * m1, k2 = c2 * m2, k3 = c3 * m3;
        const double kk2 = k1 * k1 + k2 * k2 + k3 * k3;
        const double kk = sqrt(kk2);
        if (kk <= p.kmax) {
            const bool canon = m3 > 0 || (m3 == 0 && (m2 > 0 || (m2 == 0 && m1 > 0)));
            const int s = canon ? 1 : -1;
            const uint64_t key = splitmix64(splitmix64(splitmix64(splitmix64((uint64_t)p.seed) ^ (uint64_t)(int64_t)(s * m1)) ^
                                                       (uint64_t)(int64_t)(s * m2)) ^
                                            (uint64_t)(int64_t)(s * m3));
            double rr[3], ri[3];
            for (int j = 0; j < 3; ++j) {
                const uint64_t ha = splitmix64(key + (uint64_t)(2 * (j + 1) - 1));
                const uint64_t hb = splitmix64(key + (uint64_t)(2 * (j + 1)));
                const double rho = sqrt(-2 * log(unit53(ha)));
                const double phi = 2 * M_PI * unit53(hb);
                rr[j] = rho * cos(phi) / sqrt(2.0);
                ri[j] = rho * sin(phi) / sqrt(2.0);
            }
            const double kc[3] = {s * k1, s * k2, s * k3};
            const double krr = (kc[0] * rr[0] + kc[1] * rr[1] + kc[2] * rr[2]) / kk2;
            const double kri = (kc[0] * ri[0] + kc[1] * ri[1] + kc[2] * ri[2]) / kk2;
            double pr = rr[p.comp] - kc[p.comp] * krr, pi = ri[p.comp] - kc[p.comp] * kri;
            if (!canon) pi = -pi;
            const double E = 16 * sqrt(2 / M_PI) * p.u_rms * p.u_rms * (kk2 * kk2) /
                             (p.k_peak * p.k_peak * p.k_peak * p.k_peak * p.k_peak) *
                             exp(-2 * (kk / p.k_peak) * (kk / p.k_peak));
            const double amp = sqrt(fmax(E, 0.0) * dV / (4 * M_PI * kk2));
            const double ph = k1 * p.x1 + k2 * p.y1 + k3 * p.z1;
            const double cr = cos(ph), ci = sin(ph);
            out = cmk<R>(R(amp * (pr * cr - pi * ci)), R(amp * (pr * ci + pi * cr)));
        }
    }
    S[t] = out;
}

// inverse complex transform along z of the spectrum (the field generator's z pass)
template <typename R>
__global__ void __launch_bounds__(FFT_THREADS(R), FFT_MINB(R)) fftz_inv_kernel(Geo g, cplx<R>* __restrict__ S, const cplx<R>* __restrict__ tw,
                                                       int NT, int tpx) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cplx<R>* buf = reinterpret_cast<cplx<R>*>(smem_raw);
    const int Mh = g.nx / 2 + 1;
    const int j = blockIdx.y, p0 = blockIdx.x * tpx;
    const long long sk = (long long)g.ny * Mh;
    const long long base = (long long)j * Mh;
    const int lt = __ffs(tpx) - 1;
#pragma unroll 16
    for (int e = threadIdx.x; e < g.nz * tpx; e += blockDim.x) {
        const int kz = e >> lt, c = e & (tpx - 1), p = p0 + c;
        buf[e] = p < Mh ? S[base + kz * sk + p] : cmk<R>(R(0), R(0));
    }
    __syncthreads();
    smem_fft<R, true, true>(buf, __ffs(g.nz) - 1, __ffs(tpx) - 1, 1, tpx, tw, NT);
    for (int e = threadIdx.x; e < g.nz * tpx; e += blockDim.x) {
        const int kz = e >> lt, c = e & (tpx - 1), p = p0 + c;
        if (p < Mh) S[base + kz * sk + p] = buf[e];
    }
}

template <typename R>
__global__ void interior_to_padded_kernel(Geo g, const R* __restrict__ a, R* __restrict__ b, R scale) {
    int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, k = blockIdx.z;
    if (i < g.nx) b[pidx(g, i, j, k)] = a[iidx(g, i, j, k)] * scale;
}

template <typename R>
__global__ void scale_padded_kernel(Geo g, R* __restrict__ a, double s) {
    int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, k = blockIdx.z;
    if (i < g.nx) {
        long long q = pidx(g, i, j, k);
        a[q] = R((double)a[q] * s);
    }
}

// per level: sum of u^2 + v^2 + w^2 (the rms of the generated field)
template <typename R>
__global__ void __launch_bounds__(256) sumsq_levels_kernel(Geo g, const R* __restrict__ u, const R* __restrict__ v,
                                                           const R* __restrict__ w, double* __restrict__ part) {
    __shared__ double red[256];
    const int k = blockIdx.x;
    double acc = 0.0;
    for (int e = threadIdx.x; e < g.nx * g.ny; e += blockDim.x) {
        const long long q = pidx(g, e % g.nx, e / g.nx, k);
        const double a = u[q], b = v[q], c = w[q];
        acc += a * a + b * b + c * c;
    }
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[k] = red[0];
}
