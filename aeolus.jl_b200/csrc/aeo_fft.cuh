// aeo_fft.cuh -- the projection's pressure solve as batched shared-memory FFT
// kernels and a batched column (Thomas) solve.
//
// Reference: FFTPoissonSolver (src/PressureSolvers.jl:103-174) and
// ColumnTridiagonalSolver (src/PressureSolvers.jl:591-805), whose FFTW plans
// (src/operators/fftw_planning.jl:258) are replaced by these kernels.  The
// spectrum S is stored [kz][ky][kx] with kx in [0, nx/2] (the r2c half
// spectrum of x), complex of the state precision.
//
//   div_fftx   divergence of the predicted velocity (plain, or W-weighted for
//              the sound-proof core) fused with the r2c transform along x
//              (src/FiniteVolume.jl:1869-1888, src/Anelastic.jl:1110-1120)
//   ffty       complex transform along y (forward or inverse)
//   fftz_solve periodic z: forward transform, scale by nrm/lambda (zero mean
//              mode), inverse transform -- one pass (src/PressureSolvers.jl:128-138,
//              :162-174)
//   thomas     walls in z: per horizontal wavenumber the tridiagonal solve in
//              FP64 with the factors recomputed on the fly, the mean mode
//              integrated (src/PressureSolvers.jl:650-661, :754-805)
//   ifftx      c2r along x into the potential phi (interior array)
//
// The transforms are Stockham autosort FFTs (radix-4 passes, a radix-2 pass
// when log2 n is odd) on lines held in shared memory; twiddles come from one
// table tw[m] = exp(-2 pi i m / NT) with NT the largest transform length.
#pragma once

#include "aeo_common.cuh"

// Batched in-place Stockham FFT in shared memory.  Line l, element e lives
// at buf[l*ls + e*es].  LINE_FAST: consecutive threads take consecutive
// lines (strided lines, es > 1); otherwise consecutive elements of a line.
// KB bounds the butterflies a thread holds per pass (checked by the host).
template <typename R, bool INV, bool LINE_FAST, int KB>
__device__ __forceinline__ void smem_fft(cplx<R>* buf, int n, int nlines, int ls, int es,
                                         const cplx<R>* __restrict__ tw, int NT) {
    const int nthr = blockDim.x * blockDim.y * blockDim.z;
    const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
    int Ns = 1;
    while (Ns < n) {
        const int RR = (n / Ns >= 4) ? 4 : 2;
        const int nb = n / RR;          // butterflies per line
        const int total = nb * nlines;
        cplx<R> v[KB][4];
        int jj[KB], ll[KB];
#pragma unroll
        for (int s = 0; s < KB; ++s) {
            int b = tid + s * nthr;
            if (b < total) {
                int l, j;
                if (LINE_FAST) { l = b % nlines; j = b / nlines; }
                else { l = b / nb; j = b % nb; }
                jj[s] = j;
                ll[s] = l;
                cplx<R>* base = buf + (long long)l * ls;
                if (RR == 4) {
#pragma unroll
                    for (int r = 0; r < 4; ++r) v[s][r] = base[(j + r * nb) * es];
                } else {
                    v[s][0] = base[j * es];
                    v[s][1] = base[(j + nb) * es];
                }
            }
        }
        __syncthreads();
#pragma unroll
        for (int s = 0; s < KB; ++s) {
            int b = tid + s * nthr;
            if (b < total) {
                int j = jj[s], l = ll[s];
                int k = j & (Ns - 1);
                int tstep = NT / (RR * Ns);
                if (Ns > 1) {
#pragma unroll
                    for (int r = 1; r < 4; ++r) {
                        if (r < RR) {
                            int m = (r * k * tstep) & (NT - 1);
                            cplx<R> wv = tw[m];
                            if (INV) wv.y = -wv.y;
                            v[s][r] = cmul(v[s][r], wv);
                        }
                    }
                }
                cplx<R> y0, y1, y2, y3;
                if (RR == 4) {
                    cplx<R> b0 = cadd(v[s][0], v[s][2]), b1 = csub(v[s][0], v[s][2]);
                    cplx<R> b2 = cadd(v[s][1], v[s][3]), b3 = csub(v[s][1], v[s][3]);
                    // forward: y1 = b1 - i b3, y3 = b1 + i b3; inverse the opposite
                    cplx<R> ib3 = cmk<R>(-b3.y, b3.x);
                    y0 = cadd(b0, b2);
                    y2 = csub(b0, b2);
                    y1 = INV ? cadd(b1, ib3) : csub(b1, ib3);
                    y3 = INV ? csub(b1, ib3) : cadd(b1, ib3);
                } else {
                    y0 = cadd(v[s][0], v[s][1]);
                    y1 = csub(v[s][0], v[s][1]);
                    y2 = y0;
                    y3 = y1;
                }
                int o = (j - k) * RR + k;
                cplx<R>* base = buf + (long long)l * ls;
                base[o * es] = y0;
                base[(o + Ns) * es] = y1;
                if (RR == 4) {
                    base[(o + 2 * Ns) * es] = y2;
                    base[(o + 3 * Ns) * es] = y3;
                }
            }
        }
        __syncthreads();
        Ns *= RR;
    }
}

constexpr int FFT_KB = 4;

// ---- divergence + r2c along x --------------------------------------------------
template <typename R, bool ANEL, bool UNI>
__device__ __forceinline__ R div_point(const Geo& g, const R* __restrict__ us, const R* __restrict__ vs,
                                       const R* __restrict__ ws, int i, int j, int k) {
    const long long q = iidx(g, i, j, k);
    R up = ld_mapped_interior(g, us, i + 1, j, k, LOC_FX);
    R vp = ld_mapped_interior(g, vs, i, j + 1, k, LOC_FY);
    R wp = ld_mapped_interior(g, ws, i, j, k + 1, LOC_FZ);
    R idz = UNI ? R(g.idz) : R(lvl(g.idzc, k));
    if (ANEL) {
        R wc = R(lvl(g.wc, k)), wfb = R(lvl(g.wf, k)), wft = R(lvl(g.wf, k + 1));
        return wc * ((up - __ldg(us + q)) * R(g.idx) + (vp - __ldg(vs + q)) * R(g.idy)) + (wft * wp - wfb * __ldg(ws + q)) * idz;
    }
    return (up - __ldg(us + q)) * R(g.idx) + (vp - __ldg(vs + q)) * R(g.idy) + (wp - __ldg(ws + q)) * idz;
}

// One CTA transforms `rows` x-rows (row = j + ny*k).  M = nx/2.
template <typename R, bool ANEL, bool UNI>
__global__ void __launch_bounds__(256) div_fftx_kernel(Geo g, const R* __restrict__ us, const R* __restrict__ vs,
                                                       const R* __restrict__ ws, cplx<R>* __restrict__ S,
                                                       const cplx<R>* __restrict__ tw, int NT, int rows) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cplx<R>* buf = reinterpret_cast<cplx<R>*>(smem_raw);
    const int M = g.nx / 2, Mh = M + 1;
    const long long nrows = (long long)g.ny * g.nz;
    const long long row0 = (long long)blockIdx.x * rows;
    const int tid = threadIdx.x, nthr = blockDim.x;
    for (int e = tid; e < rows * M; e += nthr) {
        int r = e / M, n = e % M;
        long long row = row0 + r;
        cplx<R> z = cmk<R>(R(0), R(0));
        if (row < nrows) {
            int j = (int)(row % g.ny), k = (int)(row / g.ny);
            z.x = div_point<R, ANEL, UNI>(g, us, vs, ws, 2 * n, j, k);
            z.y = div_point<R, ANEL, UNI>(g, us, vs, ws, 2 * n + 1, j, k);
        }
        buf[r * M + n] = z;
    }
    __syncthreads();
    smem_fft<R, false, false, FFT_KB>(buf, M, rows, M, 1, tw, NT);
    const int tstep = NT / g.nx;
    for (int e = tid; e < rows * Mh; e += nthr) {
        int r = e / Mh, kk = e % Mh;
        long long row = row0 + r;
        if (row >= nrows) continue;
        cplx<R> a = buf[r * M + (kk == M ? 0 : kk)];
        cplx<R> b = buf[r * M + (kk == 0 ? 0 : M - kk)];
        R er = R(0.5) * (a.x + b.x), ei = R(0.5) * (a.y - b.y);
        R orr = R(0.5) * (a.y + b.y), oi = R(-0.5) * (a.x - b.x);
        cplx<R> wv = tw[(kk * tstep) & (NT - 1)];
        if (kk == M) wv = cmk<R>(R(-1), R(0));
        cplx<R> X = cmk<R>(er + (wv.x * orr - wv.y * oi), ei + (wv.x * oi + wv.y * orr));
        S[row * Mh + kk] = X;
    }
}

// ---- c2r along x into phi ---------------------------------------------------------
template <typename R>
__global__ void __launch_bounds__(256) ifftx_kernel(Geo g, const cplx<R>* __restrict__ S, R* __restrict__ phi,
                                                    const cplx<R>* __restrict__ tw, int NT, int rows, R scale) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cplx<R>* buf = reinterpret_cast<cplx<R>*>(smem_raw);
    const int M = g.nx / 2, Mh = M + 1;
    const long long nrows = (long long)g.ny * g.nz;
    const long long row0 = (long long)blockIdx.x * rows;
    const int tid = threadIdx.x, nthr = blockDim.x;
    const int tstep = NT / g.nx;
    for (int e = tid; e < rows * M; e += nthr) {
        int r = e / M, kk = e % M;
        long long row = row0 + r;
        cplx<R> z = cmk<R>(R(0), R(0));
        if (row < nrows) {
            cplx<R> a = S[row * Mh + kk], b = S[row * Mh + (M - kk)];
            R er = a.x + b.x, ei = a.y - b.y;
            R dr = a.x - b.x, di = a.y + b.y;
            cplx<R> wv = tw[(kk * tstep) & (NT - 1)];
            R orr = dr * wv.x + di * wv.y, oi = di * wv.x - dr * wv.y;
            z = cmk<R>(er - oi, ei + orr);
        }
        buf[r * M + kk] = z;
    }
    __syncthreads();
    smem_fft<R, true, false, FFT_KB>(buf, M, rows, M, 1, tw, NT);
    for (int e = tid; e < rows * M; e += nthr) {
        int r = e / M, n = e % M;
        long long row = row0 + r;
        if (row >= nrows) continue;
        cplx<R> z = buf[r * M + n];
        phi[row * g.nx + 2 * n] = z.x * scale;
        phi[row * g.nx + 2 * n + 1] = z.y * scale;
    }
}

// ---- complex transform along y (MODE 0 forward, 1 inverse) ----------------------
// CTA: tile of `tpx` consecutive kx columns at one kz, all ky.
template <typename R, int MODE>
__global__ void __launch_bounds__(256) ffty_kernel(Geo g, cplx<R>* __restrict__ S, const cplx<R>* __restrict__ tw,
                                                   int NT, int tpx) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cplx<R>* buf = reinterpret_cast<cplx<R>*>(smem_raw);
    const int Mh = g.nx / 2 + 1;
    const int k = blockIdx.y, p0 = blockIdx.x * tpx;
    const int tid = threadIdx.x, nthr = blockDim.x;
    const long long base = (long long)k * g.ny * Mh;
    for (int e = tid; e < g.ny * tpx; e += nthr) {
        int jj = e / tpx, c = e % tpx, p = p0 + c;
        buf[jj * tpx + c] = p < Mh ? S[base + (long long)jj * Mh + p] : cmk<R>(R(0), R(0));
    }
    __syncthreads();
    smem_fft<R, MODE == 1, true, FFT_KB>(buf, g.ny, tpx, 1, tpx, tw, NT);
    for (int e = tid; e < g.ny * tpx; e += nthr) {
        int jj = e / tpx, c = e % tpx, p = p0 + c;
        if (p < Mh) S[base + (long long)jj * Mh + p] = buf[jj * tpx + c];
    }
}

// ---- periodic z: forward, scale by nrm/lambda, inverse -------------------------
template <typename R>
__global__ void __launch_bounds__(256) fftz_solve_kernel(Geo g, cplx<R>* __restrict__ S, const cplx<R>* __restrict__ tw,
                                                         int NT, int tpx, const double* __restrict__ kx2,
                                                         const double* __restrict__ ky2, const double* __restrict__ kz2,
                                                         double nrm) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cplx<R>* buf = reinterpret_cast<cplx<R>*>(smem_raw);
    const int Mh = g.nx / 2 + 1;
    const int j = blockIdx.y, p0 = blockIdx.x * tpx;
    const int tid = threadIdx.x, nthr = blockDim.x;
    const long long sk = (long long)g.ny * Mh;
    const long long base = (long long)j * Mh;
    for (int e = tid; e < g.nz * tpx; e += nthr) {
        int kz = e / tpx, c = e % tpx, p = p0 + c;
        buf[kz * tpx + c] = p < Mh ? S[base + kz * sk + p] : cmk<R>(R(0), R(0));
    }
    __syncthreads();
    smem_fft<R, false, true, FFT_KB>(buf, g.nz, tpx, 1, tpx, tw, NT);
    for (int e = tid; e < g.nz * tpx; e += nthr) {
        int kz = e / tpx, c = e % tpx, p = p0 + c;
        if (p < Mh) {
            double lam = -(kx2[p] + ky2[j] + kz2[kz]);
            R il = lam == 0.0 ? R(0) : R(nrm / lam);
            cplx<R> z = buf[kz * tpx + c];
            buf[kz * tpx + c] = cmk<R>(z.x * il, z.y * il);
        }
    }
    __syncthreads();
    smem_fft<R, true, true, FFT_KB>(buf, g.nz, tpx, 1, tpx, tw, NT);
    for (int e = tid; e < g.nz * tpx; e += nthr) {
        int kz = e / tpx, c = e % tpx, p = p0 + c;
        if (p < Mh) S[base + kz * sk + p] = buf[kz * tpx + c];
    }
}

// ---- walls in z: the batched column solve ------------------------------------------
struct ColumnCoef {
    const double* lower;   // a_k (0 at k = 0)
    const double* upper;   // c_k (0 at k = nz-1)
    const double* hw;      // h_k
    const double* meas;    // m_k
    const double* iota;    // iota_k (nz+1)
    const double* gauge;   // gauge_k
    double meas_sum, gauge_sum;
    const double* kx2;     // r2r eigenvalues, kx in [0, nx/2]
    const double* ky2;     // ky in [0, ny)
};

// One warp per CTA: lane = kx, blockIdx.y = ky.  dsc: FP64 scratch column
// storage (nz x ny x Mh complex) holding the forward-elimination values.
template <typename R>
__global__ void __launch_bounds__(32) thomas_kernel(Geo g, cplx<R>* S, cplx<double>* dsc,  // S and dsc alias in FP64
                                                    ColumnCoef c) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double* cp = reinterpret_cast<double*>(smem_raw);   // [nz][32]
    const int Mh = g.nx / 2 + 1;
    const int lane = threadIdx.x;
    const int p = blockIdx.x * 32 + lane, j = blockIdx.y;
    if (p >= Mh) return;
    const long long sk = (long long)g.ny * Mh;
    const long long base = (long long)j * Mh + p;
    const int nz = g.nz;
    if (p == 0 && j == 0) {
        // the mean mode (_mean_mode!, src/PressureSolvers.jl:780-805), real
        double mb = 0.0;
        for (int k = 0; k < nz; ++k) mb += (double)S[base + k * sk].x * c.meas[k];
        mb /= c.meas_sum;
        double F = 0.0, ph = 0.0, prev = (double)S[base].x - mb;
        dsc[base].x = 0.0;
        for (int k = 1; k < nz; ++k) {
            F += prev * c.meas[k - 1];
            ph += F * c.iota[k];
            prev = (double)S[base + k * sk].x - mb;
            dsc[base + k * sk].x = ph;
        }
        double mp = 0.0;
        for (int k = 0; k < nz; ++k) mp += dsc[base + k * sk].x * c.gauge[k];
        double sh = mp / c.gauge_sum;
        for (int k = 0; k < nz; ++k) S[base + k * sk] = cmk<R>(R(dsc[base + k * sk].x - sh), R(0));
        return;
    }
    const double lam = c.kx2[p] + c.ky2[j];
    double cprev = 0.0;
    double dr = 0.0, di = 0.0;
    for (int k = 0; k < nz; ++k) {
        double lo = __ldg(c.lower + k), up = __ldg(c.upper + k);
        double b = -(lo + up) - lam * __ldg(c.hw + k);
        double den = b - lo * cprev;
        double id = 1.0 / den;
        cprev = up / den;
        cp[k * 32 + lane] = cprev;
        cplx<R> s = S[base + k * sk];
        if (k == 0) {
            dr = (double)s.x * id;
            di = (double)s.y * id;
        } else {
            dr = ((double)s.x - lo * dr) * id;
            di = ((double)s.y - lo * di) * id;
        }
        dsc[base + k * sk] = cmk<double>(dr, di);
    }
    S[base + (nz - 1) * sk] = cmk<R>(R(dr), R(di));
    for (int k = nz - 2; k >= 0; --k) {
        cplx<double> d = dsc[base + k * sk];
        double cc = cp[k * 32 + lane];
        dr = d.x - cc * dr;
        di = d.y - cc * di;
        S[base + k * sk] = cmk<R>(R(dr), R(di));
    }
}

// r2c of an interior source along x: pack pairs, FFT, post-process (the
// div_fftx kernel body with the source read directly).
template <typename R>
__global__ void __launch_bounds__(256) src_fftx_kernel(Geo g, const R* __restrict__ src, cplx<R>* __restrict__ S,
                                                       const cplx<R>* __restrict__ tw, int NT, int rows) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cplx<R>* buf = reinterpret_cast<cplx<R>*>(smem_raw);
    const int M = g.nx / 2, Mh = M + 1;
    const long long nrows = (long long)g.ny * g.nz;
    const long long row0 = (long long)blockIdx.x * rows;
    for (int e = threadIdx.x; e < rows * M; e += blockDim.x) {
        int r = e / M, n = e % M;
        long long row = row0 + r;
        cplx<R> z = cmk<R>(R(0), R(0));
        if (row < nrows) z = cmk<R>(src[row * g.nx + 2 * n], src[row * g.nx + 2 * n + 1]);
        buf[r * M + n] = z;
    }
    __syncthreads();
    smem_fft<R, false, false, FFT_KB>(buf, M, rows, M, 1, tw, NT);
    const int tstep = NT / g.nx;
    for (int e = threadIdx.x; e < rows * Mh; e += blockDim.x) {
        int r = e / Mh, kk = e % Mh;
        long long row = row0 + r;
        if (row >= nrows) continue;
        cplx<R> a = buf[r * M + (kk == M ? 0 : kk)];
        cplx<R> b = buf[r * M + (kk == 0 ? 0 : M - kk)];
        R er = R(0.5) * (a.x + b.x), ei = R(0.5) * (a.y - b.y);
        R orr = R(0.5) * (a.y + b.y), oi = R(-0.5) * (a.x - b.x);
        cplx<R> wv = tw[(kk * tstep) & (NT - 1)];
        S[row * Mh + kk] = cmk<R>(er + (wv.x * orr - wv.y * oi), ei + (wv.x * oi + wv.y * orr));
    }
}
