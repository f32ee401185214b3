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
// at buf[l*ls + e*es]; n = 2^logn points per line, 2^lognl lines.
// LINE_FAST: consecutive threads take consecutive lines (strided lines,
// es > 1); otherwise consecutive elements of a line.  KB bounds the
// butterflies a thread holds per pass (checked by the host).  Every size is a
// power of two, so all index arithmetic is shifts and masks.
template <typename R, bool INV, bool LINE_FAST, int KB>
__device__ __forceinline__ void smem_fft(cplx<R>* buf, int logn, int lognl, int ls, int es,
                                         const cplx<R>* __restrict__ tw, int NT) {
    const int nthr = blockDim.x * blockDim.y * blockDim.z;
    const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
    const int logNT = __ffs(NT) - 1;
    for (int logNs = 0; logNs < logn;) {
        const int lr = (logn - logNs >= 2) ? 2 : 1;    // radix 4, or 2 for the last pass of an odd log n
        const int RR = 1 << lr;
        const int lognb = logn - lr, nb = 1 << lognb;  // butterflies per line
        const int total = nb << lognl;
        const int Ns = 1 << logNs;
        const int tsh = logNT - lr - logNs;            // twiddle step NT / (RR Ns) as a shift
        cplx<R> v[KB][4];
        int jj[KB], ll[KB];
#pragma unroll
        for (int s = 0; s < KB; ++s) {
            int b = tid + s * nthr;
            if (b < total) {
                int l, j;
                if (LINE_FAST) { l = b & ((1 << lognl) - 1); j = b >> lognl; }
                else { l = b >> lognb; j = b & (nb - 1); }
                jj[s] = j;
                ll[s] = l;
                cplx<R>* base = buf + l * ls;
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
                if (Ns > 1) {
#pragma unroll
                    for (int r = 1; r < 4; ++r) {
                        if (r < RR) {
                            int m = ((r * k) << tsh) & (NT - 1);
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
                int o = ((j - k) << lr) + k;
                cplx<R>* base = buf + l * ls;
                base[o * es] = y0;
                base[(o + Ns) * es] = y1;
                if (RR == 4) {
                    base[(o + 2 * Ns) * es] = y2;
                    base[(o + 3 * Ns) * es] = y3;
                }
            }
        }
        __syncthreads();
        logNs += lr;
    }
}

constexpr int FFT_KB = 4;

// ---- divergence + r2c along x --------------------------------------------------
// The neighbours i+1, j+1, k+1 are plain loads inside the domain; only the
// last cell of a row, column or level goes through the boundary map.
template <typename R, bool ANEL, bool UNI>
__device__ __forceinline__ R div_point(const Geo& g, const Met<R, UNI>& m, const R* __restrict__ us,
                                       const R* __restrict__ vs, const R* __restrict__ ws, int i, int j, int k) {
    const long long q = iidx(g, i, j, k);
    const R up = i + 1 < g.nx ? __ldg(us + q + 1) : ld_mapped_interior(g, us, i + 1, j, k, LOC_FX);
    const R vp = j + 1 < g.ny ? __ldg(vs + q + g.nx) : ld_mapped_interior(g, vs, i, j + 1, k, LOC_FY);
    const R wp = k + 1 < g.nz ? __ldg(ws + q + (long long)g.nx * g.ny) : ld_mapped_interior(g, ws, i, j, k + 1, LOC_FZ);
    const R idz = m.idz(k);
    if (ANEL) {
        const R wc = m.wc(k), wfb = m.wf(k), wft = m.wf(k + 1);
        return wc * ((up - __ldg(us + q)) * R(g.idx) + (vp - __ldg(vs + q)) * R(g.idy)) + (wft * wp - wfb * __ldg(ws + q)) * idz;
    }
    return (up - __ldg(us + q)) * R(g.idx) + (vp - __ldg(vs + q)) * R(g.idy) + (wp - __ldg(ws + q)) * idz;
}

// The r2c post-process of bin kk from the packed M-point transform of one row.
template <typename R>
__device__ __forceinline__ cplx<R> r2c_bin(const cplx<R>* rowbuf, int M, int kk, cplx<R> wv) {
    const cplx<R> a = rowbuf[kk == M ? 0 : kk];
    const cplx<R> b = rowbuf[kk == 0 ? 0 : M - kk];
    const R er = R(0.5) * (a.x + b.x), ei = R(0.5) * (a.y - b.y);
    const R orr = R(0.5) * (a.y + b.y), oi = R(-0.5) * (a.x - b.x);
    return cmk<R>(er + (wv.x * orr - wv.y * oi), ei + (wv.x * oi + wv.y * orr));
}

// One CTA transforms `rows` x-rows (row = j + ny*k).  M = nx/2; rows, M and
// ny are powers of two.
template <typename R, bool ANEL, bool UNI>
__global__ void __launch_bounds__(256) div_fftx_kernel(Geo g, const R* __restrict__ us, const R* __restrict__ vs,
                                                       const R* __restrict__ ws, cplx<R>* __restrict__ S,
                                                       const cplx<R>* __restrict__ tw, int NT, int rows) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cplx<R>* buf = reinterpret_cast<cplx<R>*>(smem_raw);
    const int M = g.nx / 2, Mh = M + 1, lM = __ffs(M) - 1, lny = __ffs(g.ny) - 1;
    const long long nrows = (long long)g.ny * g.nz;
    const long long row0 = (long long)blockIdx.x * rows;
    const int tid = threadIdx.x, nthr = blockDim.x;
    const Met<R, UNI> m(g);
    for (int e = tid; e < (rows << lM); e += nthr) {
        const int r = e >> lM, n = e & (M - 1);
        const long long row = row0 + r;
        cplx<R> z = cmk<R>(R(0), R(0));
        if (row < nrows) {
            const int j = (int)(row & (g.ny - 1)), k = (int)(row >> lny);
            z.x = div_point<R, ANEL, UNI>(g, m, us, vs, ws, 2 * n, j, k);
            z.y = div_point<R, ANEL, UNI>(g, m, us, vs, ws, 2 * n + 1, j, k);
        }
        buf[e] = z;
    }
    __syncthreads();
    smem_fft<R, false, false, FFT_KB>(buf, lM, __ffs(rows) - 1, M, 1, tw, NT);
    const int tstep = NT / g.nx;
    for (int e = tid; e < (rows << lM); e += nthr) {
        const int r = e >> lM, kk = e & (M - 1);
        const long long row = row0 + r;
        if (row < nrows) S[row * Mh + kk] = r2c_bin(buf + r * M, M, kk, tw[(kk * tstep) & (NT - 1)]);
    }
    for (int r = tid; r < rows; r += nthr) {   // the Nyquist bin, twiddle exactly -1
        const long long row = row0 + r;
        if (row < nrows) S[row * Mh + M] = r2c_bin(buf + r * M, M, M, cmk<R>(R(-1), R(0)));
    }
}

// ---- c2r along x into phi ---------------------------------------------------------
template <typename R>
__global__ void __launch_bounds__(256) ifftx_kernel(Geo g, const cplx<R>* __restrict__ S, R* __restrict__ phi,
                                                    const cplx<R>* __restrict__ tw, int NT, int rows, R scale) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cplx<R>* buf = reinterpret_cast<cplx<R>*>(smem_raw);
    const int M = g.nx / 2, Mh = M + 1, lM = __ffs(M) - 1;
    const long long nrows = (long long)g.ny * g.nz;
    const long long row0 = (long long)blockIdx.x * rows;
    const int tid = threadIdx.x, nthr = blockDim.x;
    const int tstep = NT / g.nx;
    for (int e = tid; e < (rows << lM); e += nthr) {
        const int r = e >> lM, kk = e & (M - 1);
        const long long row = row0 + r;
        cplx<R> z = cmk<R>(R(0), R(0));
        if (row < nrows) {
            cplx<R> a = S[row * Mh + kk], b = S[row * Mh + (M - kk)];
            R er = a.x + b.x, ei = a.y - b.y;
            R dr = a.x - b.x, di = a.y + b.y;
            cplx<R> wv = tw[(kk * tstep) & (NT - 1)];
            R orr = dr * wv.x + di * wv.y, oi = di * wv.x - dr * wv.y;
            z = cmk<R>(er - oi, ei + orr);
        }
        buf[e] = z;
    }
    __syncthreads();
    smem_fft<R, true, false, FFT_KB>(buf, lM, __ffs(rows) - 1, M, 1, tw, NT);
    for (int e = tid; e < (rows << lM); e += nthr) {
        const int r = e >> lM, n = e & (M - 1);
        const long long row = row0 + r;
        if (row >= nrows) continue;
        const cplx<R> z = buf[e];
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
    const int lt = __ffs(tpx) - 1;
    for (int e = tid; e < g.ny * tpx; e += nthr) {
        const int jj = e >> lt, c = e & (tpx - 1), p = p0 + c;
        buf[e] = p < Mh ? S[base + (long long)jj * Mh + p] : cmk<R>(R(0), R(0));
    }
    __syncthreads();
    smem_fft<R, MODE == 1, true, FFT_KB>(buf, __ffs(g.ny) - 1, __ffs(tpx) - 1, 1, tpx, tw, NT);
    for (int e = tid; e < g.ny * tpx; e += nthr) {
        const int jj = e >> lt, c = e & (tpx - 1), p = p0 + c;
        if (p < Mh) S[base + (long long)jj * Mh + p] = buf[e];
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
    const int lt = __ffs(tpx) - 1;
    for (int e = tid; e < g.nz * tpx; e += nthr) {
        const int kz = e >> lt, c = e & (tpx - 1), p = p0 + c;
        buf[e] = p < Mh ? S[base + kz * sk + p] : cmk<R>(R(0), R(0));
    }
    __syncthreads();
    smem_fft<R, false, true, FFT_KB>(buf, __ffs(g.nz) - 1, __ffs(tpx) - 1, 1, tpx, tw, NT);
    for (int e = tid; e < g.nz * tpx; e += nthr) {
        const int kz = e >> lt, c = e & (tpx - 1), p = p0 + c;
        if (p < Mh) {
            double lam = -(kx2[p] + ky2[j] + kz2[kz]);
            R il = lam == 0.0 ? R(0) : R(nrm / lam);
            cplx<R> z = buf[kz * tpx + c];
            buf[kz * tpx + c] = cmk<R>(z.x * il, z.y * il);
        }
    }
    __syncthreads();
    smem_fft<R, true, true, FFT_KB>(buf, __ffs(g.nz) - 1, __ffs(tpx) - 1, 1, tpx, tw, NT);
    for (int e = tid; e < g.nz * tpx; e += nthr) {
        const int kz = e >> lt, c = e & (tpx - 1), p = p0 + c;
        if (p < Mh) S[base + kz * sk + p] = buf[e];
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

// One thread per (kx, ky) column, columns flattened as col = ky * (nx/2+1) + kx
// so that a warp's loads of one level are one contiguous run.  Each lane
// streams its column through a shared-memory ring with cp.async, THOMAS_PF
// levels ahead of the recurrence, and waits (cp.async.wait_group) for exactly
// the level it needs, so the loads overlap the FP64 recurrence instead of
// exposing one memory latency per level.  The modified upper diagonal c'_k
// sits in shared memory [nz][32] after the ring, followed by the three
// coefficient vectors of the diagonals; the forward-elimination values d'_k go to
// dsc, an FP64 column scratch of the spectrum's layout (dsc may alias S when
// S is FP64: d'_k overwrites the level it came from after that level was read).
constexpr int THOMAS_PF = 16;
// the largest nz whose column state fits a CTA's 227 KB of shared memory
#define AEO_COLUMN_NZ_MAX 800

__device__ __forceinline__ void thomas_cp8(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)), "l"(src)
                 : "memory");
}
__device__ __forceinline__ void thomas_cp16(void* dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)), "l"(src)
                 : "memory");
}
template <int N>
__device__ __forceinline__ void thomas_cp(void* dst, const void* src) {
    if (N == 8) thomas_cp8(dst, src);
    else thomas_cp16(dst, src);
}
__device__ __forceinline__ void thomas_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void thomas_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// Block 0 is the mean mode; blocks 1.. hold 32 columns each.
inline unsigned thomas_blocks(const Geo& g) {
    return 1u + (unsigned)(((long long)g.ny * (g.nx / 2 + 1) + 31) / 32);
}
// the ring [THOMAS_PF][32] of cplx<double>, then c' [nz][32] and lower, upper, h [nz] each
inline size_t thomas_smem(const Geo& g) {
    return (size_t)g.nz * 35 * sizeof(double) + (size_t)THOMAS_PF * 32 * 2 * sizeof(double);
}

template <typename R>
__global__ void __launch_bounds__(32) thomas_kernel(Geo g, cplx<R>* S, cplx<double>* dsc, ColumnCoef c) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cplx<double>* ring = reinterpret_cast<cplx<double>*>(smem_raw);   // [THOMAS_PF][32], 16-byte entries
    double* cp = reinterpret_cast<double*>(ring + THOMAS_PF * 32);     // [nz][32]
    const int Mh = g.nx / 2 + 1;
    const int lane = threadIdx.x;
    const long long sk = (long long)g.ny * Mh;
    const int nz = g.nz;
    if (blockIdx.x == 0) {
        // the mean mode (_mean_mode!, src/PressureSolvers.jl:780-805), real:
        // the warp loads the column into shared memory, lane 0 runs the
        // sums and the double integration in the reference's order, the
        // warp writes the gauged profile back (the serial loops read shared
        // memory only)
        double* sv = cp;             // [nz] the column's real parts
        double* ph = sv + nz;        // [nz] the integrated profile
        double* me = ph + nz;        // [nz] measures
        double* io = me + nz;        // [nz + 1] iota
        double* ga = io + nz + 1;    // [nz] gauge weights
        for (int k = lane; k < nz; k += 32) {
            sv[k] = (double)S[k * sk].x;
            me[k] = c.meas[k];
            ga[k] = c.gauge[k];
        }
        for (int k = lane; k <= nz; k += 32) io[k] = c.iota[k];
        __syncwarp();
        if (lane == 0) {
            double mb = 0.0;
            for (int k = 0; k < nz; ++k) mb += sv[k] * me[k];
            mb /= c.meas_sum;
            double F = 0.0, acc = 0.0, prev = sv[0] - mb;
            ph[0] = 0.0;
            for (int k = 1; k < nz; ++k) {
                F += prev * me[k - 1];
                acc += F * io[k];
                prev = sv[k] - mb;
                ph[k] = acc;
            }
            double mp = 0.0;
            for (int k = 0; k < nz; ++k) mp += ph[k] * ga[k];
            sv[0] = mp / c.gauge_sum;
        }
        __syncwarp();
        const double sh = sv[0];
        for (int k = lane; k < nz; k += 32) S[k * sk] = cmk<R>(R(ph[k] - sh), R(0));
        return;
    }
    // the diagonals' per-level coefficients, staged once
    double* s_lo = cp + 32 * nz;
    double* s_up = s_lo + nz;
    double* s_hw = s_up + nz;
    for (int k = lane; k < nz; k += 32) {
        s_lo[k] = c.lower[k];
        s_up[k] = c.upper[k];
        s_hw[k] = c.hw[k];
    }
    __syncwarp();
    const long long col = (long long)(blockIdx.x - 1) * 32 + lane;
    if (col == 0 || col >= sk) return;
    const int p = (int)(col % Mh), j = (int)(col / Mh);
    const double lam = c.kx2[p] + c.ky2[j];
    constexpr int D = THOMAS_PF;
    // forward elimination: level k waits in slot k % D; the copy of level
    // k + D - 1 goes to the slot read one level earlier
    cplx<R>* rs = reinterpret_cast<cplx<R>*>(ring);   // this lane's entries at [slot * 32 + lane]
#pragma unroll
    for (int q = 0; q < D - 1; ++q) {
        if (q < nz) thomas_cp<sizeof(cplx<R>)>(rs + q * 32 + lane, S + col + q * sk);
        thomas_commit();
    }
    double cprev = 0.0, dr = 0.0, di = 0.0;
    for (int k = 0; k < nz; ++k) {
        const int kn = k + D - 1;
        if (kn < nz) thomas_cp<sizeof(cplx<R>)>(rs + (kn % D) * 32 + lane, S + col + (long long)kn * sk);
        thomas_commit();
        thomas_wait<D - 1>();   // level k has landed
        const cplx<R> s = rs[(k % D) * 32 + lane];
        const double lo = s_lo[k], up = s_up[k];
        const double b = -(lo + up) - lam * s_hw[k];
        const double den = b - lo * cprev;
        const double id = 1.0 / den;
        cprev = up * id;
        cp[k * 32 + lane] = cprev;
        dr = ((double)s.x - lo * dr) * id;   // lo = 0 at k = 0
        di = ((double)s.y - lo * di) * id;
        if (k < nz - 1) dsc[col + (long long)k * sk] = cmk<double>(dr, di);
    }
    thomas_wait<0>();
    S[col + (long long)(nz - 1) * sk] = cmk<R>(R(dr), R(di));
    // back substitution over k = nz-2 .. 0, the d' values streamed alike
    // (slot t holds level nz-2-t modulo D)
#pragma unroll
    for (int q = 0; q < D - 1; ++q) {
        const int k = nz - 2 - q;
        if (k >= 0) thomas_cp16(ring + q * 32 + lane, dsc + col + (long long)k * sk);
        thomas_commit();
    }
    for (int t = 0; t <= nz - 2; ++t) {
        const int k = nz - 2 - t;
        const int tn = t + D - 1, kn = nz - 2 - tn;
        if (kn >= 0) thomas_cp16(ring + (tn % D) * 32 + lane, dsc + col + (long long)kn * sk);
        thomas_commit();
        thomas_wait<D - 1>();
        const cplx<double> d = ring[(t % D) * 32 + lane];
        const double cc = cp[k * 32 + lane];
        dr = d.x - cc * dr;
        di = d.y - cc * di;
        S[col + (long long)k * sk] = cmk<R>(R(dr), R(di));
    }
    thomas_wait<0>();
}

// r2c of an interior source along x: pack pairs, FFT, post-process (the
// div_fftx kernel body with the source read directly).
template <typename R>
__global__ void __launch_bounds__(256) src_fftx_kernel(Geo g, const R* __restrict__ src, cplx<R>* __restrict__ S,
                                                       const cplx<R>* __restrict__ tw, int NT, int rows) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cplx<R>* buf = reinterpret_cast<cplx<R>*>(smem_raw);
    const int M = g.nx / 2, Mh = M + 1, lM = __ffs(M) - 1;
    const long long nrows = (long long)g.ny * g.nz;
    const long long row0 = (long long)blockIdx.x * rows;
    const int tid = threadIdx.x, nthr = blockDim.x;
    for (int e = tid; e < (rows << lM); e += nthr) {
        const int r = e >> lM, n = e & (M - 1);
        const long long row = row0 + r;
        cplx<R> z = cmk<R>(R(0), R(0));
        if (row < nrows) z = cmk<R>(src[row * g.nx + 2 * n], src[row * g.nx + 2 * n + 1]);
        buf[e] = z;
    }
    __syncthreads();
    smem_fft<R, false, false, FFT_KB>(buf, lM, __ffs(rows) - 1, M, 1, tw, NT);
    const int tstep = NT / g.nx;
    for (int e = tid; e < (rows << lM); e += nthr) {
        const int r = e >> lM, kk = e & (M - 1);
        const long long row = row0 + r;
        if (row < nrows) S[row * Mh + kk] = r2c_bin(buf + r * M, M, kk, tw[(kk * tstep) & (NT - 1)]);
    }
    for (int r = tid; r < rows; r += nthr) {   // the Nyquist bin
        const long long row = row0 + r;
        if (row < nrows) S[row * Mh + M] = r2c_bin(buf + r * M, M, M, tw[(M * tstep) & (NT - 1)]);
    }
}
