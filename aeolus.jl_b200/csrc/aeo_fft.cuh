// aeo_fft.cuh -- the projection's pressure solve as batched shared-memory FFT
// kernels and a batched column (Thomas) solve.
//
// Reference: FFTPoissonSolver (src/PressureSolvers.jl:103-174) and
// ColumnTridiagonalSolver (src/PressureSolvers.jl:591-805), whose FFTW plans
// (src/operators/fftw_planning.jl:258) are replaced by these kernels.  The
// spectrum S is stored [kz][ky][kx] with kx in [0, nx/2] (the r2c half
// spectrum of x), complex of the state precision.
//
//   div        divergence of the predicted velocity (plain, or W-weighted for
//              the sound-proof core), one cell per thread
//              (src/FiniteVolume.jl:1869-1888, src/Anelastic.jl:1110-1120)
//   src_fftx   r2c transform along x of an interior source (the divergence)
//   ffty       complex transform along y (forward or inverse)
//   fftz_solve periodic z: forward transform, scale by nrm/lambda (zero mean
//              mode), inverse transform -- one pass (src/PressureSolvers.jl:128-138,
//              :162-174)
//   thomas     walls in z: per horizontal wavenumber the tridiagonal solve in
//              FP64 with the factors recomputed on the fly, the mean mode
//              integrated (src/PressureSolvers.jl:650-661, :754-805)
//   ifftx      c2r along x into the potential phi (interior array)
//
// The transforms are Stockham autosort FFTs on lines held in shared memory,
// each pass an in-register DFT of radix 16, 8 or 4; the inter-pass twiddles
// come from one table tw[m] = exp(-2 pi i m / NT) with NT the largest
// transform length.
#pragma once

#include "aeo_common.cuh"

// Launch shape of every transform CTA: a CTA holds at most 2048 points (the
// host sizes rows / column tiles so), PTS per thread: 128 threads x 16 points
// (radix up to 16) in FP32, 256 x 8 (radix up to 8) in FP64, where 16
// complex doubles would not fit the register budget.
template <typename R>
struct FftCfg {
    static constexpr int THREADS = sizeof(R) == 8 ? 256 : 128;
    static constexpr int PTS = 2048 / THREADS;
    static constexpr int MAXLR = PTS == 16 ? 4 : 3;
    static constexpr int MINB = sizeof(R) == 8 ? 2 : 4;   // CTAs per SM compiled for (128 registers)
};
#define FFT_THREADS(R) (FftCfg<R>::THREADS)
#define FFT_MINB(R) (FftCfg<R>::MINB)

// exp(-2 pi i m / 16), m = 0..15: the exact values of cos and sin at
// multiples of pi/8 (cos pi/8 = sqrt(2 + sqrt 2)/2, cos pi/4 = sqrt(2)/2,
// cos 3pi/8 = sqrt(2 - sqrt 2)/2), so every in-register DFT of R | 16 points
// uses constants, not table loads.
__device__ __forceinline__ double w16_re(int m) {
    constexpr double c[16] = {1.0, 0.92387953251128675613, 0.70710678118654752440, 0.38268343236508977173,
                              0.0, -0.38268343236508977173, -0.70710678118654752440, -0.92387953251128675613,
                              -1.0, -0.92387953251128675613, -0.70710678118654752440, -0.38268343236508977173,
                              0.0, 0.38268343236508977173, 0.70710678118654752440, 0.92387953251128675613};
    return c[m & 15];
}
__device__ __forceinline__ double w16_im(int m) { return -w16_re((m + 12) & 15); }   // -sin(2 pi m / 16)

// In-register DFT of R points (natural order in and out), decimation in time:
// y_q = sum_r v_r W_R^{rq}, W_R = exp(-+2 pi i / R).
template <typename R, int N, bool INV>
__device__ __forceinline__ void dft_reg(cplx<R>* v) {
    if constexpr (N == 1) {
        return;
    } else if constexpr (N == 2) {
        const cplx<R> a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    } else {
        constexpr int H = N / 2;
        cplx<R> e[H], o[H];
#pragma unroll
        for (int i = 0; i < H; ++i) {
            e[i] = v[2 * i];
            o[i] = v[2 * i + 1];
        }
        dft_reg<R, H, INV>(e);
        dft_reg<R, H, INV>(o);
#pragma unroll
        for (int k = 0; k < H; ++k) {
            cplx<R> t = o[k];
            const int m = k * (16 / N);              // W_N^k = W_16^m
            if (m == 4) {                            // -i (forward) / +i (inverse)
                t = INV ? cmk<R>(-t.y, t.x) : cmk<R>(t.y, -t.x);
            } else if (m != 0) {
                const R wr = R(w16_re(m)), wi = INV ? R(-w16_im(m)) : R(w16_im(m));
                t = cmk<R>(t.x * wr - t.y * wi, t.x * wi + t.y * wr);
            }
            v[k] = cadd(e[k], t);
            v[k + H] = csub(e[k], t);
        }
    }
}

// Row-contiguous lines (es = 1) are stored skewed, element e at e + e/16, so
// that the stride-R writes of a radix-R pass fall in distinct banks; a line
// of M elements then spans M + M/16 slots; one more holds a raw half
// spectrum's M + 1 bins before the c2r pre-process.
__host__ __device__ __forceinline__ int xrow(int M) { return M + (M >> 4) + 1; }
template <bool SKEW>
__device__ __forceinline__ int sk16(int e) { return SKEW ? e + (e >> 4) : e; }

// One Stockham pass of radix 2^LR over all lines: butterfly j of a line reads
// x[j + r n/R], applies the twiddles W_{R Ns}^{r k} (k = j mod Ns), does the
// R-point DFT in registers and writes y[(j - k) R + k + q Ns].  A thread
// holds FftCfg::PTS / R butterflies; everything but the in-place stores happens
// before the barrier, so only the results and their offsets live across it.
template <typename R, int LR, bool INV, bool LINE_FAST, bool SKEW = !LINE_FAST>
__device__ __forceinline__ void fft_pass(cplx<R>* buf, int logn, int lognl, int ls, int es, int logNs,
                                         const cplx<R>* __restrict__ tw, int NT, int logNT) {
    constexpr int RR = 1 << LR, KB = FftCfg<R>::PTS / RR;
    const int nthr = blockDim.x;
    const int tid = threadIdx.x;
    const int lognb = logn - LR, nb = 1 << lognb;
    const int total = nb << lognl;
    const int Ns = 1 << logNs;
    const int tsh = logNT - LR - logNs;
    asm volatile("" ::: "memory");   // keep this variant's loads below the radix dispatch
    cplx<R> v[KB][RR];
    int oo[KB];   // output offset of butterfly s (-1: none)
#pragma unroll
    for (int s = 0; s < KB; ++s) {
        const int b = tid + s * nthr;
        oo[s] = -1;
        if (b < total) {
            int l, j;
            if (LINE_FAST) { l = b & ((1 << lognl) - 1); j = b >> lognl; }
            else { l = b >> lognb; j = b & (nb - 1); }
            const int k = j & (Ns - 1);
            const cplx<R>* base = buf + l * ls;
            v[s][0] = base[sk16<SKEW>(j) * es];
#pragma unroll
            for (int r = 1; r < RR; ++r) {
                v[s][r] = base[sk16<SKEW>(j + r * nb) * es];
                if (logNs > 0) {
                    cplx<R> wv = tw[((r * k) << tsh) & (NT - 1)];
                    if (INV) wv.y = -wv.y;
                    v[s][r] = cmul(v[s][r], wv);
                }
            }
            dft_reg<R, RR, INV>(v[s]);
            // SKEW: the line offset and the first output index, packed (both < 2^15)
            oo[s] = SKEW ? ((l * ls) | ((((j - k) << LR) + k) << 16)) : l * ls + (((j - k) << LR) + k) * es;
        }
    }
    __syncthreads();
    const int st = Ns * es;
#pragma unroll
    for (int s = 0; s < KB; ++s) {
        if (oo[s] >= 0) {
            if (SKEW) {
                const int lo = oo[s] & 0xFFFF, o = oo[s] >> 16;
#pragma unroll
                for (int q = 0; q < RR; ++q) buf[lo + sk16<true>(o + q * Ns)] = v[s][q];
            } else {
#pragma unroll
                for (int q = 0; q < RR; ++q) buf[oo[s] + q * st] = v[s][q];
            }
        }
    }
    __syncthreads();
}

// Batched in-place Stockham FFT in shared memory.  Line l, element e lives
// at buf[l*ls + e*es]; n = 2^logn points per line, 2^lognl lines, at most
// FftCfg::PTS points per thread.  LINE_FAST: consecutive threads take
// consecutive lines (strided lines, es > 1); otherwise consecutive elements
// of a line.  The passes have radix 2^2 .. 2^MAXLR (ceil(logn / MAXLR)
// passes, the logs spread evenly, larger first; radix 2 only for a 2-point
// line), so all index arithmetic is shifts and masks and each pass's DFT
// lives in registers.
template <typename R, bool INV, bool LINE_FAST>
__device__ __forceinline__ void smem_fft(cplx<R>* buf, int logn, int lognl, int ls, int es,
                                         const cplx<R>* __restrict__ tw, int NT) {
    constexpr int MAXLR = FftCfg<R>::MAXLR;
    const int logNT = __ffs(NT) - 1;
    if (logn == 1) {
        fft_pass<R, 1, INV, LINE_FAST>(buf, logn, lognl, ls, es, 0, tw, NT, logNT);
        return;
    }
    const int np = (logn + MAXLR - 1) / MAXLR;
    int logNs = 0;
    for (int pass = 0; pass < np; ++pass) {
        const int rest = logn - logNs, left = np - pass;
        const int lr = (rest + left - 1) / left;
        if (MAXLR >= 4 && lr == 4) fft_pass<R, (MAXLR >= 4 ? 4 : 3), INV, LINE_FAST>(buf, logn, lognl, ls, es, logNs, tw, NT, logNT);
        else if (lr == 3) fft_pass<R, 3, INV, LINE_FAST>(buf, logn, lognl, ls, es, logNs, tw, NT, logNT);
        else fft_pass<R, 2, INV, LINE_FAST>(buf, logn, lognl, ls, es, logNs, tw, NT, logNT);
        logNs += lr;
    }
}

// ---- compile-time lengths -----------------------------------------------------------
// The same Stockham passes with the length n = 2^LOGN and the line count
// 2^LOGL (n 2^LOGL = 2048 points a CTA) known at compile time: every shift,
// mask and offset of the index arithmetic folds to a constant, the pass
// schedule unrolls, and the inter-pass twiddles come from a table of the n
// roots W_n^m staged in shared memory by the kernel (twn).  The pass
// schedule is smem_fft's (ceil(rest / passes left), largest first).
template <int LOGN, int MAXLR>
struct FftPlan {
    static constexpr int NP = (LOGN + MAXLR - 1) / MAXLR;
    static constexpr int ns(int p) {   // log2 Ns before pass p
        int l = 0;
        for (int q = 0; q < p; ++q) l += (LOGN - l + (NP - q) - 1) / (NP - q);
        return l;
    }
    static constexpr int lr(int p) { return (LOGN - ns(p) + (NP - p) - 1) / (NP - p); }
};

template <typename R, int LR, bool INV, bool LINE_FAST, int LOGN, int LOGL, int LOGNS>
__device__ __forceinline__ void fft_pass_ct(cplx<R>* buf, const cplx<R>* twn) {
    constexpr bool SKEW = !LINE_FAST;
    constexpr int NTHR = FftCfg<R>::THREADS;
    constexpr int RR = 1 << LR, KB = FftCfg<R>::PTS / RR;
    constexpr int LOGNB = LOGN - LR, NB = 1 << LOGNB;
    constexpr int TOTAL = NB << LOGL;
    constexpr int NS = 1 << LOGNS;
    constexpr int ES = LINE_FAST ? (1 << LOGL) : 1;
    constexpr int LS = LINE_FAST ? 1 : ((1 << LOGN) + ((1 << LOGN) >> 4) + 1);
    constexpr int TSH = LOGN - LR - LOGNS;
    static_assert(KB * NTHR == TOTAL, "every butterfly of the pass has a thread slot");
    const int tid = threadIdx.x;
    cplx<R> v[KB][RR];
    int oo[KB];
#pragma unroll
    for (int s = 0; s < KB; ++s) {
        const int b = tid + s * NTHR;
        int l, j;
        if (LINE_FAST) { l = b & ((1 << LOGL) - 1); j = b >> LOGL; }
        else { l = b >> LOGNB; j = b & (NB - 1); }
        const int k = j & (NS - 1);
        const cplx<R>* base = buf + l * LS;
#pragma unroll
        for (int r = 0; r < RR; ++r) {
            v[s][r] = base[sk16<SKEW>(j + r * NB) * ES];
            if (LOGNS > 0 && r > 0) {
                cplx<R> wv = twn[((r * k) << TSH) & ((1 << LOGN) - 1)];
                if (INV) wv.y = -wv.y;
                v[s][r] = cmul(v[s][r], wv);
            }
        }
        dft_reg<R, RR, INV>(v[s]);
        oo[s] = l * LS + (SKEW ? 0 : (((j - k) << LR) + k) * ES);
        if (SKEW) oo[s] |= ((((j - k) << LR) + k) << 16);
    }
    __syncthreads();
#pragma unroll
    for (int s = 0; s < KB; ++s) {
        if (SKEW) {
            const int lo = oo[s] & 0xFFFF, o = oo[s] >> 16;
#pragma unroll
            for (int q = 0; q < RR; ++q) buf[lo + sk16<true>(o + q * NS)] = v[s][q];
        } else {
#pragma unroll
            for (int q = 0; q < RR; ++q) buf[oo[s] + q * NS * ES] = v[s][q];
        }
    }
    __syncthreads();
}

template <typename R, bool INV, bool LINE_FAST, int LOGN, int LOGL, int P = 0>
__device__ __forceinline__ void smem_fft_ct(cplx<R>* buf, const cplx<R>* twn) {
    using PL = FftPlan<LOGN, FftCfg<R>::MAXLR>;
    if constexpr (P < PL::NP) {
        fft_pass_ct<R, PL::lr(P), INV, LINE_FAST, LOGN, LOGL, PL::ns(P)>(buf, twn);
        smem_fft_ct<R, INV, LINE_FAST, LOGN, LOGL, P + 1>(buf, twn);
    }
}

// The transform of a kernel: compile-time lengths (LOGN > 0; the lines fill
// the CTA's 2048 points) or the general form.
template <typename R, bool INV, bool LINE_FAST, int LOGN>
__device__ __forceinline__ void run_fft(cplx<R>* buf, int logn, int lognl, int ls, int es,
                                        const cplx<R>* __restrict__ tw, int NT, const cplx<R>* twn) {
    if constexpr (LOGN > 0) smem_fft_ct<R, INV, LINE_FAST, LOGN, 11 - LOGN>(buf, twn);
    else smem_fft<R, INV, LINE_FAST>(buf, logn, lognl, ls, es, tw, NT);
}
// Stage the roots W_n^m, m < n = 2^LOGN, from the NT-point table (NT >= n).
template <typename R, int LOGN>
__device__ __forceinline__ void stage_roots(cplx<R>* twn, const cplx<R>* __restrict__ tw, int NT) {
    if constexpr (LOGN > 0) {
        const int sh = (__ffs(NT) - 1) - LOGN;
        for (int m = threadIdx.x; m < (1 << LOGN); m += blockDim.x) twn[m] = tw[m << sh];
    }
}
// the extra shared memory of a compile-time-length kernel
template <typename R>
inline size_t roots_smem(int logn) { return (logn >= 7 && logn <= 9) ? ((size_t)1 << logn) * sizeof(cplx<R>) : 0; }

// ---- divergence ------------------------------------------------------------------
// The divergence of the predicted velocity (the source of the pressure solve)
// for N = 16/sizeof(R) x-consecutive cells per thread, 16-byte loads and
// stores.  The east, north and top neighbours follow the boundary maps:
// periodic x and y, and in z periodic or the zero wall face.
template <typename R, bool ANEL, bool UNI>
__global__ void __launch_bounds__(256) div_kernel(Geo g, const R* __restrict__ us, const R* __restrict__ vs,
                                                  const R* __restrict__ ws, R* __restrict__ out) {
    constexpr int N = Vec16<R>::N;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= g.nin / N) return;
    const long long q = t * N;
    const int lnx = __ffs(g.nx) - 1, lny = __ffs(g.ny) - 1;
    const int i0 = (int)(q & (g.nx - 1)), j = (int)((q >> lnx) & (g.ny - 1)), k = (int)(q >> (lnx + lny));
    const long long pl = (long long)g.nx * g.ny;
    const Met<R, UNI> m(g);
    R uc[N], vc[N], wc[N], vn[N], wn[N];
    vld(us + q, uc);
    const R ue = __ldg(us + (i0 + N < g.nx ? q + N : q + N - g.nx));
    vld(vs + q, vc);
    vld(vs + (j + 1 < g.ny ? q + g.nx : q - (long long)(g.ny - 1) * g.nx), vn);
    vld(ws + q, wc);
    if (k + 1 < g.nz) vld(ws + q + pl, wn);
    else if (g.bc_z == 0) vld(ws + q - (long long)(g.nz - 1) * pl, wn);
    else {
#pragma unroll
        for (int n = 0; n < N; ++n) wn[n] = R(0);   // the top wall face
    }
    const R idx = R(g.idx), idy = R(g.idy), idz = m.idz(k);
    R d[N];
    if (ANEL) {
        const R wcv = m.wc(k), wfb = m.wf(k), wft = m.wf(k + 1);
#pragma unroll
        for (int n = 0; n < N; ++n) {
            const R up = n + 1 < N ? uc[n + 1] : ue;
            d[n] = wcv * ((up - uc[n]) * idx + (vn[n] - vc[n]) * idy) + (wft * wn[n] - wfb * wc[n]) * idz;
        }
    } else {
#pragma unroll
        for (int n = 0; n < N; ++n) {
            const R up = n + 1 < N ? uc[n + 1] : ue;
            d[n] = (up - uc[n]) * idx + (vn[n] - vc[n]) * idy + (wn[n] - wc[n]) * idz;
        }
    }
    vst(out + q, d);
}

// The r2c post-process of bin kk from the packed M-point transform of one row.
template <typename R>
__device__ __forceinline__ cplx<R> r2c_bin(const cplx<R>* rowbuf, int M, int kk, cplx<R> wv) {
    const cplx<R> a = rowbuf[sk16<true>(kk == M ? 0 : kk)];
    const cplx<R> b = rowbuf[sk16<true>(kk == 0 ? 0 : M - kk)];
    const R er = R(0.5) * (a.x + b.x), ei = R(0.5) * (a.y - b.y);
    const R orr = R(0.5) * (a.y + b.y), oi = R(-0.5) * (a.x - b.x);
    return cmk<R>(er + (wv.x * orr - wv.y * oi), ei + (wv.x * oi + wv.y * orr));
}

// ---- c2r along x into phi ---------------------------------------------------------
// The pre-process of output bin kk from the half-spectrum bins a = X_kk and
// b = X_{M-kk} of a row (the inverse of r2c_bin's packing).
template <typename R>
__device__ __forceinline__ cplx<R> c2r_pre(cplx<R> a, cplx<R> b, cplx<R> wv) {
    const R er = a.x + b.x, ei = a.y - b.y;
    const R dr = a.x - b.x, di = a.y + b.y;
    const R orr = dr * wv.x + di * wv.y, oi = di * wv.x - dr * wv.y;
    return cmk<R>(er - oi, ei + orr);
}

// The CTA stages its rows' half spectra with one coalesced load per bin,
// pre-processes the bin pairs (u, M-u) (unit 0 of a row: bins 0 and M/2) in
// registers, writes the packed M-point lines skewed, runs the inverse FFT
// and stores the real pairs.
template <typename R, int LOGN = 0>
__global__ void __launch_bounds__(FFT_THREADS(R), FFT_MINB(R)) ifftx_kernel(Geo g, const cplx<R>* __restrict__ S, R* __restrict__ phi,
                                                    const cplx<R>* __restrict__ tw, int NT, int rows, R scale) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cplx<R>* buf = reinterpret_cast<cplx<R>*>(smem_raw);
    constexpr int UPT = FftCfg<R>::PTS / 2;
    const int M = LOGN > 0 ? (1 << LOGN) : g.nx / 2, Mh = M + 1, lM = LOGN > 0 ? LOGN : __ffs(M) - 1, LS = xrow(M);
    if (LOGN > 0) rows = 1 << (11 - LOGN);
    cplx<R>* twn = buf + rows * LS;
    stage_roots<R, LOGN>(twn, tw, NT);
    const long long nrows = (long long)g.ny * g.nz;
    const long long row0 = (long long)blockIdx.x * rows;
    const int tid = threadIdx.x, nthr = blockDim.x;
    const int tstep = NT / g.nx;
#pragma unroll 16
    for (int e = tid; e < (rows << lM); e += nthr) {
        const int r = e >> lM, kk = e & (M - 1);
        const long long row = row0 + r;
        buf[r * LS + kk] = row < nrows ? S[row * Mh + kk] : cmk<R>(R(0), R(0));
    }
    for (int r = tid; r < rows; r += nthr) {
        const long long row = row0 + r;
        buf[r * LS + M] = row < nrows ? S[row * Mh + M] : cmk<R>(R(0), R(0));
    }
    __syncthreads();
    const int lH = lM - 1, H = M >> 1;
    const int nunits = rows << lH;
    cplx<R> z0[UPT], z1[UPT];
    int pos[UPT];
#pragma unroll
    for (int s = 0; s < UPT; ++s) {
        const int e = tid + s * nthr;
        pos[s] = -1;
        if (e < nunits) {
            const int r = e >> lH, u = e & (H - 1);
            const cplx<R>* rb = buf + r * LS;
            const cplx<R> a = rb[u], b = rb[M - u];
            z0[s] = c2r_pre(a, b, tw[(u * tstep) & (NT - 1)]);
            if (u == 0) z1[s] = c2r_pre(rb[H], rb[H], tw[(H * tstep) & (NT - 1)]);
            else z1[s] = c2r_pre(b, a, tw[((M - u) * tstep) & (NT - 1)]);
            pos[s] = (r << 16) | u;
        }
    }
    __syncthreads();
#pragma unroll
    for (int s = 0; s < UPT; ++s) {
        if (pos[s] >= 0) {
            const int r = pos[s] >> 16, u = pos[s] & 0xFFFF;
            cplx<R>* rb = buf + r * LS;
            rb[sk16<true>(u)] = z0[s];
            rb[sk16<true>(u == 0 ? H : M - u)] = z1[s];
        }
    }
    __syncthreads();
    run_fft<R, true, false, LOGN>(buf, lM, __ffs(rows) - 1, LS, 1, tw, NT, twn);
    for (int e = tid; e < (rows << lM); e += nthr) {
        const int r = e >> lM, n = e & (M - 1);
        const long long row = row0 + r;
        if (row >= nrows) continue;
        const cplx<R> z = buf[r * LS + sk16<true>(n)];
        phi[row * g.nx + 2 * n] = z.x * scale;
        phi[row * g.nx + 2 * n + 1] = z.y * scale;
    }
}

// ---- complex transform along y (MODE 0 forward, 1 inverse) ----------------------
// CTA: tile of `tpx` consecutive kx columns at one kz, all ky.
template <typename R, int MODE, int LOGN = 0>
__global__ void __launch_bounds__(FFT_THREADS(R), FFT_MINB(R)) ffty_kernel(Geo g, cplx<R>* __restrict__ S, const cplx<R>* __restrict__ tw,
                                                   int NT, int tpx) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cplx<R>* buf = reinterpret_cast<cplx<R>*>(smem_raw);
    if (LOGN > 0) tpx = 1 << (11 - LOGN);
    cplx<R>* twn = buf + g.ny * tpx;
    stage_roots<R, LOGN>(twn, tw, NT);
    const int Mh = g.nx / 2 + 1;
    const int k = blockIdx.y, p0 = blockIdx.x * tpx;
    const int tid = threadIdx.x, nthr = blockDim.x;
    const long long base = (long long)k * g.ny * Mh;
    const int lt = __ffs(tpx) - 1;
#pragma unroll 16
    for (int e = tid; e < g.ny * tpx; e += nthr) {
        const int jj = e >> lt, c = e & (tpx - 1), p = p0 + c;
        buf[e] = p < Mh ? S[base + (long long)jj * Mh + p] : cmk<R>(R(0), R(0));
    }
    __syncthreads();
    run_fft<R, MODE == 1, true, LOGN>(buf, __ffs(g.ny) - 1, __ffs(tpx) - 1, 1, tpx, tw, NT, twn);
    for (int e = tid; e < g.ny * tpx; e += nthr) {
        const int jj = e >> lt, c = e & (tpx - 1), p = p0 + c;
        if (p < Mh) S[base + (long long)jj * Mh + p] = buf[e];
    }
}

// ---- periodic z: forward, scale by nrm/lambda, inverse -------------------------
template <typename R, int LOGN = 0>
__global__ void __launch_bounds__(FFT_THREADS(R), FFT_MINB(R)) fftz_solve_kernel(Geo g, cplx<R>* __restrict__ S, const cplx<R>* __restrict__ tw,
                                                         int NT, int tpx, const double* __restrict__ kx2,
                                                         const double* __restrict__ ky2, const double* __restrict__ kz2,
                                                         double nrm) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cplx<R>* buf = reinterpret_cast<cplx<R>*>(smem_raw);
    if (LOGN > 0) tpx = 1 << (11 - LOGN);
    cplx<R>* twn = buf + g.nz * tpx;
    stage_roots<R, LOGN>(twn, tw, NT);
    const int Mh = g.nx / 2 + 1;
    const int j = blockIdx.y, p0 = blockIdx.x * tpx;
    const int tid = threadIdx.x, nthr = blockDim.x;
    const long long sk = (long long)g.ny * Mh;
    const long long base = (long long)j * Mh;
    const int lt = __ffs(tpx) - 1;
#pragma unroll 16
    for (int e = tid; e < g.nz * tpx; e += nthr) {
        const int kz = e >> lt, c = e & (tpx - 1), p = p0 + c;
        buf[e] = p < Mh ? S[base + kz * sk + p] : cmk<R>(R(0), R(0));
    }
    __syncthreads();
    run_fft<R, false, true, LOGN>(buf, __ffs(g.nz) - 1, __ffs(tpx) - 1, 1, tpx, tw, NT, twn);
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
    run_fft<R, true, true, LOGN>(buf, __ffs(g.nz) - 1, __ffs(tpx) - 1, 1, tpx, tw, NT, twn);
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
// exposing one memory latency per level.  The forward-elimination values d'_k
// go to dsc, a column scratch of the spectrum's layout in precision RD (dsc
// may alias S when RD is S's type: d'_k overwrites the level it came from
// after that level was read).  The modified upper diagonal c'_k goes either
// to an RD scratch of the same layout (CPG: streamed back with d'_k, so a CTA
// needs only its rings and every column warp of the grid is resident at
// once) or to shared memory [nz][32] (no scratch: the allocation-free entry).
// The recurrence itself runs in FP64 whatever RD is; the FP32-mixed step
// stores d' and c' in FP32 in place (S and an FP32 c' array), so the stored
// intermediates carry the rounding of the FP32 spectrum they came from and
// the solve moves 40 bytes an element instead of 64.
constexpr int THOMAS_PF = 16;
// the largest nz whose column state fits a CTA's 227 KB of shared memory
#define AEO_COLUMN_NZ_MAX 800

__device__ __forceinline__ void thomas_cp4(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)), "l"(src)
                 : "memory");
}
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
    if (N == 4) thomas_cp4(dst, src);
    else if (N == 8) thomas_cp8(dst, src);
    else thomas_cp16(dst, src);
}
__device__ __forceinline__ void thomas_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void thomas_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// Block 0 is the mean mode; blocks 1.. hold 32 columns each.
inline unsigned thomas_blocks(const Geo& g) {
    return 1u + (unsigned)(((long long)g.ny * (g.nx / 2 + 1) + 31) / 32);
}
// Shared memory: the d' ring [THOMAS_PF][32] of cplx<double>, then (CPG) the
// c' ring [THOMAS_PF][32] of double or (shared c') c' [nz][32], then the
// lower, upper and h vectors [nz] each; at least the mean mode's 5 nz + 1.
inline size_t thomas_smem(const Geo& g, bool cpg) {
    const size_t ring = (size_t)THOMAS_PF * 32 * 2 * sizeof(double);
    const size_t cols = cpg ? (size_t)THOMAS_PF * 32 * sizeof(double) + (size_t)g.nz * 3 * sizeof(double)
                            : (size_t)g.nz * 35 * sizeof(double);
    const size_t mean = (size_t)(5 * g.nz + 1) * sizeof(double);
    return ring + (cols > mean ? cols : mean);
}

// The elimination factors of every non-mean column, once per grid: the
// multiplier m_k = 1 / (b_k - lo_k c'_{k-1}) of level k and c'_k = up_k m_k,
// in precision RD at the spectrum's layout (mtab, ctab).  They depend on the
// column's coefficients and its eigenvalue kx^2 + ky^2 only, so the solves
// of a run stream them instead of recomputing the division chain; the FP64
// arithmetic and its order are those of the solve kernel's own elimination,
// so an FP64 table reproduces it exactly.
template <typename RD>
__global__ void __launch_bounds__(256) thomas_factor_kernel(Geo g, RD* __restrict__ mtab, RD* __restrict__ ctab,
                                                            ColumnCoef c) {
    const int Mh = g.nx / 2 + 1;
    const long long sk = (long long)g.ny * Mh;
    const long long col = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (col == 0 || col >= sk) return;
    const int p = (int)(col % Mh), j = (int)(col / Mh);
    const double lam = c.kx2[p] + c.ky2[j];
    double cprev = 0.0;
    for (int k = 0; k < g.nz; ++k) {
        const double lo = c.lower[k], up = c.upper[k];
        const double b = -(lo + up) - lam * c.hw[k];
        const double den = b - lo * cprev;
        const double id = 1.0 / den;
        cprev = up * id;
        mtab[col + (long long)k * sk] = RD(id);
        if (k < g.nz - 1) ctab[col + (long long)k * sk] = RD(cprev);
    }
}

// FAC: the elimination factors come from thomas_factor_kernel's tables
// (mtab; cpg holds c'), streamed through the c' ring in the forward pass, so
// the recurrence is two multiply-adds a level and writes no c'.
template <typename R, bool CPG, typename RD = double, bool FAC = false>
__global__ void __launch_bounds__(32) thomas_kernel(Geo g, cplx<R>* S, cplx<RD>* dsc, RD* cpg, ColumnCoef c,
                                                    const RD* __restrict__ mtab = nullptr) {
    static_assert(!FAC || CPG, "the factored solve streams c' from its table");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int D = THOMAS_PF;
    cplx<double>* ring = reinterpret_cast<cplx<double>*>(smem_raw);   // [D][32], 16-byte entries
    double* after = reinterpret_cast<double*>(ring + D * 32);
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
        double* sv = after;          // [nz] the column's real parts
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
    RD* cring = reinterpret_cast<RD*>(after);           // CPG: [D][32] c' ring
    double* cp = after;                                 // shared c': [nz][32]
    double* s_lo = CPG ? after + D * 32 : after + 32 * nz;
    double* s_up = s_lo + nz;
    double* s_hw = s_up + nz;
    // the diagonals' per-level coefficients, staged once
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
    // forward elimination: level k waits in slot k % D; the copy of level
    // k + D - 1 goes to the slot read one level earlier
    cplx<R>* rs = reinterpret_cast<cplx<R>*>(ring);   // this lane's entries at [slot * 32 + lane]
#pragma unroll
    for (int q = 0; q < D - 1; ++q) {
        if (q < nz) {
            thomas_cp<sizeof(cplx<R>)>(rs + q * 32 + lane, S + col + q * sk);
            if (FAC) thomas_cp<sizeof(RD)>(cring + q * 32 + lane, mtab + col + q * sk);
        }
        thomas_commit();
    }
    double cprev = 0.0, dr = 0.0, di = 0.0;
    for (int k = 0; k < nz; ++k) {
        const int kn = k + D - 1;
        if (kn < nz) {
            thomas_cp<sizeof(cplx<R>)>(rs + (kn % D) * 32 + lane, S + col + (long long)kn * sk);
            if (FAC) thomas_cp<sizeof(RD)>(cring + (kn % D) * 32 + lane, mtab + col + (long long)kn * sk);
        }
        thomas_commit();
        thomas_wait<D - 1>();   // level k has landed
        const cplx<R> s = rs[(k % D) * 32 + lane];
        const double lo = s_lo[k];
        double id;
        if constexpr (FAC) {
            id = (double)cring[(k % D) * 32 + lane];
        } else {
            const double up = s_up[k];
            const double b = -(lo + up) - lam * s_hw[k];
            const double den = b - lo * cprev;
            id = 1.0 / den;
            cprev = up * id;
        }
        dr = ((double)s.x - lo * dr) * id;   // lo = 0 at k = 0
        di = ((double)s.y - lo * di) * id;
        if (k < nz - 1) {
            if (!FAC) {
                if (CPG) cpg[col + (long long)k * sk] = RD(cprev);
                else cp[k * 32 + lane] = cprev;
            }
            dsc[col + (long long)k * sk] = cmk<RD>(RD(dr), RD(di));
        }
    }
    thomas_wait<0>();
    S[col + (long long)(nz - 1) * sk] = cmk<R>(R(dr), R(di));
    // back substitution over k = nz-2 .. 0, the d' (and c') values streamed
    // alike (slot t holds level nz-2-t modulo D)
    cplx<RD>* dring = reinterpret_cast<cplx<RD>*>(ring);
    auto fetch = [&](int slot, int k) {
        thomas_cp<sizeof(cplx<RD>)>(dring + slot * 32 + lane, dsc + col + (long long)k * sk);
        if (CPG) thomas_cp<sizeof(RD)>(cring + slot * 32 + lane, cpg + col + (long long)k * sk);
    };
#pragma unroll
    for (int q = 0; q < D - 1; ++q) {
        const int k = nz - 2 - q;
        if (k >= 0) fetch(q, k);
        thomas_commit();
    }
    for (int t = 0; t <= nz - 2; ++t) {
        const int k = nz - 2 - t;
        const int tn = t + D - 1, kn = nz - 2 - tn;
        if (kn >= 0) fetch(tn % D, kn);
        thomas_commit();
        thomas_wait<D - 1>();
        const cplx<RD> d = dring[(t % D) * 32 + lane];
        const double cc = CPG ? (double)cring[(t % D) * 32 + lane] : cp[k * 32 + lane];
        dr = (double)d.x - cc * dr;
        di = (double)d.y - cc * di;
        S[col + (long long)k * sk] = cmk<R>(R(dr), R(di));
    }
    thomas_wait<0>();
}

// r2c of an interior source along x: pack pairs, FFT, post-process.
// DIV: the source is the divergence of the predicted velocity (us, vs, ws:
// interior arrays), formed while the rows are staged with div_kernel's
// arithmetic (plain, or W-weighted for the sound-proof core), instead of
// being read from src: the divergence never goes to memory.
template <typename R, bool ANEL, bool UNI>
__device__ __forceinline__ cplx<R> div_pair(const Geo& g, const R* __restrict__ us, const R* __restrict__ vs,
                                            const R* __restrict__ ws, long long row, int i0) {
    const int j = (int)(row % g.ny), k = (int)(row / g.ny);
    const long long q = row * g.nx + i0, pl = (long long)g.nx * g.ny;
    const Met<R, UNI> m(g);
    const R uc0 = __ldg(us + q), uc1 = __ldg(us + q + 1);
    const R ue = __ldg(us + (i0 + 2 < g.nx ? q + 2 : q + 2 - g.nx));
    const long long qn = j + 1 < g.ny ? q + g.nx : q - (long long)(g.ny - 1) * g.nx;
    const R vc0 = __ldg(vs + q), vc1 = __ldg(vs + q + 1), vn0 = __ldg(vs + qn), vn1 = __ldg(vs + qn + 1);
    const R wc0 = __ldg(ws + q), wc1 = __ldg(ws + q + 1);
    R wn0 = R(0), wn1 = R(0);   // the top wall face
    if (k + 1 < g.nz) { wn0 = __ldg(ws + q + pl); wn1 = __ldg(ws + q + pl + 1); }
    else if (g.bc_z == 0) {
        const long long qb = q - (long long)(g.nz - 1) * pl;
        wn0 = __ldg(ws + qb); wn1 = __ldg(ws + qb + 1);
    }
    const R idx = R(g.idx), idy = R(g.idy), idz = m.idz(k);
    if (ANEL) {
        const R wcv = m.wc(k), wfb = m.wf(k), wft = m.wf(k + 1);
        return cmk<R>(wcv * ((uc1 - uc0) * idx + (vn0 - vc0) * idy) + (wft * wn0 - wfb * wc0) * idz,
                      wcv * ((ue - uc1) * idx + (vn1 - vc1) * idy) + (wft * wn1 - wfb * wc1) * idz);
    }
    return cmk<R>((uc1 - uc0) * idx + (vn0 - vc0) * idy + (wn0 - wc0) * idz,
                  (ue - uc1) * idx + (vn1 - vc1) * idy + (wn1 - wc1) * idz);
}

template <typename R, int LOGN = 0, int DIV = 0>   // DIV: 0 src; 1 plain, 2 W-weighted divergence (+4: stretched)
__global__ void __launch_bounds__(FFT_THREADS(R), FFT_MINB(R)) src_fftx_kernel(Geo g, const R* __restrict__ src, cplx<R>* __restrict__ S,
                                                       const cplx<R>* __restrict__ tw, int NT, int rows,
                                                       const R* __restrict__ us = nullptr, const R* __restrict__ vs = nullptr,
                                                       const R* __restrict__ ws = nullptr) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cplx<R>* buf = reinterpret_cast<cplx<R>*>(smem_raw);
    const int M = LOGN > 0 ? (1 << LOGN) : g.nx / 2, Mh = M + 1, lM = LOGN > 0 ? LOGN : __ffs(M) - 1, LS = xrow(M);
    if (LOGN > 0) rows = 1 << (11 - LOGN);
    cplx<R>* twn = buf + rows * LS;
    stage_roots<R, LOGN>(twn, tw, NT);
    const long long nrows = (long long)g.ny * g.nz;
    const long long row0 = (long long)blockIdx.x * rows;
    const int tid = threadIdx.x, nthr = blockDim.x;
#pragma unroll 16
    for (int e = tid; e < (rows << lM); e += nthr) {
        const int r = e >> lM, n = e & (M - 1);
        const long long row = row0 + r;
        cplx<R> z = cmk<R>(R(0), R(0));
        if (row < nrows) {
            if constexpr (DIV == 0) z = cmk<R>(src[row * g.nx + 2 * n], src[row * g.nx + 2 * n + 1]);
            else z = div_pair<R, (DIV & 3) == 2, (DIV & 4) == 0>(g, us, vs, ws, row, 2 * n);
        }
        buf[r * LS + sk16<true>(n)] = z;
    }
    __syncthreads();
    run_fft<R, false, false, LOGN>(buf, lM, __ffs(rows) - 1, LS, 1, tw, NT, twn);
    const int tstep = NT / g.nx;
    for (int e = tid; e < (rows << lM); e += nthr) {
        const int r = e >> lM, kk = e & (M - 1);
        const long long row = row0 + r;
        if (row < nrows) S[row * Mh + kk] = r2c_bin(buf + r * LS, M, kk, tw[(kk * tstep) & (NT - 1)]);
    }
    for (int r = tid; r < rows; r += nthr) {   // the Nyquist bin, twiddle exactly -1
        const long long row = row0 + r;
        if (row < nrows) S[row * Mh + M] = r2c_bin(buf + r * LS, M, M, cmk<R>(R(-1), R(0)));
    }
}
