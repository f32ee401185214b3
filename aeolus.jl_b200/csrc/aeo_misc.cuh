// aeo_misc.cuh -- halo fills, the projection's correction, host-layout
// packing, reductions and the Philox input generator.
#pragma once

#include "aeo_common.cuh"

// ---- halo fill of padded arrays (gather form) ------------------------------------
// Every point of the AEO_H-wide shell around the interior takes the value of
// the composite boundary map (zmap / wrap), which is what the reference's
// axis-ordered fill (x, then y, then z) leaves there
// (src/boundary_conditions/halo_kernels.jl:100-140, src/BoundaryConditions.jl:228-258).
template <typename R>
struct HaloSet {
    R* f[5];
    int loc[5];
    int nf;
};

__device__ __forceinline__ void shell_point(const Geo& g, long long t, int* i, int* j, int* k) {
    const int H = AEO_H;
    const long long bx = g.nx + 2 * H, by = g.ny + 2 * H;
    const long long nzs = 2LL * H * bx * by;          // the two z slabs
    if (t < nzs) {
        long long s = t;
        *i = (int)(s % bx) - H; s /= bx;
        *j = (int)(s % by) - H; s /= by;
        int kz = (int)s;
        *k = kz < H ? kz - H : g.nz + (kz - H);
        return;
    }
    t -= nzs;
    const long long nys = 2LL * H * bx * g.nz;        // the two y slabs (interior k)
    if (t < nys) {
        long long s = t;
        *i = (int)(s % bx) - H; s /= bx;
        int jy = (int)(s % (2 * H)); s /= (2 * H);
        *j = jy < H ? jy - H : g.ny + (jy - H);
        *k = (int)s;
        return;
    }
    t -= nys;                                          // the two x slabs (interior j, k)
    long long s = t;
    int ix = (int)(s % (2 * H)); s /= (2 * H);
    *i = ix < H ? ix - H : g.nx + (ix - H);
    *j = (int)(s % g.ny); s /= g.ny;
    *k = (int)s;
}

__host__ __device__ __forceinline__ long long shell_count(const Geo& g) {
    const long long H = AEO_H, bx = g.nx + 2 * H, by = g.ny + 2 * H;
    return 2 * H * bx * by + 2 * H * bx * g.nz + 2 * H * (long long)g.ny * g.nz;
}

template <typename R>
__global__ void __launch_bounds__(256) halo_fill_kernel(Geo g, HaloSet<R> hs) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= shell_count(g)) return;
    int i, j, k;
    shell_point(g, t, &i, &j, &k);
    int ii = wrapi(i, g.nx), jj = wrapi(j, g.ny);
    // every field's source first, then the stores: the loads do not wait for
    // the stores of the fields before them (the arrays could alias, as far as
    // the compiler knows), so one memory latency a point instead of one a field
    R v[5];
#pragma unroll
    for (int f = 0; f < 5; ++f) {
        if (f < hs.nf) {
            int kk;
            const int s = zmap(g, k, hs.loc[f], &kk);
            v[f] = s == 0 ? R(0) : hs.f[f][pidx(g, ii, jj, kk)];
            if (s < 0) v[f] = -v[f];
        }
    }
    const long long q = pidx(g, i, j, k);
#pragma unroll
    for (int f = 0; f < 5; ++f)
        if (f < hs.nf) hs.f[f][q] = v[f];
}

// ---- open lateral faces (src/boundary_conditions/open_boundary.jl:722-807) -------
// The plane buffers of the open faces in the reference's storage extents
// (halo H = AEO_H on every axis): x planes [field][side][NZ][NY][L], y planes
// [field][side][NZ][L][NX] (field u, v, w, theta; side 0 west/south, 1
// east/north; NZ, NY, NX the storage extents; layer = storage index along the
// normal on the low side, storage index - (H + N) on the high side, L = H + 1
// so the low side holds the normal velocity's boundary face, interior 0).
// mode[f] = 1: the field takes the zero-gradient mirror on open faces, as
// every field without a plane does (pid < 0: the pressure, nu_t, closure
// state).  The boundary-face values of the normal velocities, bw/be [k][j]
// and bs/bn [k][i] (interior), feed the projection.
template <typename R>
struct OpenSet {
    const R* xp;
    const R* yp;
    const R* bw;
    const R* be;
    const R* bs;
    const R* bn;
    int ox, oy, L;
    int mode[4];
};

// The composite map of the reference's fill order (x, then y, then z) with
// open faces: z first (the z fill copies whole x-y planes), then y (an open y
// face copies its plane over every x, halos included), then x.
template <typename R>
__device__ __forceinline__ R open_halo_value(const Geo& g, const OpenSet<R>& ob, const R* f, int loc, int pid, int i,
                                             int j, int k) {
    int kk;
    const int s = zmap(g, k, loc, &kk);
    if (s == 0) return R(0);
    const bool plane = pid >= 0 && ob.mode[pid] == 0;
    const int NX = g.nx + 2 * AEO_H, NY = g.ny + 2 * AEO_H, NZ = g.nz + 2 * AEO_H;
    R v;
    int ii = i, jj = j;
    if (j < 0 || j >= g.ny) {
        if (ob.oy) {
            if (plane) {
                const int side = j >= g.ny, l = side ? j - g.ny : j + AEO_H;
                v = ob.yp[((((size_t)(pid * 2 + side) * NZ + kk + AEO_H) * ob.L + l) * NX) + i + AEO_H];
                return s > 0 ? v : -v;
            }
            jj = j < 0 ? -1 - j : 2 * g.ny - 1 - j;
        } else {
            jj = wrapi(j, g.ny);
        }
    }
    if (i < 0 || i >= g.nx) {
        if (ob.ox) {
            if (plane) {
                const int side = i >= g.nx, l = side ? i - g.nx : i + AEO_H;
                v = ob.xp[((((size_t)(pid * 2 + side) * NZ + kk + AEO_H) * NY + jj + AEO_H) * ob.L) + l];
                return s > 0 ? v : -v;
            }
            ii = i < 0 ? -1 - i : 2 * g.nx - 1 - i;
        } else {
            ii = wrapi(i, g.nx);
        }
    }
    v = f[pidx(g, ii, jj, kk)];
    return s > 0 ? v : -v;
}

// The boundary face of a normal velocity on a west / south open face lies in
// the interior (index 0) and takes the plane's value on every fill
// (_open_range, src/boundary_conditions/open_boundary.jl:46-51): u[0, j, k]
// (axis 0) or v[i, 0, k] (axis 1) over the interior of the two other axes.
template <typename R>
__global__ void open_face_kernel(Geo g, R* f, OpenSet<R> ob, int axis) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x, k = blockIdx.y;
    const int NX = g.nx + 2 * AEO_H, NY = g.ny + 2 * AEO_H, NZ = g.nz + 2 * AEO_H;
    if (axis == 0) {
        if (a >= g.ny) return;
        f[pidx(g, 0, a, k)] = ob.xp[((((size_t)0 * NZ + k + AEO_H) * NY + a + AEO_H) * ob.L) + AEO_H];
    } else {
        if (a >= g.nx) return;
        f[pidx(g, a, 0, k)] = ob.yp[((((size_t)(1 * 2) * NZ + k + AEO_H) * ob.L + AEO_H) * NX) + a + AEO_H];
    }
}

// halo_fill_kernel with open faces; pid[f] the plane of field f (-1: none)
template <typename R>
__global__ void __launch_bounds__(256) open_halo_fill_kernel(Geo g, HaloSet<R> hs, OpenSet<R> ob, int4 pid4) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= shell_count(g)) return;
    int i, j, k;
    shell_point(g, t, &i, &j, &k);
    const int pid[4] = {pid4.x, pid4.y, pid4.z, pid4.w};
    R v[4];
#pragma unroll
    for (int f = 0; f < 4; ++f)
        if (f < hs.nf) v[f] = open_halo_value(g, ob, hs.f[f], hs.loc[f], pid[f], i, j, k);
    const long long q = pidx(g, i, j, k);
#pragma unroll
    for (int f = 0; f < 4; ++f)
        if (f < hs.nf) hs.f[f][q] = v[f];
}

// The wall face of w (interior k = 0) is zero after every fill.
template <typename R>
__global__ void wall_face_zero_kernel(Geo g, R* w) {
    int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y;
    if (i < g.nx) w[pidx(g, i, j, 0)] = R(0);
}

// ---- the projection's correction (src/FiniteVolume.jl:1823-1849) ---------------
// u = c(u* - d(phi)/dx, u0) (likewise v, w), p = phi/dt; c(x, s) = ca*s + cb*x
// in RK3 stages 2 and 3 (_Lin2r, src/Simulations.jl:1194-1198).
// N = 16/sizeof(R) x-consecutive cells per thread, 16-byte loads and stores;
// the west, south and bottom neighbours of phi follow the centred-field
// maps: periodic x and y, in z periodic or the wall mirror.
template <typename R, bool UNI>
__global__ void __launch_bounds__(256) correct_kernel(Geo g, const R* __restrict__ us, const R* __restrict__ vs,
                                                      const R* __restrict__ ws, const R* __restrict__ phi,
                                                      const R* u0, const R* v0,
                                                      const R* w0, R* uo, R* vo,
                                                      R* wo, R* __restrict__ p, const double* __restrict__ dtp, R ca, R cb,
                                                      int stage) {
    constexpr int N = Vec16<R>::N;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= g.nin / N) return;
    const long long qi = t * N;
    const int lnx = __ffs(g.nx) - 1, lny = __ffs(g.ny) - 1;
    const int i0 = (int)(qi & (g.nx - 1)), j = (int)((qi >> lnx) & (g.ny - 1)), k = (int)(qi >> (lnx + lny));
    const long long qp = pidx(g, i0, j, k), pl = (long long)g.nx * g.ny;
    R pc[N], ps[N], pb[N];
    vld(phi + qi, pc);
    const R pwl = __ldg(phi + (i0 > 0 ? qi - 1 : qi + g.nx - 1));
    vld(phi + (j > 0 ? qi - g.nx : qi + (long long)(g.ny - 1) * g.nx), ps);
    // k - 1 = -1: periodic wrap, or the wall mirror (level 0 itself)
    vld(phi + (k > 0 ? qi - pl : (g.bc_z == 0 ? qi + (long long)(g.nz - 1) * pl : qi)), pb);
    const R idzf = UNI ? R(g.idz) : Met<R, UNI>(g).idzf(k);
    R uc[N], vc[N], wc[N];
    vld(us + qi, uc);
    vld(vs + qi, vc);
    vld(ws + qi, wc);
    R un[N], vn[N], wn[N];
#pragma unroll
    for (int n = 0; n < N; ++n) {
        const R pw = n > 0 ? pc[n - 1] : pwl;
        un[n] = uc[n] - (pc[n] - pw) * R(g.idx);
        vn[n] = vc[n] - (pc[n] - ps[n]) * R(g.idy);
        wn[n] = wc[n] - (pc[n] - pb[n]) * idzf;
    }
    if (stage) {
        R a0[N];
        vld(u0 + qp, a0);
#pragma unroll
        for (int n = 0; n < N; ++n) un[n] = rk_combine(ca, cb, a0[n], un[n]);
        vld(v0 + qp, a0);
#pragma unroll
        for (int n = 0; n < N; ++n) vn[n] = rk_combine(ca, cb, a0[n], vn[n]);
        vld(w0 + qp, a0);
#pragma unroll
        for (int n = 0; n < N; ++n) wn[n] = rk_combine(ca, cb, a0[n], wn[n]);
    }
    vst(uo + qp, un);
    vst(vo + qp, vn);
    vst(wo + qp, wn);
    const R dt = R(__ldg(dtp));
#pragma unroll
    for (int n = 0; n < N; ++n) pc[n] = pc[n] / dt;   // p = phi/dt (_DivBy, src/Simulations.jl:1207-1211)
    vst(p + qi, pc);
}

// ---- host-layout packing ----------------------------------------------------------
// Host storage (reference layout, halos hh) <-> device padded interior.
template <typename R, typename S = double>
__global__ void unpack_host_kernel(Geo g, const S* __restrict__ hsrc, int hx, int hy, int hz,
                                   R* __restrict__ dst, int padded, double off) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int j = blockIdx.y, k = blockIdx.z;
    if (i >= g.nx) return;
    long long HX = g.nx + 2LL * hx, HY = g.ny + 2LL * hy;
    double v = (double)hsrc[(i + hx) + HX * ((j + hy) + HY * (long long)(k + hz))] - off;
    if (padded) dst[pidx(g, i, j, k)] = R(v);
    else dst[iidx(g, i, j, k)] = R(v);
}

// Fill the whole host storage array from the device interior through the
// composite boundary map (loc < 0: halos zero); `off` is added back to every
// mapped value (the stored offset of theta, 0 otherwise).
template <typename R, typename S = double>
__global__ void pack_host_kernel(Geo g, S* __restrict__ hdst, int hx, int hy, int hz,
                                 const R* __restrict__ src, int padded, int loc, double off) {
    long long HX = g.nx + 2LL * hx, HY = g.ny + 2LL * hy, HZ = g.nz + 2LL * hz;
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= HX * HY * HZ) return;
    int i = (int)(t % HX) - hx;
    int j = (int)((t / HX) % HY) - hy;
    int k = (int)(t / (HX * HY)) - hz;
    bool inside = i >= 0 && i < g.nx && j >= 0 && j < g.ny && k >= 0 && k < g.nz;
    double v = 0.0;
    if (inside || loc >= 0) {
        int kk;
        int s = inside ? 1 : zmap(g, k, loc, &kk);
        if (inside) kk = k;
        if (s != 0) {
            int ii = inside ? i : wrapi(i, g.nx), jj = inside ? j : wrapi(j, g.ny);
            R r = padded ? src[pidx(g, ii, jj, kk)] : src[iidx(g, ii, jj, kk)];
            v = (s > 0 ? (double)r : -(double)r) + off;
        }
    }
    hdst[t] = S(v);
}

// interior-sized double <-> interior R
template <typename R>
__global__ void convert_kernel(long long n, const double* __restrict__ a, R* __restrict__ b) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) b[t] = R(a[t]);
}
template <typename R>
__global__ void convert_back_kernel(long long n, const R* __restrict__ a, double* __restrict__ b) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) b[t] = double(a[t]);
}

// ---- deterministic FP64 reductions --------------------------------------------------
// Per-level partial sums, each level summed by one CTA in a fixed order,
// then the levels in ascending k (the canonical plane sums of
// src/Backends.jl:1349-1357; src/Simulations.jl:992-1014).
template <typename R, bool UNI>
__global__ void __launch_bounds__(256) ke_levels_kernel(Geo g, const R* __restrict__ u, const R* __restrict__ v,
                                                        const R* __restrict__ w, double* __restrict__ part) {
    __shared__ double red[256];
    int k = blockIdx.x;
    double acc = 0.0;
    double dzc = UNI ? 1.0 : 1.0 / lvl(g.idzc, k), dzf = UNI ? 1.0 : 1.0 / lvl(g.idzf, k);
    for (int e = threadIdx.x; e < g.nx * g.ny; e += blockDim.x) {
        int i = e % g.nx, j = e / g.nx;
        long long q = pidx(g, i, j, k);
        double uu = u[q], vv = v[q], ww = w[q];
        if (UNI) acc += uu * uu + vv * vv + ww * ww;
        else acc += (uu * uu + vv * vv) * dzc + ww * ww * dzf;
    }
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[k] = red[0];
}

template <typename R, bool ANEL, bool UNI>
__global__ void __launch_bounds__(256) maxdiv_levels_kernel(Geo g, const R* __restrict__ u, const R* __restrict__ v,
                                                            const R* __restrict__ w, double* __restrict__ part) {
    __shared__ double red[256];
    int k = blockIdx.x;
    double acc = 0.0;
    double idz = UNI ? g.idz : lvl(g.idzc, k);
    for (int e = threadIdx.x; e < g.nx * g.ny; e += blockDim.x) {
        int i = e % g.nx, j = e / g.nx;
        long long q = pidx(g, i, j, k);
        double du = ((double)u[q + 1] - (double)u[q]) * g.idx;
        double dv = ((double)v[q + g.sy] - (double)v[q]) * g.idy;
        double d;
        if (ANEL) {
            double wc = lvl(g.wc, k), wfb = lvl(g.wf, k), wft = lvl(g.wf, k + 1);
            d = (wc * (du + dv) + (wft * (double)w[q + g.sz] - wfb * (double)w[q]) * idz) / wc;
        } else {
            d = du + dv + ((double)w[q + g.sz] - (double)w[q]) * idz;
        }
        acc = fmax(acc, fabs(d));
    }
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + s]);
        __syncthreads();
    }
    if (threadIdx.x == 0) part[k] = red[0];
}

// The loop of the multi-step graph: a conditional WHILE node whose body is two
// RK3 steps runs while step pairs remain (the count in device memory).
__global__ void steps_set_kernel(int* left, int pairs) { *left = pairs; }
__global__ void steps_begin_kernel(const int* left, cudaGraphConditionalHandle h) {
    cudaGraphSetConditional(h, *left > 0 ? 1u : 0u);
}
__global__ void steps_next_kernel(int* left, cudaGraphConditionalHandle h) {
    const int n = *left - 1;
    *left = n;
    cudaGraphSetConditional(h, n > 0 ? 1u : 0u);
}

// non-finite check of the four state fields (status word for the host): a
// grid-stride pass over the interiors, N = 16/sizeof(R) x-consecutive values a
// 16-byte load; one flag update per block
template <typename R>
__global__ void __launch_bounds__(256) finite_check_kernel(Geo g, const R* __restrict__ f0, const R* __restrict__ f1,
                                                           const R* __restrict__ f2, const R* __restrict__ f3,
                                                           int* __restrict__ flag) {
    constexpr int N = Vec16<R>::N;
    const int per = (int)(g.nin / N);   // vectors of one field (nx is a multiple of N)
    const int lnx = __ffs(g.nx) - 1, lny = __ffs(g.ny) - 1;
    const int stride = gridDim.x * blockDim.x;
    bool bad = false;
#pragma unroll
    for (int f = 0; f < 4; ++f) {
        const R* a = f == 0 ? f0 : (f == 1 ? f1 : (f == 2 ? f2 : f3));
        for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < per; t += stride) {
            const long long qi = (long long)t * N;
            const int i0 = (int)(qi & (g.nx - 1)), j = (int)((qi >> lnx) & (g.ny - 1)), k = (int)(qi >> (lnx + lny));
            R v[N];
            vld(a + pidx(g, i0, j, k), v);
#pragma unroll
            for (int n = 0; n < N; ++n) bad = bad || !isfinite(v[n]);
        }
    }
    if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(flag, 1);
}

// ---- Philox4x32-10 (src/Backends.jl:1607-1640) ------------------------------------
__device__ __forceinline__ void philox4x32(uint32_t c[4], uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int r = 1; r <= 10; ++r) {
        uint32_t hi0 = __umulhi(0xD2511F53u, c[0]), lo0 = 0xD2511F53u * c[0];
        uint32_t hi1 = __umulhi(0xCD9E8D57u, c[2]), lo1 = 0xCD9E8D57u * c[2];
        uint32_t n0 = hi1 ^ c[1] ^ k0, n1 = lo1, n2 = hi0 ^ c[3] ^ k1, n3 = lo0;
        c[0] = n0; c[1] = n1; c[2] = n2; c[3] = n3;
        if (r < 10) { k0 += 0x9E3779B9u; k1 += 0xBB67AE85u; }
    }
}

// out(interior id) = amp*(2U-1), U from the first 64-bit draw of stream
// (seed, stream, id): its top 53 bits over 2^53.
template <typename R>
__global__ void philox_fill_kernel(Geo g, R* __restrict__ dst, int padded, uint64_t seed, uint32_t stream, double amp,
                                   int add, double off) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= g.nin) return;
    uint32_t c[4] = {0u, stream, (uint32_t)t, (uint32_t)((unsigned long long)t >> 32)};
    philox4x32(c, (uint32_t)(seed >> 32), (uint32_t)seed);
    uint64_t x = ((uint64_t)c[1] << 32) | (uint64_t)c[0];
    double u01 = (double)(x >> 11) * 0x1.0p-53;
    double val = amp * (2.0 * u01 - 1.0);
    int i = (int)(t % g.nx), j = (int)((t / g.nx) % g.ny), k = (int)(t / ((long long)g.nx * g.ny));
    long long q = padded ? pidx(g, i, j, k) : t;
    dst[q] = add ? R((double)dst[q] + val) : R(val - off);
}

template <typename R>
__global__ void padded_to_interior_kernel(Geo g, const R* __restrict__ a, R* __restrict__ b) {
    int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, k = blockIdx.z;
    if (i < g.nx) b[iidx(g, i, j, k)] = a[pidx(g, i, j, k)];
}
