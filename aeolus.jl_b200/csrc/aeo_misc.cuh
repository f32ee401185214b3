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
    R* xp;
    R* yp;
    R* bw;
    R* be;
    R* bs;
    R* bn;
    int ox, oy, L;
    int mode[4];
    // radiating (:convective) outflow (src/boundary_conditions/outflow.jl):
    // per side (west, east, south, north) the flag; the raw data planes, the
    // step-start snapshot and the stage-start buffers (the layout of xp / yp);
    // per plane point ([f][side][NZ][NY] x faces, [f][side][NZ][NX] y faces)
    // the phase speed (NaN: an inflow point) and the two stage-start
    // interior layers; the correction mode (0 uniform, 1 outflow only, 2
    // none) and the ledger (Q, residual, delta) of the last correction
    int rad[4];
    int corr;
    const R* xd;
    const R* yd;
    R* xs;
    R* ys;
    R* xv;
    R* yv;
    R* xc;
    R* yc;
    R* x1;
    R* y1;
    R* x2;
    R* y2;
    double* led;
    const double* xw;     // weights of the normal planes' boundary faces, [side][Nz][Ny] / [side][Nz][Nx] (0 solid)
    const double* yw;
    // the :orlanski outflow (rad[q] == 2): the interior layer next to the face
    // at the previous step start per plane point, and (device) whether it is
    // set and the length of the previous step
    R* xh;
    R* yh;
    int* hist_ok;
    double* last_dt;
};

// ---- radiating outflow (src/boundary_conditions/outflow.jl) --------------------
// Plane geometry: element (layer l, tangential a, b) of plane (f, side) of
// axis 0 (a = storage j, b = storage k) or 1 (a = storage i, b = storage k).
template <typename R>
__device__ __forceinline__ size_t ob_pi(const Geo& g, const OpenSet<R>& ob, int axis, int f, int side, int l, int a,
                                        int b) {
    const int NX = g.nx + 2 * AEO_H, NY = g.ny + 2 * AEO_H, NZ = g.nz + 2 * AEO_H;
    if (axis == 0) return (((size_t)(f * 2 + side) * NZ + b) * NY + a) * ob.L + l;
    return (((size_t)(f * 2 + side) * NZ + b) * ob.L + l) * NX + a;
}
// the storage index of a plane's boundary layer, its local layer, the
// outward step and the layer count (_boundary_storage / _boundary_local /
// _outward, outflow.jl:104-106)
__device__ __forceinline__ void ob_geom(const Geo& g, int axis, int f, int side, int* sb, int* lb, int* o, int* nl) {
    const int H = AEO_H, N = axis == 0 ? g.nx : g.ny;
    if (side) { *sb = H + N; *lb = 0; *o = 1; *nl = H; }
    else { *sb = f == axis ? H : H - 1; *lb = *sb; *o = -1; *nl = *sb + 1; }
}
// a tangential plane point t of the x faces (t < 8 NZ NY) or the y faces
__device__ __forceinline__ bool ob_point(const Geo& g, long long t, int* axis, int* f, int* side, int* a, int* b) {
    const long long NX = g.nx + 2 * AEO_H, NY = g.ny + 2 * AEO_H, NZ = g.nz + 2 * AEO_H;
    long long n = 8 * NZ * NY;
    int ax = 0;
    if (t >= n) { t -= n; ax = 1; n = 8 * NZ * NX; if (t >= n) return false; }
    const long long NA = ax == 0 ? NY : NX;
    *a = (int)(t % NA); t /= NA;
    *b = (int)(t % NZ); t /= NZ;
    *side = (int)(t % 2);
    *f = (int)(t / 2);
    *axis = ax;
    return true;
}
template <typename R>
__device__ __forceinline__ R field_at(const Geo& g, const R* d, int axis, int li, int a, int b) {
    return axis == 0 ? d[pidx(g, li - AEO_H, a - AEO_H, b - AEO_H)] : d[pidx(g, a - AEO_H, li - AEO_H, b - AEO_H)];
}

// prepare_open_boundaries! (open_boundary.jl:1189-1200, outflow.jl:113-182):
// per radiating plane point the phase speed c = the outward normal velocity
// of the boundary face (the mean of two faces for a component staggered
// along the face), NaN where it does not point out (the data is kept)
//
// :orlanski (outflow.jl:152-181): for the tangential velocities and the
// scalars, c = -(dphi/dt)/(dphi/dn) at the interior layer next to the face
// from its value at this and at the previous step start, clipped to
// [0, dn/dtau] (Miller & Thorpe 1981), NaN -> 0; the convective speed on the
// first step and for the normal velocity.  The fields are the step-start state.
template <typename R>
__global__ void ob_phase_kernel(Geo g, OpenSet<R> ob, const R* u, const R* v, const R* w, const R* th,
                                const double* __restrict__ dtp) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    int axis, f, side, a, b;
    if (!ob_point(g, t, &axis, &f, &side, &a, &b)) return;
    R* C = axis == 0 ? ob.xc : ob.yc;
    const long long ti = t - (axis == 0 ? 0 : 8LL * (g.nz + 2 * AEO_H) * (g.ny + 2 * AEO_H));
    const int mode = ob.rad[axis * 2 + side];
    if (!mode || ob.mode[f] != 0) { C[ti] = R(NAN); return; }
    R phi1 = R(0), phi2 = R(0);
    if (mode == 2) {
        int sb, lb, o, nl;
        ob_geom(g, axis, f, side, &sb, &lb, &o, &nl);
        const R* d = f == 0 ? u : f == 1 ? v : f == 2 ? w : th;
        phi1 = field_at(g, d, axis, sb - o, a, b);
        phi2 = field_at(g, d, axis, sb - 2 * o, a, b);
    }
    const R* P = axis == 0 ? ob.xp : ob.yp;
    const int fl = side ? 0 : AEO_H;
    const R sg = side ? R(1) : R(-1);
    const bool st1 = (axis == 0 && f == 1) || (axis == 1 && f == 0), st2 = f == 2;
    R un;
    if (st1) {
        const int am = a > 0 ? a - 1 : 0;
        un = sg * (P[ob_pi(g, ob, axis, axis, side, fl, am, b)] + P[ob_pi(g, ob, axis, axis, side, fl, a, b)]) / R(2);
    } else if (st2) {
        const int bm = b > 0 ? b - 1 : 0;
        un = sg * (P[ob_pi(g, ob, axis, axis, side, fl, a, bm)] + P[ob_pi(g, ob, axis, axis, side, fl, a, b)]) / R(2);
    } else {
        un = sg * P[ob_pi(g, ob, axis, axis, side, fl, a, b)];
    }
    R* Hs = axis == 0 ? ob.xh : ob.yh;
    if (!(un > R(0))) {
        C[ti] = R(NAN);
    } else if (mode == 2 && f != axis && *ob.hist_ok) {
        const double dtau = *ob.last_dt, dn = axis == 0 ? g.dx : g.dy;
        const double num = -((double)phi1 - (double)Hs[ti]) / dtau;
        const double den = ((double)phi1 - (double)phi2) / dn;
        const double c = num / den;
        const double cmax = dn / dtau;
        C[ti] = R(c != c ? 0.0 : (c < 0.0 ? 0.0 : (c > cmax ? cmax : c)));
    } else {
        C[ti] = un;
    }
    if (mode == 2) Hs[ti] = phi1;
    (void)dtp;
}

// after the phase speeds of a step: the history is set, and this step's length
// is the next one's tau
__global__ void ob_hist_kernel(int* hist_ok, double* last_dt, const double* __restrict__ dtp) {
    *hist_ok = 1;
    *last_dt = *dtp;
}

// mark_open_boundary_stage! (outflow.jl:198-237): the two interior layers next
// to every radiating face at the start of a (sub)stage
template <typename R>
__global__ void ob_mark_kernel(Geo g, OpenSet<R> ob, const R* u, const R* v, const R* w, const R* th) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    int axis, f, side, a, b;
    if (!ob_point(g, t, &axis, &f, &side, &a, &b)) return;
    if (!ob.rad[axis * 2 + side]) return;
    const long long ti = t - (axis == 0 ? 0 : 8LL * (g.nz + 2 * AEO_H) * (g.ny + 2 * AEO_H));
    int sb, lb, o, nl;
    ob_geom(g, axis, f, side, &sb, &lb, &o, &nl);
    const R* d = f == 0 ? u : f == 1 ? v : f == 2 ? w : th;
    (axis == 0 ? ob.x1 : ob.y1)[ti] = field_at(g, d, axis, sb - o, a, b);
    (axis == 0 ? ob.x2 : ob.y2)[ti] = field_at(g, d, axis, sb - 2 * o, a, b);
}

// _radiate_body! (outflow.jl:262-285): at an outflow point every layer from
// the face outward, phi_b = phi_b0 - r (3 phi_b0 - 4 phi_{b-1}0 + phi_{b-2}0) / 2,
// r = min(c dt / dn, 1), from the stage-start values (the buffer before the
// update and the marked interior layers)
template <typename R>
__global__ void ob_radiate_kernel(Geo g, OpenSet<R> ob, const double* __restrict__ dtp) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    int axis, f, side, a, b;
    if (!ob_point(g, t, &axis, &f, &side, &a, &b)) return;
    if (!ob.rad[axis * 2 + side]) return;
    const long long ti = t - (axis == 0 ? 0 : 8LL * (g.nz + 2 * AEO_H) * (g.ny + 2 * AEO_H));
    const R c = (axis == 0 ? ob.xc : ob.yc)[ti];
    if (c != c) return;                                   // NaN: an inflow point keeps the data
    const R dn = R(axis == 0 ? g.dx : g.dy);
    const R r0 = c * R(*dtp) / dn, r = r0 < R(1) ? r0 : R(1);
    R i1 = (axis == 0 ? ob.x1 : ob.y1)[ti], i2 = (axis == 0 ? ob.x2 : ob.y2)[ti];
    int sb, lb, o, nl;
    ob_geom(g, axis, f, side, &sb, &lb, &o, &nl);
    R* Pl = axis == 0 ? ob.xp : ob.yp;
    const R* P0 = axis == 0 ? ob.xv : ob.yv;
    for (int q = 0, l = lb; q < nl; ++q, l += o) {
        const size_t e = ob_pi(g, ob, axis, f, side, l, a, b);
        const R p0 = P0[e];
        Pl[e] = p0 - r * (R(3) * p0 - R(4) * i1 + i2) / R(2);
        i2 = i1;
        i1 = p0;
    }
}

// correct_boundary_mass_flux! (open_boundary.jl:1024-1083) on the buffers, one
// block (FP64 sums in a fixed order), then the boundary-face arrays of the
// projection from the corrected buffers; led = (Q, residual, delta)
template <typename R>
__global__ void __launch_bounds__(1024) ob_correct_kernel(Geo g, OpenSet<R> ob) {
    __shared__ double red[3][1024];
    const int tid = threadIdx.x;
    const long long nxf = ob.ox ? 2LL * g.ny * g.nz : 0, nyf = ob.oy ? 2LL * g.nx * g.nz : 0;
    // face e of the normal planes: its buffer value, weighted area (0: solid) and outward sign
    auto face = [&](long long e, R** pv, double* area, double* sg) {
        int axis = 0;
        if (e >= nxf) { e -= nxf; axis = 1; }
        const double wt = (axis == 0 ? ob.xw : ob.yw)[e];
        const int nt = axis == 0 ? g.ny : g.nx;
        const int a = (int)(e % nt) + AEO_H;
        e /= nt;
        const int b = (int)(e % g.nz) + AEO_H;
        const int side = (int)(e / g.nz);
        *pv = (axis == 0 ? ob.xp : ob.yp) + ob_pi(g, ob, axis, axis, side, side ? 0 : AEO_H, a, b);
        *area = (axis == 0 ? g.dy : g.dx) * g.dz * wt;
        *sg = side ? 1.0 : -1.0;
    };
    double q = 0, ao = 0, aa = 0;
    for (long long e = tid; e < nxf + nyf; e += blockDim.x) {
        R* pv; double area, sg;
        face(e, &pv, &area, &sg);
        if (!(area > 0)) continue;
        const double out = sg * (double)*pv;
        q += out * area;
        if (out > 0) ao += area;
        aa += area;
    }
    red[0][tid] = q; red[1][tid] = ao; red[2][tid] = aa;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (tid < w)
            for (int c = 0; c < 3; ++c) red[c][tid] += red[c][tid + w];
        __syncthreads();
    }
    const double Q = red[0][0], Aout = red[1][0], Aall = red[2][0];
    __syncthreads();
    double delta = 0;
    bool only_out = ob.corr == 1;
    if (ob.corr != 2 && Q != 0) {
        double A = only_out ? Aout : Aall;
        if (A == 0) { only_out = false; A = Aall; }
        delta = Q / A;
        for (long long e = tid; e < nxf + nyf; e += blockDim.x) {
            R* pv; double area, sg;
            face(e, &pv, &area, &sg);
            if (area > 0 && (!only_out || sg * (double)*pv > 0)) *pv = R((double)*pv - sg * delta);
        }
    }
    __syncthreads();
    double rr = 0;
    for (long long e = tid; e < nxf + nyf; e += blockDim.x) {
        R* pv; double area, sg;
        face(e, &pv, &area, &sg);
        if (area > 0) rr += sg * (double)*pv * area;
    }
    red[0][tid] = rr;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (tid < w) red[0][tid] += red[0][tid + w];
        __syncthreads();
    }
    if (tid == 0) { ob.led[0] = Q; ob.led[1] = red[0][0]; ob.led[2] = delta; }
    // the projection's boundary-face values
    const int H = AEO_H;
    for (long long e = tid; e < (long long)g.ny * g.nz && ob.ox; e += blockDim.x) {
        const int j = (int)(e % g.ny), k = (int)(e / g.ny);
        ob.bw[e] = ob.xp[ob_pi(g, ob, 0, 0, 0, H, j + H, k + H)];
        ob.be[e] = ob.xp[ob_pi(g, ob, 0, 0, 1, 0, j + H, k + H)];
    }
    for (long long e = tid; e < (long long)g.nx * g.nz && ob.oy; e += blockDim.x) {
        const int i = (int)(e % g.nx), k = (int)(e / g.nx);
        ob.bs[e] = ob.yp[ob_pi(g, ob, 1, 1, 0, H, i + H, k + H)];
        ob.bn[e] = ob.yp[ob_pi(g, ob, 1, 1, 1, 0, i + H, k + H)];
    }
}

// combine_open_boundaries! (open_boundary.jl:1262-1280): buffer = a snapshot + b buffer
template <typename R>
__global__ void ob_combine_kernel(R* __restrict__ p, const R* __restrict__ snap, long long n, R ca, R cb) {
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
        p[q] = ca * snap[q] + cb * p[q];
}

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
    // v's south boundary face (interior j = 0) belongs to the south plane's
    // slab, which the y fill writes over every x after the x fill: beyond an
    // open x face it takes the south plane, not the x plane
    if (ob.oy && plane && pid == 1 && j == 0 && (i < 0 || i >= g.nx)) {
        v = ob.yp[((((size_t)(1 * 2) * NZ + kk + AEO_H) * ob.L + AEO_H) * NX) + i + AEO_H];
        return s > 0 ? v : -v;
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
