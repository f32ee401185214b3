// aeo_sweep_wpair.cuh -- the FP32 WENO sweep on cell pairs, every face once.
//
// The WENO-JS5 / WENO-Z5 flux forms of the uniform Boussinesq core
// (src/AdvectionSchemes.jl:240-255, :319-333, :623-699, :1203-1256) on the
// paired FP32 instructions of sm_100 (aeo_f2.cuh): a thread owns two
// x-adjacent cells, and every reconstruction runs on two faces at once.
//
// A CTA owns a 32 x 8 tile (16 x 8 threads) and marches up a chunk of
// levels.  The planes of u, v, w and theta (x from i0-4, 40 wide; y halo 3)
// come by TMA into a ring of seven slots: levels k-3 .. k+3 at the chunk's
// first level, then k-2 .. k+3 with one level in flight.  Per level:
//   face phase -- the x faces (8 rows x 33 faces) and the y faces (9 rows x
//     32 faces) of all four fields, two faces an item, into shared memory;
//     x and y items fill whole warps, so every branch is warp-uniform;
//   cell phase -- each pair takes the differences of its shared x and y
//     fluxes, computes the top z face of its own column (the bottom one is
//     the top face of the level below, carried in registers), and the rest
//     of the tendency (viscosity, buoyancy, Coriolis, sponge) runs the same
//     sweep_point arithmetic as every other form.
// Each face is reconstructed once: 12.6 reconstructions a cell pair and
// level against 20 a cell in the cell-local FP32 form.  The x and y items run
// in rows of 16 pairs, so a half-warp reads one 128-byte row of a plane.
//
// The advecting velocity of a face and the face value multiply exactly as in
// the FP64 shared-face form (aeo_sweep_tile.cuh), so the two precisions run
// the same expression tree; the WENO divisions are a reciprocal and a product
// (2 ulp; every denominator lies in the normal range, as for wdiv).
//
// Waits are bounded (AEO_WAIT_LIMIT): a CTA whose plane did not arrive
// records AEO_ERR_FLAG_TMA, drains the copies it issued (bounded) and returns.
#pragma once

#include "aeo_f2.cuh"
#include "aeo_sweep_pair.cuh"   // PairAcc, PairNut (and the tile machinery)

__device__ __forceinline__ F2 ld2s(const float* p) { return F2(*reinterpret_cast<const float2*>(p)); }
__device__ __forceinline__ float2 ldf2(const float* p) { return *reinterpret_cast<const float2*>(p); }
__device__ __forceinline__ F2 f2abs(F2 x) { return F2(fabsf(x.v.x), fabsf(x.v.y)); }
// a / b as a times the approximate reciprocal of b (rcp.approx, 1 ulp; the
// quotient within 2 ulp, as __fdividef), the two products one paired multiply
__device__ __forceinline__ float rcp_approx(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ F2 f2wdiv(F2 a, F2 b) { return F2(a * F2(rcp_approx(b.v.x), rcp_approx(b.v.y))); }
__device__ __forceinline__ F2 f2pick(bool px, bool py, F2 a, F2 b) {
    return F2(px ? a.v.x : b.v.x, py ? a.v.y : b.v.y);
}

// weno5_left (aeo_sweep.cuh) on two faces
template <int ADV>
__device__ __forceinline__ F2 weno5_left_f2(F2 v1, F2 v2, F2 v3, F2 v4, F2 v5) {
    // the candidate values as the integer combinations over 6 (rounded
    // coefficients 1/3, 7/6, 11/6 would not sum to one, and a uniform field
    // would reconstruct with a bias that drifts the kinetic energy); the half
    // second differences with the 1/2 folded in (exact for a uniform field)
    const F2 s6(float(1.0 / 6.0)), two(2.f), half(0.5f), c133(float(13.0 / 3.0));
    const F2 q0 = F2(two * v1 - F2(7.f) * v2 + F2(11.f) * v3) * s6;
    const F2 q1 = F2(F2(5.f) * v3 - v2 + two * v4) * s6;
    const F2 q2 = F2(two * v3 + F2(5.f) * v4 - v5) * s6;
    const F2 d2a = half * (v1 + v3) - v2;
    const F2 d2b = half * (v2 + v4) - v3;
    const F2 d2c = half * (v3 + v5) - v4;
    const F2 e0 = F2(v1 - F2(4.f) * v2 + F2(3.f) * v3) * half;
    const F2 e1 = (v4 - v2) * half;
    const F2 e2 = F2(F2(4.f) * v4 - F2(3.f) * v3 - v5) * half;
    const F2 b0 = e0 * e0 + c133 * (d2a * d2a);
    const F2 b1 = e1 * e1 + c133 * (d2b * d2b);
    const F2 b2 = e2 * e2 + c133 * (d2c * d2c);
    F2 a0, a1, a2;
    if constexpr (ADV == 2) {   // WENO-Z5, p = 2, eps = eps(Float32)^2
        const F2 eps(1.4210854715202004e-14f), one(1.f);
        const F2 tau = f2abs(b0 - b2);
        const F2 t0 = f2wdiv(tau, b0 + eps), t1 = f2wdiv(tau, b1 + eps), t2 = f2wdiv(tau, b2 + eps);
        a0 = F2(0.1f) * (one + t0 * t0);
        a1 = F2(0.6f) * (one + t1 * t1);
        a2 = F2(0.3f) * (one + t2 * t2);
    } else {                    // WENO-JS5, eps = 1e-6
        const F2 e(1e-6f);
        const F2 s0 = b0 + e, s1 = b1 + e, s2 = b2 + e;
        a0 = f2wdiv(F2(0.1f), s0 * s0);
        a1 = f2wdiv(F2(0.6f), s1 * s1);
        a2 = f2wdiv(F2(0.3f), s2 * s2);
    }
    return f2wdiv(a0 * q0 + a1 * q1 + a2 * q2, a0 + a1 + a2);
}

// the upwinded value of two faces (weno_upwind lane by lane)
template <int ADV>
__device__ __forceinline__ F2 weno_upwind_f2(F2 vel, F2 f0, F2 f1, F2 f2, F2 f3, F2 f4, F2 f5) {
    const bool px = vel.v.x >= 0.f, py = vel.v.y >= 0.f;
    return weno5_left_f2<ADV>(f2pick(px, py, f0, f5), f2pick(px, py, f1, f4), f2pick(px, py, f2, f3),
                              f2pick(px, py, f3, f2), f2pick(px, py, f4, f1));
}

struct WPairShape {
    static constexpr int TXT = 16, TX = 2 * TXT, TY = 8, NT = TXT * TY, NWARP = NT / 32;
    static constexpr int HH = 3;
    static constexpr int NS = 7;
    static constexpr int PW = TX + 8, PH = TY + 2 * HH, PSZ = PW * PH;
    static constexpr int PSZA = (int)(((PSZ * sizeof(float) + 127) / 128) * 128 / sizeof(float));
    static constexpr int FXW = TX + 2;                  // x faces 0 .. TX of a row (+1 unused)
    static constexpr int FXN = TY * FXW, FYN = (TY + 1) * TX;
    // face-pair items of a level, whole warps of one kind: y faces two rows of
    // 16 pairs a warp (4 fields x 9 rows), x faces 0 .. 31 two rows a warp
    // (4 fields x 8 rows), and one warp of the 32 east-edge faces (face 32 of
    // every row and field, paired with face 33)
    static constexpr int NYW = 4 * (TY + 1) / 2, NXW = 4 * TY / 2;
    static constexpr size_t PLANES_BYTES = (size_t)NS * 4 * PSZA * sizeof(float);
    static constexpr size_t FLUX_BYTES = (((size_t)4 * (FXN + FYN) * sizeof(float) + 127) / 128) * 128;
    static constexpr size_t BAR_BYTES = 128;
    static constexpr size_t SMEM = PLANES_BYTES + FLUX_BYTES + BAR_BYTES + 128;
    static constexpr int CTAS_PER_SM = 3;
    static_assert(TXT == 16 && 4 * TY == 32, "two rows of pairs a warp; one edge warp");
    static_assert(NS * 8 <= (int)BAR_BYTES, "mbarrier block");
    static_assert(PW % 2 == 0 && PSZA % 2 == 0 && FXW % 2 == 0, "pairs stay 8-byte aligned");
    static_assert(SMEM + 1024 <= 228 * 1024 / CTAS_PER_SM, "three CTAs an SM");
};

// One face-pair item of field f: b is the plane offset of the cell after the
// first face (x faces: faces fi, fi+1 with b at cell fi; y faces: the faces
// below the cells of row fj).  The advecting velocity is the mean of the
// component at b and its second point: f = 0 the lower neighbour in x (y),
// read as the upper half of the pair two floats down; f = 1 one row down;
// f = 2 one level down; f = 3 the point itself.
template <int ADV, bool XF>
__device__ __forceinline__ F2 face_item(const float* pk, const float* pkm, int f, int b) {
    using S = WPairShape;
    const float* vb = pk + (XF ? 0 : S::PSZA) + b;   // the advecting component: u for x faces, v for y
    const F2 p0 = ld2s(vb);
    const float* pa = f == 0 ? vb - 2 : (f == 1 ? vb - S::PW : (f == 2 ? pkm + (XF ? 0 : S::PSZA) + b : vb));
    const float2 A = ldf2(pa);
    const F2 vel = (F2(f == 0 ? make_float2(A.y, p0.v.x) : A) + p0) * F2(0.5f);
    const float* F = pk + f * S::PSZA + b;
    F2 val;
    if constexpr (XF) {
        const float2 L0 = ldf2(F - 4), L1 = ldf2(F - 2), L2 = ldf2(F), L3 = ldf2(F + 2);
        val = weno_upwind_f2<ADV>(vel, F2(L0.y, L1.x), F2(L1), F2(L1.y, L2.x), F2(L2), F2(L2.y, L3.x), F2(L3));
    } else {
        val = weno_upwind_f2<ADV>(vel, ld2s(F - 3 * S::PW), ld2s(F - 2 * S::PW), ld2s(F - S::PW), ld2s(F),
                                  ld2s(F + S::PW), ld2s(F + 2 * S::PW));
    }
    return F2(vel * val);
}

template <int ADV>
__global__ void __launch_bounds__(128, 3) sweep_wpair_kernel(const __grid_constant__ TileMaps maps,
                                                             SweepArgs<float> a, int kchunk, int* err) {
    using S = WPairShape;
    using R = float;
    extern __shared__ __align__(128) unsigned char smem_tile[];
    unsigned char* sbase = smem_tile + ((128u - (smem_u32(smem_tile) & 127u)) & 127u);
    float* planes = reinterpret_cast<float*>(sbase);
    float* fxs = reinterpret_cast<float*>(sbase + S::PLANES_BYTES);
    float* fys = fxs + 4 * S::FXN;
    uint64_t* bars = reinterpret_cast<uint64_t*>(sbase + S::PLANES_BYTES + S::FLUX_BYTES);

    const Geo& g = a.g;
    const int tx = threadIdx.x, ty = threadIdx.y, tid = tx + S::TXT * ty;
    const int lane = tid & 31, warp = tid >> 5;
    const int i0 = blockIdx.x * S::TX, j0 = blockIdx.y * S::TY;
    const int kbeg = blockIdx.z * kchunk, kend = min(g.nz, kbeg + kchunk);
    const int i = i0 + 2 * tx, j = j0 + ty;
    const bool active = i < g.nx && j < g.ny;   // nx is even: the pair is whole
    const int Lfirst = kbeg - 3;                 // the bottom face of level kbeg reads kbeg-3
    const int Llast = kend + 2;                  // the top face of level kend-1 reads kend+2
    const uint32_t bytes = 4u * S::PSZ * sizeof(float);

    auto slot_of = [&](int L) { return (L - Lfirst) % S::NS; };
    auto parity_of = [&](int L) { return (uint32_t)(((L - Lfirst) / S::NS) & 1); };
    auto issue = [&](int L) {
        uint64_t* b = bars + slot_of(L);
        mbar_expect_tx(b, bytes);
        const int x = i0 + AEO_HX - 4, y = j0 + AEO_H - S::HH, z = L + AEO_H;
        float* d = planes + slot_of(L) * 4 * S::PSZA;
        tma_load_3d(d, &maps.u, b, x, y, z);
        tma_load_3d(d + S::PSZA, &maps.v, b, x, y, z);
        tma_load_3d(d + 2 * S::PSZA, &maps.w, b, x, y, z);
        tma_load_3d(d + 3 * S::PSZA, &maps.t, b, x, y, z);
    };

    if (tid == 0) {
        for (int s = 0; s < S::NS; ++s) mbar_init(bars + s, 1);
        fence_mbar_init();
    }
    __syncthreads();
    int Lissued = min(Llast, Lfirst + S::NS - 1);
    if (tid == 0)
        for (int L = Lfirst; L <= Lissued; ++L) issue(L);

    // the thread's face items: a warp takes rows 2w and 2w+1 (half-warp hrow,
    // pair pc) of the 36 (field, face row) y rows, w = warp, warp+4, ..., then
    // of the 32 (field, row) x rows; the edge warp (w = NXW) takes the east
    // faces 32, 33 of row lane (field lane / 8, row lane % 8)
    const int hrow = lane >> 4, pc = lane & 15;
    const R dt = R(__ldg(a.dtp));
    const Met<R, true> m(g);
    const int vbase = (ty + S::HH) * S::PW + 4 + 2 * tx;   // the thread's pair on a plane
    F2 zb[4];          // the bottom z fluxes of the level (the top ones of the level below)
    bool zvalid = false;
    bool failed = false;
    int c0 = 0;        // ring slot of level k-3
    for (int k = kbeg; k < kend; ++k, c0 = (c0 + 1 == S::NS) ? 0 : c0 + 1) {
        if (k > kbeg) {
            // every thread is past level k-1: the slots of the levels below k-2 are free
            if (__syncthreads_or(failed)) { failed = true; break; }
            const int Lto = min(Llast, k + 4);
            if (tid == 0)
                for (int L = Lissued + 1; L <= Lto; ++L) issue(L);
            Lissued = max(Lissued, Lto);
        }
        // the plane of level k-3+d
        const float* pl[S::NS];
#pragma unroll
        for (int d = 0; d < S::NS; ++d) pl[d] = planes + ((c0 + d) % S::NS) * (4 * S::PSZA);
        bool ok = true;
        for (int L = (k == kbeg ? Lfirst : k + 3); L <= min(Llast, k + 3); ++L)
            ok = ok && mbar_wait_bounded(bars + slot_of(L), parity_of(L));
        failed = !ok;

        // the step-start theta of the pair (stages 2, 3), loaded ahead of the face phase
        float2 th0v = make_float2(0.f, 0.f);
        if (a.stage && active) th0v = *reinterpret_cast<const float2*>(a.th0 + pidx(g, i, j, k));

        // ---- face phase: the x and y faces of the tile, two a thread-item
        {
            const float* pk = pl[3];
            const float* pkm = pl[2];
#pragma unroll 2
            for (int w = warp; w < S::NYW; w += S::NWARP) {
                const int row = 2 * w + hrow, f = row / (S::TY + 1), fj = row - f * (S::TY + 1);
                const int b = (fj + S::HH) * S::PW + 4 + 2 * pc;
                *reinterpret_cast<float2*>(fys + f * S::FYN + fj * S::TX + 2 * pc) =
                    face_item<ADV, false>(pk, pkm, f, b).v;
            }
            // (started two warps on, so that the edge warp lands on a warp with four y items)
#pragma unroll 2
            for (int w = (warp + 2) % S::NWARP; w <= S::NXW; w += S::NWARP) {
                int f, fj, fi;
                if (w < S::NXW) {
                    const int row = 2 * w + hrow;
                    f = row / S::TY; fj = row - f * S::TY; fi = 2 * pc;
                } else {
                    f = lane / S::TY; fj = lane - f * S::TY; fi = S::TX;
                }
                const int b = (fj + S::HH) * S::PW + 4 + fi;
                *reinterpret_cast<float2*>(fxs + f * S::FXN + fj * S::FXW + fi) = face_item<ADV, true>(pk, pkm, f, b).v;
            }
        }
        if (__syncthreads_or(failed)) { failed = true; break; }

        // ---- cell phase
        if (active) {
            const float* lp[3] = {pl[2] + vbase, pl[3] + vbase, pl[4] + vbase};
            const PairAcc<1, S::PW, 0> U{lp};
            const PairAcc<1, S::PW, S::PSZA> V{lp};
            const PairAcc<1, S::PW, 2 * S::PSZA> W{lp};
            const PairAcc<1, S::PW, 3 * S::PSZA> T{lp};
            PairNut<S::PW> N;
            N.p[0] = N.p[1] = N.p[2] = planes;
            // the z face above level k-3+d of field f at the thread's pair (d = 2: the
            // bottom face of level k, d = 3: its top face)
            auto zflux = [&](int f, int d) -> F2 {
                const float* wq = pl[d + 1] + 2 * S::PSZA + vbase;
                const F2 p0 = ld2s(wq);
                const float* pa = f == 0 ? wq - 2 : (f == 1 ? wq - S::PW : (f == 2 ? pl[d] + 2 * S::PSZA + vbase : wq));
                const float2 A = ldf2(pa);
                const F2 vel = (F2(f == 0 ? make_float2(A.y, p0.v.x) : A) + p0) * F2(0.5f);
                const int fo = f * S::PSZA + vbase;
                const F2 val = weno_upwind_f2<ADV>(vel, ld2s(pl[d - 2] + fo), ld2s(pl[d - 1] + fo), ld2s(pl[d] + fo),
                                                   ld2s(pl[d + 1] + fo), ld2s(pl[d + 2] + fo), ld2s(pl[d + 3] + fo));
                return F2(vel * val);
            };
            const F2 idx(R(g.idx)), idy(R(g.idy)), idz(R(g.idz));
            F2 adv[4];
#pragma unroll
            for (int f = 0; f < 4; ++f) {
                const F2 ft = zflux(f, 3);
                const F2 fb = zvalid ? zb[f] : zflux(f, 2);
                zb[f] = ft;
                const float* fx = fxs + f * S::FXN + ty * S::FXW + 2 * tx;
                const float2 xa = ldf2(fx), xb = ldf2(fx + 2);
                const float* fy = fys + f * S::FYN + ty * S::TX + 2 * tx;
                const F2 dx = (F2(xa.y, xb.x) - F2(xa)) * idx;
                const F2 dy = (ld2s(fy + S::TX) - ld2s(fy)) * idy;
                adv[f] = F2(0.f) - (dx + dy + (ft - fb) * idz);
            }
            zvalid = true;
            F2 tu = adv[0], tv = adv[1], tw = adv[2], tt = adv[3];
            sweep_point<R, ADV, false, false, true, true, false>(m, a, g, k, U, V, W, T, N, tu, tv, tw, tt);
            const long long qi = iidx(g, i, j, k), q = pidx(g, i, j, k);
            const F2 fdt(dt);
            *reinterpret_cast<float2*>(a.us + qi) = (U(0, 0, 0) + fdt * tu).v;
            *reinterpret_cast<float2*>(a.vs + qi) = (V(0, 0, 0) + fdt * tv).v;
            *reinterpret_cast<float2*>(a.ws + qi) =
                (g.bc_z == 1 && k == 0) ? make_float2(0.f, 0.f) : (W(0, 0, 0) + fdt * tw).v;
            F2 tn = T(0, 0, 0) + fdt * tt;
            if (a.stage) tn = rk_combine(a.ca, a.cb, F2(th0v), tn);
            *reinterpret_cast<float2*>(a.th_out + q) = tn.v;
        }
    }
    if (failed) {
        if (tid == 0) atomicOr(err, AEO_ERR_FLAG_TMA);
        // drain the copies this CTA issued before returning (bounded)
        for (int L = max(Lfirst, Lissued - S::NS + 1); L <= Lissued; ++L) mbar_wait_bounded(bars + slot_of(L), parity_of(L));
    }
}
