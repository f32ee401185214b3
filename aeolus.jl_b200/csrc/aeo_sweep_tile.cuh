// aeo_sweep_tile.cuh -- the tiled form of the fused sweep for sm_100a.
//
// A CTA owns a 32 x 8 column tile and marches up a chunk of levels.  The
// xy-planes of u, v, w and theta (with an xy halo) live in a shared-memory
// ring of slots that TMA fills: one elected thread issues a 3-D tile load
// (cp.async.bulk.tensor, no multicast) per field and level, completing on the
// slot's mbarrier, one level ahead of the one being computed.  The
// Smagorinsky eddy viscosity is computed in-tile for each level into a
// three-plane ring, so the separate nut pass and its halo fill disappear.
// Every point then runs the same sweep_point arithmetic as the direct form
// (aeo_sweep.cuh), reading its neighbours from shared memory.
//
// Waits on the mbarriers are bounded: after AEO_WAIT_LIMIT polls the CTA
// records AEO_ERR_FLAG_TMA in the error word, drains the copies it issued
// (again bounded) and returns; the host reports the failure after the step.
#pragma once

#include <cuda.h>

#include "aeo_sweep.cuh"
#include "aeo_dynamic.cuh"

#define AEO_WAIT_LIMIT (1u << 22)
#define AEO_ERR_FLAG_TMA 2

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
    for (uint32_t it = 0; it < AEO_WAIT_LIMIT; ++it)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y, int z) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], [%2];"
        ::"r"(smem_u32(dst)), "l"(map), "r"(smem_u32(bar)), "r"(x), "r"(y), "r"(z)
        : "memory");
}

template <typename R, int ADV, bool SGS>
struct TileShape {
    static constexpr int TX = 32, TY = 8, NT = TX * TY;
    static constexpr int HH = ADV ? 3 : 2;               // xy halo of the planes
    static constexpr int ZL = ADV ? 3 : (SGS ? 2 : 1);   // levels below the point
    static constexpr int ZH = ADV ? 3 : (SGS ? 2 : 1);   // levels above
    static constexpr int NW = ZL + ZH + 1;
    // ring slots: FP32 rounds the window + 1 up to a power of two (slot
    // arithmetic is a mask; the extra slots load further ahead), FP64 keeps
    // window + 1 so that two CTAs fit an SM
    static constexpr int NS = sizeof(R) == 8 ? NW + 1 : (NW + 1 <= 4 ? 4 : (NW + 1 <= 8 ? 8 : 16));
    static constexpr int LOOK = NS - NW;                 // levels loaded ahead
    static constexpr int PW = TX + 8;                    // row: x from i0-4 (16-byte aligned TMA start)
    static constexpr int PH = TY + 2 * HH;
    static constexpr int PSZ = PW * PH;                  // elements of one field-plane (the TMA box)
    static constexpr int PSZA = (int)(((PSZ * sizeof(R) + 127) / 128) * 128 / sizeof(R));
    static constexpr int NPW = TX + 2, NPH = TY + 2, NPS = NPW * NPH;  // nut plane with halo 1
    static constexpr size_t PLANES_BYTES = (size_t)NS * 4 * PSZA * sizeof(R);
    static constexpr size_t NUT_BYTES = SGS ? (((size_t)3 * NPS * sizeof(R) + 127) / 128) * 128 : 0;
    // WENO in FP64: the x- and y-face fluxes of the level's tile, [4][TY][TX+1] and
    // [4][TY+1][TX], computed once per face; FP32 reconstructions are cheap
    // enough that recomputing a face in both cells (straight-line code, no
    // extra barrier) is faster
    static constexpr bool SHARE = ADV > 0 && sizeof(R) == 8;
    static constexpr int FXN = TY * (TX + 1), FYN = (TY + 1) * TX;
    static constexpr int FPF = 576;                      // face entries per field: x 264 padded to 288, y 288
    static constexpr size_t FLUX_BYTES = SHARE ? (((size_t)4 * (FXN + FYN) * sizeof(R) + 127) / 128) * 128 : 0;
    static constexpr size_t BAR_BYTES = 128;
    static_assert(NS * 8 <= (int)BAR_BYTES, "mbarrier block");
    static_assert(TX == 32 && NPS == TX * NPH + 2 * NPH, "the eddy-viscosity loop maps warps to 32-column rows");
    // + the chunk's per-level factors, LV_N rows of NLT (a chunk has at most
    // KCH levels), + alignment slack
    static constexpr int KCH = 32, NLT = KCH + 2 * AEO_LH;
    static constexpr size_t SMEM =
        PLANES_BYTES + NUT_BYTES + FLUX_BYTES + BAR_BYTES + (size_t)LV_N * NLT * sizeof(R) + 128;
    // the AMD closure's kappa_t planes (the nut planes' layout) after the rest
    static constexpr size_t KT_BYTE = ((SMEM - 128 + 127) / 128) * 128;
    static constexpr int KT_OFS = (int)((KT_BYTE - PLANES_BYTES) / sizeof(R));   // elements past nutp
    static constexpr size_t SMEM_AMD = KT_BYTE + NUT_BYTES + 128;
    static_assert(!ADV || (FPF % 32 == 0 && FXN <= FPF / 2 && FYN == FPF / 2 && (4 * FPF) % NT == 0),
                  "one field per warp in the face phase");
};

struct TileMaps {
    CUtensorMap u, v, w, t;
};

// Accessor of one field around the thread's point: level k+dk is the ring
// plane lp[dk+ZL] (pointers at the thread's point, field 0), field f sits
// FOFS elements further.  Every index but the plane pointer is a constant.
template <typename R, int ZL, int PW, int FOFS>
struct SmAcc {
    const R* const* lp;
    __device__ __forceinline__ R operator()(int di, int dj, int dk) const { return lp[dk + ZL][FOFS + dj * PW + di]; }
};

// the same with the field offset a (warp-uniform) runtime value
template <typename R, int ZL, int PW>
struct SmAccF {
    const R* const* lp;
    int fofs;
    __device__ __forceinline__ R operator()(int di, int dj, int dk) const { return lp[dk + ZL][fofs + dj * PW + di]; }
};

template <typename R, int NPW>
struct NutAcc {
    const R* p[3];  // levels k-1, k, k+1 at the thread's point
    __device__ __forceinline__ R operator()(int di, int dj, int dk) const { return p[dk + 1][dj * NPW + di]; }
    __device__ __forceinline__ NutAcc shifted(int o) const { return NutAcc{{p[0] + o, p[1] + o, p[2] + o}}; }
};

// CLOS: the closure of the coefficient pass: 0 the static ones (smag_point),
// 1 the anisotropic minimum-dissipation closure (its kappa_t planes KT_OFS
// elements past the nut planes), 2 dynamic Smagorinsky (cs2 per level or
// cell), 3 the TKE closure (tke_point; its kappa_t planes as the AMD's)
template <typename R, int ADV, bool SGS, bool ANEL, bool UNI, int CLOS = 0>
__global__ void __launch_bounds__(256) sweep_tile_kernel(const __grid_constant__ TileMaps maps, SweepArgs<R> a,
                                                         int kchunk, int* err) {
    using S = TileShape<R, ADV, SGS>;
    extern __shared__ __align__(128) unsigned char smem_tile[];
    // offsets from the shared array itself keep every pointer below in the
    // shared state space (plain ld.shared with constant offsets)
    unsigned char* sbase = smem_tile + ((128u - (smem_u32(smem_tile) & 127u)) & 127u);
    R* planes = reinterpret_cast<R*>(sbase);
    R* nutp = reinterpret_cast<R*>(sbase + S::PLANES_BYTES);
    R* fxs = reinterpret_cast<R*>(sbase + S::PLANES_BYTES + S::NUT_BYTES);   // WENO face fluxes
    R* fys = fxs + 4 * S::FXN;
    uint64_t* bars = reinterpret_cast<uint64_t*>(sbase + S::PLANES_BYTES + S::NUT_BYTES + S::FLUX_BYTES);
    R* lvs = reinterpret_cast<R*>(sbase + S::PLANES_BYTES + S::NUT_BYTES + S::FLUX_BYTES + S::BAR_BYTES);

    const Geo& g = a.g;
    const int tx = threadIdx.x, ty = threadIdx.y, tid = tx + S::TX * ty;
    const int i0 = blockIdx.x * S::TX, j0 = blockIdx.y * S::TY;
    const int kbeg = blockIdx.z * kchunk;
    const int kend = min(g.nz, kbeg + kchunk);
    const int i = i0 + tx, j = j0 + ty;
    const bool active = i < g.nx && j < g.ny;
    const int Lfirst = kbeg - S::ZL;             // first level held
    const int Llast = kend - 1 + S::ZH;          // last level needed
    const uint32_t bytes = 4u * S::PSZ * sizeof(R);

    auto slot_of = [&](int L) { return (L - Lfirst) % S::NS; };
    auto parity_of = [&](int L) { return (uint32_t)(((L - Lfirst) / S::NS) & 1); };
    auto plane = [&](int L) { return planes + (size_t)slot_of(L) * 4 * S::PSZA; };
    auto issue = [&](int L) {
        uint64_t* b = bars + slot_of(L);
        mbar_expect_tx(b, bytes);
        const int x = i0 + AEO_HX - 4, y = j0 + AEO_H - S::HH, z = L + AEO_H;
        R* d = plane(L);
        tma_load_3d(d, &maps.u, b, x, y, z);
        tma_load_3d(d + S::PSZA, &maps.v, b, x, y, z);
        tma_load_3d(d + 2 * S::PSZA, &maps.w, b, x, y, z);
        tma_load_3d(d + 3 * S::PSZA, &maps.t, b, x, y, z);
    };

    if (tid == 0) {
        for (int s = 0; s < S::NS; ++s) mbar_init(bars + s, 1);
        fence_mbar_init();
    }
    // the chunk's per-level factors: level k of row f at lvs[f * NLT + k + AEO_LH - kbeg]
    // (a compile-time row stride: every factor is one ld.shared off the level's base)
    const int nlt = kend - kbeg + 2 * AEO_LH;
    {
        const R* src = static_cast<const R*>(g.lvr);
        for (int e = tid; e < LV_N * S::NLT; e += S::NT) {
            const int f = e / S::NLT, kk = e - f * S::NLT;
            if (kk < nlt) lvs[e] = src[(size_t)f * g.lvn + kbeg + kk];
        }
    }
    __syncthreads();
    const Met<R, UNI> m(g, lvs, S::NLT, AEO_LH - kbeg);
    int Lissued = min(Llast, kbeg + S::ZH + S::LOOK);
    if (tid == 0)
        for (int L = Lfirst; L <= Lissued; ++L) issue(L);

    const R dt = R(__ldg(a.dtp));
    const int vbase = (ty + S::HH) * S::PW + (tx + 4);
    ZCarry<R> zc;   // the WENO z fluxes carried up the column
    zc.valid = false;
    bool failed = false;
    for (int k = kbeg; k < kend; ++k) {
        // the levels this iteration needs
        const int Lw0 = (k == kbeg) ? Lfirst : k + S::ZH;
        // one warp polls the mbarriers; the CTA barrier then releases the
        // others (it orders the copies the poll observed before their reads)
        bool ok = true;
        if (tid < 32)
            for (int L = Lw0; L <= k + S::ZH; ++L) ok = ok && mbar_wait_bounded(bars + slot_of(L), parity_of(L));
        if (__syncthreads_or(!ok)) { failed = true; break; }
        // every thread is past level k-1: the slot of level k-1-ZL takes level k+ZH+LOOK
        if (k > kbeg) {
            const int Ln = k + S::ZH + S::LOOK;
            if (Ln <= Llast) {
                if (tid == 0) issue(Ln);
                Lissued = Ln;
            }
        }

        const R* lp[S::NW];
#pragma unroll
        for (int d = 0; d < S::NW; ++d) lp[d] = plane(k - S::ZL + d) + vbase;
        const SmAcc<R, S::ZL, S::PW, 0> U{lp};
        const SmAcc<R, S::ZL, S::PW, S::PSZA> V{lp};
        const SmAcc<R, S::ZL, S::PW, 2 * S::PSZA> W{lp};
        const SmAcc<R, S::ZL, S::PW, 3 * S::PSZA> T{lp};

        NutAcc<R, S::NPW> N;
        if (SGS) {
            // eddy viscosity of the levels k-1 .. k+1 (first iteration) or k+1
            const int Lz0 = (k == kbeg) ? k - 1 : k + 1;
            bool mirror = false;
            for (int L = Lz0; L <= k + 1; ++L) {
                if (g.bc_z == 1 && (L < 0 || L >= g.nz)) { mirror = true; continue; }  // from the level inside
                R* np = nutp + (size_t)((L + 3) % 3) * S::NPS;
                const R* sp[3];
#pragma unroll
                for (int d = 0; d < 3; ++d) sp[d] = plane(L - 1 + d);
                // warps take whole rows of the tile's 32 columns (contiguous,
                // conflict-free), the two edge columns come last
                for (int e = tid; e < S::NPS; e += S::NT) {
                    int cj, ci;
                    if (e < S::TX * S::NPH) { cj = e >> 5; ci = (e & 31) + 1; }
                    else { const int x = e - S::TX * S::NPH; cj = x >> 1; ci = (x & 1) ? S::NPW - 1 : 0; }
                    // open faces: a ring cell beyond one takes the mirrored cell's value
                    const int gi = open_src(g.ox, i0 + ci - 1, g.nx), gj = open_src(g.oy, j0 + cj - 1, g.ny);
                    const int b = (gj - j0 + S::HH) * S::PW + (gi - i0 + 4);
                    const R* q[3] = {sp[0] + b, sp[1] + b, sp[2] + b};
                    const SmAcc<R, 1, S::PW, 0> Uq{q};
                    const SmAcc<R, 1, S::PW, S::PSZA> Vq{q};
                    const SmAcc<R, 1, S::PW, 2 * S::PSZA> Wq{q};
                    if constexpr (CLOS == 2) {
                        const R c = R(dyn_cs2_cell(g, a.cs2, a.cs2f, gi, gj, L) * a.dyn_d2);
                        np[cj * S::NPW + ci] = c * strain_at<R, UNI>(m, g, L, Uq, Vq, Wq, (R*)nullptr);
                    } else if constexpr (CLOS == 1) {
                        const SmAcc<R, 1, S::PW, 3 * S::PSZA> Tq{q};
                        const NuKappa<R> nk = amd_point<R, UNI>(m, g, L, R(a.c_s), m.lv(LV_BGC, L), a.pr_t, Uq, Vq, Wq, Tq);
                        np[cj * S::NPW + ci] = nk.nu;
                        np[cj * S::NPW + ci + S::KT_OFS] = nk.ka;
                    } else if constexpr (CLOS == 3) {
                        const SmAcc<R, 1, S::PW, 3 * S::PSZA> Tq{q};
                        const NuKappa<R> nk = tke_point<R>(g, gi, gj, L, Tq(0, 0, -1), Tq(0, 0, 0), Tq(0, 0, 1));
                        np[cj * S::NPW + ci] = nk.nu;
                        np[cj * S::NPW + ci + S::KT_OFS] = nk.ka;
                    } else {
                        np[cj * S::NPW + ci] = smag_point<R, UNI>(m, g, L, R(a.c_s), Uq, Vq, Wq);
                    }
                }
            }
            __syncthreads();
            if (mirror) {
                // walls: the halo levels take the mirrored interior value
                for (int L = Lz0; L <= k + 1; ++L) {
                    if (!(g.bc_z == 1 && (L < 0 || L >= g.nz))) continue;
                    const int Ls = L < 0 ? -L - 1 : 2 * g.nz - 1 - L;
                    R* dst = nutp + (size_t)((L + 3) % 3) * S::NPS;
                    const R* src = nutp + (size_t)((Ls + 3) % 3) * S::NPS;
                    for (int e = tid; e < S::NPS; e += S::NT) dst[e] = src[e];
                    if (CLOS == 1 || CLOS == 3)
                        for (int e = tid; e < S::NPS; e += S::NT) dst[e + S::KT_OFS] = src[e + S::KT_OFS];
                }
                __syncthreads();
            }
            const int nb = (ty + 1) * S::NPW + (tx + 1);
#pragma unroll
            for (int d = 0; d < 3; ++d) N.p[d] = nutp + (size_t)((k - 1 + d + 3) % 3) * S::NPS + nb;
        } else {
            N.p[0] = N.p[1] = N.p[2] = nutp;
        }

        R tu, tv, tw, tt;
        if constexpr (S::SHARE) {
            // face phase: every x- and y-face flux of the tile once (a face is
            // shared by the two cells beside it); one field per warp
            const R* lp0[S::NW];
#pragma unroll
            for (int d = 0; d < S::NW; ++d) lp0[d] = plane(k - S::ZL + d);
#pragma unroll 3
            for (int q = 0; q < 4 * S::FPF / S::NT; ++q) {
                // branch-free: an x face and a y face differ only in the stencil
                // stride and the advecting field (u or v); the second velocity
                // point depends on the field only (f is warp-uniform, so is isx)
                const int e = tid + q * S::NT;
                const int f = e / S::FPF, r = e - f * S::FPF;
                const bool isx = r < S::FPF / 2;
                int rr = isx ? r : r - S::FPF / 2;
                const bool valid = !isx || rr < S::FXN;
                rr = valid ? rr : 0;
                const int fjx = rr / (S::TX + 1), fjy = rr / S::TX;
                const int fj = isx ? fjx : fjy;
                const int fi = isx ? rr - fjx * (S::TX + 1) : rr - fjy * S::TX;
                const int fb = (fj + S::HH) * S::PW + (fi + 4);
                const int st = isx ? 1 : S::PW;
                const int vofs = isx ? 0 : S::PSZA;
                const R* p0 = lp0[S::ZL] + fb;
                const R* p1 = (f == 2 ? lp0[S::ZL - 1] : lp0[S::ZL]) + fb + vofs + (f == 0 ? -1 : (f == 1 ? -S::PW : 0));
                const R a0 = p0[vofs], a1 = *p1;
                const R vel = f == 3 ? a0 : (a1 + a0) / R(2);
                const R* pf = p0 + f * S::PSZA;
                const R flux = vel * weno_upwind<R, ADV>(vel >= R(0), pf[-3 * st], pf[-2 * st], pf[-st], pf[0], pf[st],
                                                        pf[2 * st]);
                if (valid) {
                    if (isx) fxs[f * S::FXN + fj * (S::TX + 1) + fi] = flux;
                    else fys[f * S::FYN + fj * S::TX + fi] = flux;
                }
            }
            __syncthreads();
            if (active) {
                // cell phase: differences of the shared fluxes, the z fluxes carried up the column
                const R idx = R(g.idx), idy = R(g.idy), idz = R(g.idz);
                R adv[4];
#pragma unroll
                for (int f = 0; f < 4; ++f) {
                    const SmAccF<R, S::ZL, S::PW> F{lp, f * S::PSZA};
                    const R ft = weno_zflux<R, ADV, 0>(f, W, F);
                    const R fb = zc.valid ? zc.f[f] : weno_zflux<R, ADV, -1>(f, W, F);
                    zc.f[f] = ft;
                    const R* fx = fxs + f * S::FXN + ty * (S::TX + 1) + tx;
                    const R* fy = fys + f * S::FYN + ty * S::TX + tx;
                    adv[f] = R(0) - ((fx[1] - fx[0]) * idx + (fy[S::TX] - fy[0]) * idy + (ft - fb) * idz);
                }
                zc.valid = true;
                tu = adv[0]; tv = adv[1]; tw = adv[2]; tt = adv[3];
            }
        }
        if (active) {
            sweep_point<R, ADV, SGS, ANEL, UNI, S::SHARE, CLOS == 1 || CLOS == 3>(m, a, g, k, U, V, W, T, N, tu, tv, tw, tt,
                                                               (ADV > 0 && !S::SHARE) ? &zc : nullptr);
            if (ADV > 0 && !S::SHARE) zc.valid = true;
            const long long qi = iidx(g, i, j, k), q = pidx(g, i, j, k);
            a.us[qi] = U(0, 0, 0) + dt * tu;
            a.vs[qi] = V(0, 0, 0) + dt * tv;
            a.ws[qi] = (g.bc_z == 1 && k == 0) ? R(0) : W(0, 0, 0) + dt * tw;
            R tn = T(0, 0, 0) + dt * tt;
            if (a.stage) tn = rk_combine(a.ca, a.cb, a.th0[q], tn);
            a.th_out[q] = tn;
        }
    }
    if (failed) {
        if (tid == 0) atomicOr(err, AEO_ERR_FLAG_TMA);
        // drain the copies this CTA issued before returning (bounded)
        for (int L = max(Lfirst, Lissued - S::NS + 1); L <= Lissued; ++L) mbar_wait_bounded(bars + slot_of(L), parity_of(L));
    }
}
