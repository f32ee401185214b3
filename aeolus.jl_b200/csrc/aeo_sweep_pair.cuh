// aeo_sweep_pair.cuh -- the FP32 centred sweep on cell pairs.
//
// The tiled sweep of aeo_sweep_tile.cuh with every thread owning two
// x-adjacent cells: the same sweep_point / smag_point arithmetic runs on F2
// values (aeo_f2.cuh), so each FP32 add, multiply or fused multiply-add
// serves both cells, and a neighbour pair at an even x-offset is one 8-byte
// shared load (an odd offset takes the halves of the two aligned pairs
// around it, which its even neighbours load anyway).
//
// A CTA owns 64 x 8 cells (32 x 8 threads) and marches up a chunk of levels;
// the planes of u, v, w and theta (x from i0-4, 72 wide, y halo 2) come by
// TMA into a ring one level ahead; the Smagorinsky eddy viscosity of each
// new level is computed in-tile on pairs (tile x -2 .. 65, y -1 .. 8).
#pragma once

#include "aeo_f2.cuh"

#include "aeo_sweep_tile.cuh"

// the AMD closure lane by lane
__device__ __forceinline__ NuKappa<F2> amd_lane(F2 ux, F2 uy, F2 uz, F2 vx, F2 vy, F2 vz, F2 wx, F2 wy, F2 wz, F2 tx,
                                                F2 ty, F2 tz, F2 d2x, F2 d2y, F2 d2z, F2 bg, F2 C, F2 pr_t) {
    const NuKappa<float> a = amd_lane<float>(ux.v.x, uy.v.x, uz.v.x, vx.v.x, vy.v.x, vz.v.x, wx.v.x, wy.v.x, wz.v.x,
                                             tx.v.x, ty.v.x, tz.v.x, d2x.v.x, d2y.v.x, d2z.v.x, bg.v.x, C.v.x, pr_t.v.x);
    const NuKappa<float> b = amd_lane<float>(ux.v.y, uy.v.y, uz.v.y, vx.v.y, vy.v.y, vz.v.y, wx.v.y, wy.v.y, wz.v.y,
                                             tx.v.y, ty.v.y, tz.v.y, d2x.v.y, d2y.v.y, d2z.v.y, bg.v.y, C.v.y, pr_t.v.y);
    NuKappa<F2> o;
    o.nu = F2(a.nu, b.nu);
    o.ka = F2(a.ka, b.ka);
    return o;
}

// the sigma-model operator lane by lane (the closed-form eigenproblem has no
// paired form)
__device__ __forceinline__ F2 sigma_operator(F2 g11, F2 g12, F2 g13, F2 g21, F2 g22, F2 g23, F2 g31, F2 g32, F2 g33) {
    return F2(sigma_operator<float>(g11.v.x, g12.v.x, g13.v.x, g21.v.x, g22.v.x, g23.v.x, g31.v.x, g32.v.x, g33.v.x),
              sigma_operator<float>(g11.v.y, g12.v.y, g13.v.y, g21.v.y, g22.v.y, g23.v.y, g31.v.y, g32.v.y, g33.v.y));
}

template <bool SGS>
struct PairShape {
    static constexpr int TXT = 32, TX = 2 * TXT, TY = 8, NT = TXT * TY;
    static constexpr int HH = 2;
    static constexpr int ZL = SGS ? 2 : 1, ZH = SGS ? 2 : 1;
    static constexpr int NW = ZL + ZH + 1;
    static constexpr int NS = NW + 1;                    // one level ahead (two CTAs per SM)
    static constexpr int PW = TX + 8;                    // x from i0-4: 16-byte aligned TMA start
    static constexpr int PH = TY + 2 * HH;
    static constexpr int PSZ = PW * PH;
    static constexpr int PSZA = (int)(((PSZ * sizeof(float) + 127) / 128) * 128 / sizeof(float));
    static constexpr int NPW = TX + 4, NPH = TY + 2, NPS = NPW * NPH;   // nut plane: x -2 .. 65, y -1 .. 8
    static constexpr int NPAIR = NPW / 2;                // nut pairs per row
    static constexpr size_t PLANES_BYTES = (size_t)NS * 4 * PSZA * sizeof(float);
    static constexpr size_t NUT_BYTES = SGS ? (((size_t)3 * NPS * sizeof(float) + 127) / 128) * 128 : 0;
    static constexpr size_t BAR_BYTES = 128;
    static constexpr int KCH = 32, NLT = KCH + 2 * AEO_LH;
    static constexpr size_t SMEM = PLANES_BYTES + NUT_BYTES + BAR_BYTES + (size_t)LV_N * NLT * sizeof(float) + 128;
    // the AMD closure's kappa_t planes (the nut planes' layout) after the rest
    static constexpr size_t KT_BYTE = ((SMEM - 128 + 127) / 128) * 128;
    static constexpr int KT_OFS = (int)((KT_BYTE - PLANES_BYTES) / sizeof(float));   // elements past nutp
    static constexpr size_t SMEM_AMD = KT_BYTE + NUT_BYTES + 128;
    static_assert(NS * 8 <= (int)BAR_BYTES, "mbarrier block");
    static_assert(TXT == 32 && NPAIR == TXT + 2, "the eddy-viscosity loop maps warps to 32-pair rows");
    static_assert(PW % 2 == 0 && PSZA % 2 == 0 && NPW % 2 == 0, "pairs stay 8-byte aligned");
};

// Pair accessor: (di, dj, dk) -> the values at x and x+1 (x = the thread's
// even cell) of level k+dk; lp[dk+ZL] points at the pair in field 0, field f
// is FOFS floats further.
template <int ZL, int PW, int FOFS>
struct PairAcc {
    const float* const* lp;
    __device__ __forceinline__ float2 ld2(int dk, int o) const {
        return *reinterpret_cast<const float2*>(lp[dk + ZL] + o);
    }
    __device__ __forceinline__ F2 operator()(int di, int dj, int dk) const {
        const int o = FOFS + dj * PW + di;
        if ((di & 1) == 0) return F2(ld2(dk, o));
        const float2 lo = ld2(dk, o - 1), hi = ld2(dk, o + 1);
        return F2(lo.y, hi.x);
    }
};

template <int NPW>
struct PairNut {
    const float* p[3];   // levels k-1, k, k+1 at the thread's pair
    __device__ __forceinline__ float2 ld2(int dk, int o) const { return *reinterpret_cast<const float2*>(p[dk + 1] + o); }
    __device__ __forceinline__ F2 operator()(int di, int dj, int dk) const {
        const int o = dj * NPW + di;
        if ((di & 1) == 0) return F2(ld2(dk, o));
        const float2 lo = ld2(dk, o - 1), hi = ld2(dk, o + 1);
        return F2(lo.y, hi.x);
    }
    __device__ __forceinline__ PairNut shifted(int o) const { return PairNut{{p[0] + o, p[1] + o, p[2] + o}}; }
};

template <bool SGS, bool ANEL, bool UNI, int CLOS = 0>   // CLOS: as in sweep_tile_kernel
__global__ void __launch_bounds__(256, 2) sweep_pair_kernel(const __grid_constant__ TileMaps maps, SweepArgs<float> a,
                                                            int kchunk, int* err) {
    using S = PairShape<SGS>;
    using R = float;
    extern __shared__ __align__(128) unsigned char smem_tile[];
    unsigned char* sbase = smem_tile + ((128u - (smem_u32(smem_tile) & 127u)) & 127u);
    float* planes = reinterpret_cast<float*>(sbase);
    float* nutp = reinterpret_cast<float*>(sbase + S::PLANES_BYTES);
    uint64_t* bars = reinterpret_cast<uint64_t*>(sbase + S::PLANES_BYTES + S::NUT_BYTES);
    float* lvs = reinterpret_cast<float*>(sbase + S::PLANES_BYTES + S::NUT_BYTES + S::BAR_BYTES);

    const Geo& g = a.g;
    const int tx = threadIdx.x, ty = threadIdx.y, tid = tx + S::TXT * ty;
    const int i0 = blockIdx.x * S::TX, j0 = blockIdx.y * S::TY;
    const int kbeg = blockIdx.z * kchunk;
    const int kend = min(g.nz, kbeg + kchunk);
    const int i = i0 + 2 * tx, j = j0 + ty;
    const bool active = i < g.nx && j < g.ny;   // nx is even: the pair is whole
    const int Lfirst = kbeg - S::ZL;
    const int Llast = kend - 1 + S::ZH;
    const uint32_t bytes = 4u * S::PSZ * sizeof(float);

    auto slot_of = [&](int L) { return (L - Lfirst) % S::NS; };
    auto parity_of = [&](int L) { return (uint32_t)(((L - Lfirst) / S::NS) & 1); };
    auto plane = [&](int L) { return planes + (size_t)slot_of(L) * 4 * S::PSZA; };
    auto issue = [&](int L) {
        uint64_t* b = bars + slot_of(L);
        mbar_expect_tx(b, bytes);
        const int x = i0 + AEO_HX - 4, y = j0 + AEO_H - S::HH, z = L + AEO_H;
        float* d = plane(L);
        tma_load_3d(d, &maps.u, b, x, y, z);
        tma_load_3d(d + S::PSZA, &maps.v, b, x, y, z);
        tma_load_3d(d + 2 * S::PSZA, &maps.w, b, x, y, z);
        tma_load_3d(d + 3 * S::PSZA, &maps.t, b, x, y, z);
    };

    if (tid == 0) {
        for (int s = 0; s < S::NS; ++s) mbar_init(bars + s, 1);
        fence_mbar_init();
    }
    const int nlt = kend - kbeg + 2 * AEO_LH;
    {
        const float* src = static_cast<const float*>(g.lvr);
        for (int e = tid; e < LV_N * S::NLT; e += S::NT) {
            const int f = e / S::NLT, kk = e - f * S::NLT;
            if (kk < nlt) lvs[e] = src[(size_t)f * g.lvn + kbeg + kk];
        }
    }
    __syncthreads();
    const Met<R, UNI> m(g, lvs, S::NLT, AEO_LH - kbeg);
    int Lissued = min(Llast, kbeg + S::ZH + 1);
    if (tid == 0)
        for (int L = Lfirst; L <= Lissued; ++L) issue(L);

    const R dt = R(__ldg(a.dtp));
    const int vbase = (ty + S::HH) * S::PW + 4 + 2 * tx;
    bool failed = false;
    for (int k = kbeg; k < kend; ++k) {
        const int Lw0 = (k == kbeg) ? Lfirst : k + S::ZH;
        bool ok = true;
        if (tid < 32)
            for (int L = Lw0; L <= k + S::ZH; ++L) ok = ok && mbar_wait_bounded(bars + slot_of(L), parity_of(L));
        if (__syncthreads_or(!ok)) { failed = true; break; }
        // every thread is past level k-1: the slot of level k-1-ZL takes level k+ZH+1
        if (k > kbeg) {
            const int Ln = k + S::ZH + 1;
            if (Ln <= Llast) {
                if (tid == 0) issue(Ln);
                Lissued = Ln;
            }
        }

        const float* lp[S::NW];
#pragma unroll
        for (int d = 0; d < S::NW; ++d) lp[d] = plane(k - S::ZL + d) + vbase;
        const PairAcc<S::ZL, S::PW, 0> U{lp};
        const PairAcc<S::ZL, S::PW, S::PSZA> V{lp};
        const PairAcc<S::ZL, S::PW, 2 * S::PSZA> W{lp};
        const PairAcc<S::ZL, S::PW, 3 * S::PSZA> T{lp};

        PairNut<S::NPW> N;
        if (SGS) {
            const int Lz0 = (k == kbeg) ? k - 1 : k + 1;
            bool mirror = false;
            for (int L = Lz0; L <= k + 1; ++L) {
                if (g.bc_z == 1 && (L < 0 || L >= g.nz)) { mirror = true; continue; }
                float* np = nutp + (size_t)((L + 3) % 3) * S::NPS;
                const float* sp[3];
#pragma unroll
                for (int d = 0; d < 3; ++d) sp[d] = plane(L - 1 + d);
                // warps take rows of the 32 interior pairs, the two edge pairs come last
                for (int e = tid; e < S::NPAIR * S::NPH; e += S::NT) {
                    int cj, pc;
                    if (e < S::TXT * S::NPH) { cj = e >> 5; pc = (e & 31) + 1; }
                    else { const int x = e - S::TXT * S::NPH; cj = x >> 1; pc = (x & 1) ? S::NPAIR - 1 : 0; }
                    // the pair's first cell sits at tile x = 2 pc - 2, plane x = 2 pc + 2
                    const int b = (cj - 1 + S::HH) * S::PW + 2 * pc + 2;
                    const float* q[3] = {sp[0] + b, sp[1] + b, sp[2] + b};
                    const PairAcc<1, S::PW, 0> Uq{q};
                    const PairAcc<1, S::PW, S::PSZA> Vq{q};
                    const PairAcc<1, S::PW, 2 * S::PSZA> Wq{q};
                    if constexpr (CLOS == 2) {
                        const F2 c = F2(float(dyn_cs2_at(g, a.cs2, L) * a.dyn_d2));
                        const F2 nv = c * strain_at<R, UNI>(m, g, L, Uq, Vq, Wq, (F2*)nullptr);
                        *reinterpret_cast<float2*>(np + cj * S::NPW + 2 * pc) = nv.v;
                    } else if constexpr (CLOS == 1) {
                        const PairAcc<1, S::PW, 3 * S::PSZA> Tq{q};
                        const NuKappa<F2> nk = amd_point<R, UNI>(m, g, L, R(a.c_s), a.sgs_bg, a.pr_t, Uq, Vq, Wq, Tq);
                        *reinterpret_cast<float2*>(np + cj * S::NPW + 2 * pc) = nk.nu.v;
                        *reinterpret_cast<float2*>(np + cj * S::NPW + 2 * pc + S::KT_OFS) = nk.ka.v;
                    } else {
                        const F2 nv = smag_point<R, UNI>(m, g, L, R(a.c_s), Uq, Vq, Wq);
                        *reinterpret_cast<float2*>(np + cj * S::NPW + 2 * pc) = nv.v;
                    }
                }
            }
            __syncthreads();
            if (mirror) {
                for (int L = Lz0; L <= k + 1; ++L) {
                    if (!(g.bc_z == 1 && (L < 0 || L >= g.nz))) continue;
                    const int Ls = L < 0 ? -L - 1 : 2 * g.nz - 1 - L;
                    float* dst = nutp + (size_t)((L + 3) % 3) * S::NPS;
                    const float* src = nutp + (size_t)((Ls + 3) % 3) * S::NPS;
                    for (int e = tid; e < S::NPS; e += S::NT) dst[e] = src[e];
                    if (CLOS == 1)
                        for (int e = tid; e < S::NPS; e += S::NT) dst[e + S::KT_OFS] = src[e + S::KT_OFS];
                }
                __syncthreads();
            }
            // the thread's pair: nut row ty + 1, column 2 tx + 2
            const int nb = (ty + 1) * S::NPW + 2 * tx + 2;
#pragma unroll
            for (int d = 0; d < 3; ++d) N.p[d] = nutp + (size_t)((k - 1 + d + 3) % 3) * S::NPS + nb;
        } else {
            N.p[0] = N.p[1] = N.p[2] = nutp;
        }

        if (active) {
            F2 tu, tv, tw, tt;
            sweep_point<R, 0, SGS, ANEL, UNI, false, CLOS == 1>(m, a, g, k, U, V, W, T, N, tu, tv, tw, tt);
            const long long qi = iidx(g, i, j, k), q = pidx(g, i, j, k);
            const F2 fdt(dt);
            *reinterpret_cast<float2*>(a.us + qi) = (U(0, 0, 0) + fdt * tu).v;
            *reinterpret_cast<float2*>(a.vs + qi) = (V(0, 0, 0) + fdt * tv).v;
            *reinterpret_cast<float2*>(a.ws + qi) =
                (g.bc_z == 1 && k == 0) ? make_float2(0.f, 0.f) : (W(0, 0, 0) + fdt * tw).v;
            F2 tn = T(0, 0, 0) + fdt * tt;
            if (a.stage) tn = rk_combine(a.ca, a.cb, F2(*reinterpret_cast<const float2*>(a.th0 + q)), tn);
            *reinterpret_cast<float2*>(a.th_out + q) = tn.v;
        }
    }
    if (failed) {
        if (tid == 0) atomicOr(err, AEO_ERR_FLAG_TMA);
        for (int L = max(Lfirst, Lissued - S::NS + 1); L <= Lissued; ++L) mbar_wait_bounded(bars + slot_of(L), parity_of(L));
    }
}
