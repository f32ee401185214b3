// aeo_sweep_pair.cuh -- the FP32 centred sweep on cell pairs.
//
// The tiled sweep of aeo_sweep_tile.cuh with every thread owning two
// x-adjacent cells: the same sweep_point / smag_point arithmetic runs on F2
// values (aeo_f2.cuh), so each FP32 add, multiply or fused multiply-add
// serves both cells, and a neighbour pair at an even x-offset is one 8-byte
// shared load (an odd offset takes the halves of the two aligned pairs
// around it, which its even neighbours load anyway).
//
// A tile is 64 x 8 cells (32 x 8 threads).  The kernel is persistent: it is
// launched with as many CTAs as the SMs hold (two per SM) and CTA c takes
// the c-th of that many equal contiguous ranges of the (tile, level) items,
// tile-major, so every CTA does the same number of levels (no partial last
// wave) in one or a few column segments.  In a segment the CTA marches up
// the column: the planes of u, v, w and theta (x from i0-4, 72 wide, y halo
// 2) come by TMA into a ring loaded one level ahead of what the level in
// hand reads; every thread polls the slot's mbarrier itself (bounded).  With
// an SGS closure the eddy viscosity of level k+2 is formed on cell pairs
// (tile x -2 .. 65, y -1 .. 8) in the same pass as the sweep of level k,
// into a ring of four planes, so one CTA barrier per level orders both the
// eddy-viscosity planes and the reuse of the ring slots.
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
    // levels read while level k is swept: k-1 .. k+1, and with SGS the
    // velocities k+1 .. k+3 of the eddy viscosity of level k+2
    static constexpr int ZH = SGS ? 3 : 1;
    static constexpr int NW = ZH + 2;                    // k-1 .. k+ZH
    static constexpr int NS = NW + 1;                    // one level in flight
    static constexpr int NNU = 4;                        // eddy-viscosity planes k-1 .. k+2
    static constexpr int PW = TX + 8;                    // x from i0-4: 16-byte aligned TMA start
    static constexpr int PH = TY + 2 * HH;
    static constexpr int PSZ = PW * PH;
    static constexpr int PSZA = (int)(((PSZ * sizeof(float) + 127) / 128) * 128 / sizeof(float));
    static constexpr int NPW = TX + 4, NPH = TY + 2, NPS = NPW * NPH;   // nut plane: x -2 .. 65, y -1 .. 8
    static constexpr int NPAIR = NPW / 2;                // nut pairs per row
    static constexpr size_t PLANES_BYTES = (size_t)NS * 4 * PSZA * sizeof(float);
    static constexpr size_t NUT_BYTES = SGS ? (((size_t)NNU * NPS * sizeof(float) + 127) / 128) * 128 : 0;
    static constexpr size_t BAR_BYTES = 128;
    // a column segment has at most KCH levels (the per-level factor table)
    static constexpr int KCH = 64, NLT = KCH + 2 * AEO_LH;
    static constexpr size_t SMEM = PLANES_BYTES + NUT_BYTES + BAR_BYTES + (size_t)LV_N * NLT * sizeof(float) + 128;
    // the AMD closure's kappa_t planes (the nut planes' layout) after the rest
    static constexpr size_t KT_BYTE = ((SMEM - 128 + 127) / 128) * 128;
    static constexpr int KT_OFS = (int)((KT_BYTE - PLANES_BYTES) / sizeof(float));   // elements past nutp
    static constexpr size_t SMEM_AMD = KT_BYTE + NUT_BYTES + 128;
    static constexpr int CTAS_PER_SM = 2;
    static_assert(NS * 8 <= (int)BAR_BYTES, "mbarrier block");
    static_assert(TXT == 32 && NPAIR == TXT + 2, "the eddy-viscosity loop maps warps to 32-pair rows");
    static_assert(PW % 2 == 0 && PSZA % 2 == 0 && NPW % 2 == 0, "pairs stay 8-byte aligned");
    static_assert(SMEM_AMD + 1024 <= 228 * 1024 / CTAS_PER_SM, "two CTAs an SM");
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

// The eddy viscosity (and the AMD closure's kappa_t) of level L on the nut
// plane np, from the ring planes of levels L-1, L, L+1: warps take rows of
// the 32 interior pairs, the two edge pairs of every row come last.
template <int CLOS, bool UNI, class S>
__device__ __forceinline__ void pair_nut_plane(const Met<float, UNI>& m, const SweepArgs<float>& a, const Geo& g,
                                               int L, const float* const* sp, float* np, int tid, int i0, int j0) {
    using R = float;
    for (int e = tid; e < S::NPAIR * S::NPH; e += S::NT) {
        int cj, pc;
        if (e < S::TXT * S::NPH) { cj = e >> 5; pc = (e & 31) + 1; }
        else { const int x = e - S::TXT * S::NPH; cj = x >> 1; pc = (x & 1) ? S::NPAIR - 1 : 0; }
        // the pair's first cell sits at tile x = 2 pc - 2, plane x = 2 pc + 2;
        // open faces: a pair beyond one takes the mirrored pair, reversed
        // (cells -2, -1 the values of 1, 0; nx, nx + 1 those of nx - 1, nx - 2)
        int gx = i0 + 2 * pc - 2;
        bool rev = false;
        if (g.ox && (gx < 0 || gx >= g.nx)) { gx = gx < 0 ? -2 - gx : 2 * g.nx - 2 - gx; rev = true; }
        const int gy = open_src(g.oy, j0 + cj - 1, g.ny);
        const int b = (gy - j0 + S::HH) * S::PW + (gx - i0) + 4;
        const float* q[3] = {sp[0] + b, sp[1] + b, sp[2] + b};
        const PairAcc<1, S::PW, 0> Uq{q};
        const PairAcc<1, S::PW, S::PSZA> Vq{q};
        const PairAcc<1, S::PW, 2 * S::PSZA> Wq{q};
        if constexpr (CLOS == 2) {
            // the pair's cells: global x = i0 + 2 pc - 2 (even), y = j0 + cj - 1
            const F2 c = a.cs2f ? F2(*reinterpret_cast<const float2*>(a.cs2f + pidx(g, gx, gy, L))) *
                                      F2(float(a.dyn_d2))
                                : F2(float(dyn_cs2_at(g, a.cs2, L) * a.dyn_d2));
            const F2 nv = c * strain_at<R, UNI>(m, g, L, Uq, Vq, Wq, (F2*)nullptr);
            *reinterpret_cast<float2*>(np + cj * S::NPW + 2 * pc) = rev ? make_float2(nv.v.y, nv.v.x) : nv.v;
        } else if constexpr (CLOS == 1) {
            const PairAcc<1, S::PW, 3 * S::PSZA> Tq{q};
            const NuKappa<F2> nk = amd_point<R, UNI>(m, g, L, R(a.c_s), m.lv(LV_BGC, L), a.pr_t, Uq, Vq, Wq, Tq);
            *reinterpret_cast<float2*>(np + cj * S::NPW + 2 * pc) = rev ? make_float2(nk.nu.v.y, nk.nu.v.x) : nk.nu.v;
            *reinterpret_cast<float2*>(np + cj * S::NPW + 2 * pc + S::KT_OFS) =
                rev ? make_float2(nk.ka.v.y, nk.ka.v.x) : nk.ka.v;
        } else if constexpr (CLOS == 3) {
            // the TKE closure, cell by cell: the pair's cells x = i0 + 2 pc - 2 (+1), y = j0 + cj - 1
            const PairAcc<1, S::PW, 3 * S::PSZA> Tq{q};
            const F2 lo = Tq(0, 0, -1), c = Tq(0, 0, 0), hi = Tq(0, 0, 1);
            const NuKappa<float> n0 = tke_point<float>(g, gx, gy, L, lo.v.x, c.v.x, hi.v.x);
            const NuKappa<float> n1 = tke_point<float>(g, gx + 1, gy, L, lo.v.y, c.v.y, hi.v.y);
            *reinterpret_cast<float2*>(np + cj * S::NPW + 2 * pc) = rev ? make_float2(n1.nu, n0.nu) : make_float2(n0.nu, n1.nu);
            *reinterpret_cast<float2*>(np + cj * S::NPW + 2 * pc + S::KT_OFS) =
                rev ? make_float2(n1.ka, n0.ka) : make_float2(n0.ka, n1.ka);
        } else {
            const F2 nv = smag_point<R, UNI>(m, g, L, R(a.c_s), Uq, Vq, Wq);
            *reinterpret_cast<float2*>(np + cj * S::NPW + 2 * pc) = rev ? make_float2(nv.v.y, nv.v.x) : nv.v;
        }
    }
}

template <bool SGS, bool ANEL, bool UNI, int CLOS = 0>   // CLOS: as in sweep_tile_kernel
__global__ void __launch_bounds__(256, 2) sweep_pair_kernel(const __grid_constant__ TileMaps maps, SweepArgs<float> a,
                                                            int ntx, int items, int* err) {
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
    const uint32_t bytes = 4u * S::PSZ * sizeof(float);
    const int w0 = (int)((long long)items * blockIdx.x / gridDim.x);
    const int w1 = (int)((long long)items * (blockIdx.x + 1) / gridDim.x);
    const R dt = R(__ldg(a.dtp));
    const int vbase = (ty + S::HH) * S::PW + 4 + 2 * tx;
    const int nb = (ty + 1) * S::NPW + 2 * tx + 2;    // the thread's pair on a nut plane
    auto nut_plane = [&](int L) { return nutp + (size_t)(L & (S::NNU - 1)) * S::NPS; };

    if (tid == 0) {
        for (int s = 0; s < S::NS; ++s) mbar_init(bars + s, 1);
        fence_mbar_init();
    }
    // loads issued before the segment in hand: the ring position and
    // mbarrier phase of every load follow from this count
    uint32_t seq0 = 0;
    bool failed = false;
    int Lfirst = 0;
    for (int w = w0; w < w1;) {
        const int tile = w / g.nz;
        const int kbeg = w - tile * g.nz;
        const int kend = min(min(g.nz, kbeg + S::KCH), w1 - tile * g.nz);
        w = tile * g.nz + kend;
        const int i0 = (tile % ntx) * S::TX, j0 = (tile / ntx) * S::TY;
        const int i = i0 + 2 * tx, j = j0 + ty;
        const bool active = i < g.nx && j < g.ny;   // nx is even: the pair is whole
        Lfirst = kbeg - (SGS ? 2 : 1);
        const int Llast = kend + (SGS ? 1 : 0);
        auto seq_of = [&](int L) { return seq0 + (uint32_t)(L - Lfirst); };
        auto slot_of = [&](int L) { return (int)(seq_of(L) % S::NS); };
        auto parity_of = [&](int L) { return (uint32_t)((seq_of(L) / S::NS) & 1u); };
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
        auto wait_upto = [&](int Lo, int Hi) {   // this thread waits for the planes Lo..Hi
            bool ok = true;
            for (int L = Lo; L <= Hi; ++L) ok = ok && mbar_wait_bounded(bars + slot_of(L), parity_of(L));
            return ok;
        };

        // the previous segment is done with the ring and the factor table
        __syncthreads();
        if (tid == 0)
            for (int L = Lfirst; L <= min(Llast, Lfirst + S::NS - 1); ++L) issue(L);
        int kfail = kbeg;   // the level at which a wait gave up
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

        // the planes of the first level (and with SGS the eddy viscosity of
        // levels kbeg-1 .. kbeg+1) before the first sweep
        bool ok = wait_upto(Lfirst, min(Llast, kbeg + (SGS ? 2 : 1)));
        if (SGS && ok)
            for (int L = kbeg - 1; L <= kbeg + 1; ++L) {
                if (g.bc_z == 1 && (L < 0 || L >= g.nz)) continue;
                const float* sp[3] = {plane(L - 1), plane(L), plane(L + 1)};
                pair_nut_plane<CLOS, UNI, S>(m, a, g, L, sp, nut_plane(L), tid, i0, j0);
            }
        failed = __syncthreads_or(!ok);
        if (SGS && !failed && g.bc_z == 1 && (kbeg == 0 || kbeg + 1 >= g.nz)) {
            // the wall mirrors: level -1 takes level 0, level nz takes nz-1
            for (int L = kbeg - 1; L <= kbeg + 1; ++L) {
                if (L >= 0 && L < g.nz) continue;
                const int Ls = L < 0 ? -L - 1 : 2 * g.nz - 1 - L;
                float* dst = nut_plane(L);
                const float* srcp = nut_plane(Ls);
                for (int e = tid; e < S::NPS; e += S::NT) dst[e] = srcp[e];
                if (CLOS == 1 || CLOS == 3)
                    for (int e = tid; e < S::NPS; e += S::NT) dst[e + S::KT_OFS] = srcp[e + S::KT_OFS];
            }
            __syncthreads();
        }

        for (int k = kbeg; k < kend && !failed; ++k) {
            if (k > kbeg) {
                // every thread is past level k-1: its planes and nut planes are
                // free, and the nut plane of level k+1 is visible
                if (__syncthreads_or(!ok)) { failed = true; kfail = k - 1; break; }
            }
            // the slot of level k-2 (read last by level k-1 or the prologue)
            // takes level k-2+NS
            const int Ln = k - 2 + S::NS;
            if (tid == 0 && k - 2 >= Lfirst && Ln <= Llast) issue(Ln);
            // the one new plane this level reads (the prologue waited for the rest)
            const int Lneed = k + S::ZH;
            if (Lneed <= Llast && (SGS || k > kbeg)) ok = mbar_wait_bounded(bars + slot_of(Lneed), parity_of(Lneed));

            // the step-start theta of the pair (stages 2, 3), loaded before the
            // eddy-viscosity pass so that its latency hides behind it
            float2 th0v = make_float2(0.f, 0.f);
            if (a.stage && active) th0v = *reinterpret_cast<const float2*>(a.th0 + pidx(g, i, j, k));

            if (SGS && k + 2 <= kend) {
                const int L = k + 2;
                if (g.bc_z == 1 && L >= g.nz) {
                    // the wall mirror: level nz takes level nz-1 (formed a level ago)
                    float* dst = nut_plane(L);
                    const float* srcp = nut_plane(2 * g.nz - 1 - L);
                    for (int e = tid; e < S::NPS; e += S::NT) dst[e] = srcp[e];
                    if (CLOS == 1 || CLOS == 3)
                        for (int e = tid; e < S::NPS; e += S::NT) dst[e + S::KT_OFS] = srcp[e + S::KT_OFS];
                } else if (ok) {
                    const float* sp[3] = {plane(L - 1), plane(L), plane(L + 1)};
                    pair_nut_plane<CLOS, UNI, S>(m, a, g, L, sp, nut_plane(L), tid, i0, j0);
                }
            }

            const float* lp[3] = {plane(k - 1) + vbase, plane(k) + vbase, plane(k + 1) + vbase};
            const PairAcc<1, S::PW, 0> U{lp};
            const PairAcc<1, S::PW, S::PSZA> V{lp};
            const PairAcc<1, S::PW, 2 * S::PSZA> W{lp};
            const PairAcc<1, S::PW, 3 * S::PSZA> T{lp};
            PairNut<S::NPW> N;
            if (SGS) {
#pragma unroll
                for (int d = 0; d < 3; ++d) N.p[d] = nut_plane(k - 1 + d) + nb;
            } else {
                N.p[0] = N.p[1] = N.p[2] = nutp;
            }
            if (active) {
                F2 tu, tv, tw, tt;
                sweep_point<R, 0, SGS, ANEL, UNI, false, CLOS == 1 || CLOS == 3>(m, a, g, k, U, V, W, T, N, tu, tv, tw, tt);
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
        if (!failed && __syncthreads_or(!ok)) { failed = true; kfail = kend - 1; }   // the last level's wait
        if (failed) {
            // drain the copies this segment issued by level kfail (bounded) before the CTA exits
            if (tid == 0) atomicOr(err, AEO_ERR_FLAG_TMA);
            const int Lissued = min(Llast, max(Lfirst + S::NS - 1, kfail - 2 + S::NS));
            for (int L = max(Lfirst, Lissued - S::NS + 1); L <= Lissued; ++L)
                mbar_wait_bounded(bars + slot_of(L), parity_of(L));
            break;
        }
        seq0 += (uint32_t)(Llast - Lfirst + 1);
    }
}
