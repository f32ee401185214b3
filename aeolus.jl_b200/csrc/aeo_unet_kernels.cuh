// aeo_unet_kernels.cuh -- kernels of the learned U-Net preconditioner
// (included by aeo_unet.cu).
//
// Tensors are channels-last bfloat16 arrays (cell-major, C channels of a
// cell contiguous, cell = x + nx (y + ny z)); the grid is periodic in x and
// y and zero outside z.  A 3x3x3 convolution is an implicit GEMM on the
// tcgen05 tensor cores: M = 128 output cells, N = C_out, K = 27 taps x C_in,
// BF16 operands from shared memory, the FP32 accumulator in TMEM.
//
// Tiles of 128 cells: mode 0 takes a 128-cell x segment of one row
// (nx % 128 == 0); mode 1 takes 128 / nx whole rows (128 % nx == 0).  The
// input tile with its one-cell halo is staged once in shared memory as
// K-major planes of 16-byte rows (8 channels of one cell), so that the A
// operand of every tap is the same canonical layout at another start
// address: mode 0 keeps a halo-ed row per (dz, dy) and shifts by dx within
// it; mode 1 keeps, per (dz, dx), rows rotated by dx (periodic) and stacked,
// so that a dy shift is a whole-row offset.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "aeo_tc.cuh"

namespace un {

constexpr int TM = 128;                 // cells per tile (the MMA M)
constexpr int CONV_THREADS = 128;
constexpr uint32_t WAIT_LIMIT = 1u << 26;   // mbarrier polls before a kernel gives up

typedef __nv_bfloat16 bf16;

struct Tiles {
    int nx, ny, nz;
    int mode, rows, tx, ntiles;
    int np, pitch;                      // staged planes per 8-channel chunk, 16-byte rows per plane
};

inline Tiles make_tiles(int nx, int ny, int nz) {
    Tiles T{};
    T.nx = nx; T.ny = ny; T.nz = nz;
    if (nx % TM == 0) {
        T.mode = 0; T.rows = 1; T.tx = nx / TM; T.ntiles = T.tx * ny * nz;
        T.np = 9; T.pitch = TM + 2;
    } else {
        T.mode = 1; T.rows = TM / nx; T.tx = ny / T.rows; T.ntiles = T.tx * nz;
        T.np = 9 * (T.rows + 2); T.pitch = nx;
    }
    return T;
}

__device__ __forceinline__ void tile_origin(const Tiles& T, int tile, int& x0, int& j0, int& k) {
    if (T.mode == 0) {
        const int xt = tile % T.tx, rest = tile / T.tx;
        x0 = xt * TM; j0 = rest % T.ny; k = rest / T.ny;
    } else {
        x0 = 0; j0 = (tile % T.tx) * T.rows; k = tile / T.tx;
    }
}

// cell of tile row m
__device__ __forceinline__ int cell_of(const Tiles& T, int x0, int j0, int k, int m) {
    if (T.mode == 0) return (k * T.ny + j0) * T.nx + x0 + m;
    return (k * T.ny + j0 + m / T.nx) * T.nx + m % T.nx;
}

// staged plane and first cell of tap t = (dz+1)*9 + (dy+1)*3 + (dx+1)
__device__ __forceinline__ void tap_plane(const Tiles& T, int t, int& P, int& xs) {
    const int dz = t / 9 - 1, dy = (t / 3) % 3 - 1, dx = t % 3 - 1;
    if (T.mode == 0) { P = (dz + 1) * 3 + (dy + 1); xs = 1 + dx; }
    else { P = ((dz + 1) * 3 + (dx + 1)) * (T.rows + 2) + 1 + dy; xs = 0; }
}

__device__ __forceinline__ void cp_async16(void* dst, const void* src, bool valid) {
    const uint32_t d = tc::smem_u32(dst);
    const int n = valid ? 16 : 0;                 // 0: zero-fill the 16 bytes
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" :: "r"(d), "l"(src), "r"(n) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" :: "n"(N) : "memory"); }

// The input tile with its halo into shared memory, row (c, P, x) at
// ((c * np + P) * pitch + x) * 16 bytes: one warp per run of a plane (a
// halo-ed row segment in mode 0, a dx-rotated row in mode 1), lanes along
// x; asynchronous 16-byte copies (cp.async), zero-filled outside z.
template <int CIN>
__device__ __forceinline__ void stage_input(const Tiles& T, const uint4* __restrict__ in, uint4* sA, int x0, int j0,
                                            int k) {
    constexpr int NCH = CIN / 8;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarp = blockDim.x >> 5;
    for (int run = warp; run < NCH * T.np; run += nwarp) {
        const int c = run / T.np, P = run - c * T.np;
        int dz, gy, xoff;
        if (T.mode == 0) {
            dz = P / 3 - 1;
            gy = j0 + (P % 3) - 1;
            xoff = x0 - 1;
        } else {
            const int nyr = T.rows + 2, yr = P % nyr, q = P / nyr;
            dz = q / 3 - 1;
            gy = j0 - 1 + yr;
            xoff = (q % 3) - 1;
        }
        gy = gy < 0 ? gy + T.ny : (gy >= T.ny ? gy - T.ny : gy);
        const int gz = k + dz;
        const bool zin = gz >= 0 && gz < T.nz;
        const uint4* row = in + ((size_t)((zin ? gz : 0) * T.ny + gy) * T.nx) * NCH + c;
        uint4* dst = sA + (size_t)run * T.pitch;
        for (int x = lane; x < T.pitch; x += 32) {
            int gx = xoff + x;
            gx = gx < 0 ? gx + T.nx : (gx >= T.nx ? gx - T.nx : gx);
            cp_async16(dst + x, row + (size_t)gx * NCH, zin);
        }
    }
}

struct ConvArgs {
    Tiles T;
    const bf16* in;        // (n, CIN)
    const uint4* wimg;     // weights in the shared-memory image [chunk][tap][co][8]
    const float* bias;     // COUT or nullptr
    const bf16* add;       // (n, COUT) added before the activation, or nullptr
    const bf16* gate;      // (n, COUT): result *= (gate > 0), or nullptr
    bf16* out;             // (n, COUT) or nullptr
    float* out0;           // channel 0 in FP32 (times out0_scale * out0_mask), or nullptr
    const float* out0_mask;
    const double* out0_scale;
    int relu;
    int dbuf;              // two staging buffers (the next tile loads while this one multiplies)
    int* err;
};

// The epilogue of one output cell: its COUT accumulators from the thread's
// TMEM lane (tacc = the accumulator's address with the lane quarter of the
// calling warp), + bias + add, ReLU, * gate, stored as BF16 and/or channel 0
// in FP32.
template <int COUT>
__device__ __forceinline__ void conv_epilogue(const ConvArgs& a, uint32_t tacc, int cell) {
    float v[COUT];
    {
        float h[16];
        tc::tmem_ld16(tacc, h);
#pragma unroll
        for (int q = 0; q < 16; ++q) v[q] = h[q];
        if constexpr (COUT == 32) {
            tc::tmem_ld16(tacc + 16u, h);
#pragma unroll
            for (int q = 0; q < 16; ++q) v[16 + q] = h[q];
        }
    }
    if (a.bias)
#pragma unroll
        for (int q = 0; q < COUT; ++q) v[q] += a.bias[q];
    if (a.add) {
        const uint4* ap = reinterpret_cast<const uint4*>(a.add + (size_t)cell * COUT);
#pragma unroll
        for (int u = 0; u < COUT / 8; ++u) {
            uint4 w = ap[u];
            const bf16* e = reinterpret_cast<const bf16*>(&w);
#pragma unroll
            for (int q = 0; q < 8; ++q) v[8 * u + q] += __bfloat162float(e[q]);
        }
    }
    if (a.relu)
#pragma unroll
        for (int q = 0; q < COUT; ++q) v[q] = fmaxf(v[q], 0.0f);
    if (a.gate) {
        const uint4* gp = reinterpret_cast<const uint4*>(a.gate + (size_t)cell * COUT);
#pragma unroll
        for (int u = 0; u < COUT / 8; ++u) {
            uint4 w = gp[u];
            const bf16* e = reinterpret_cast<const bf16*>(&w);
#pragma unroll
            for (int q = 0; q < 8; ++q)
                if (!(__bfloat162float(e[q]) > 0.0f)) v[8 * u + q] = 0.0f;
        }
    }
    if (a.out) {
        uint4* op = reinterpret_cast<uint4*>(a.out + (size_t)cell * COUT);
#pragma unroll
        for (int u = 0; u < COUT / 8; ++u) {
            uint4 w;
            bf16* e = reinterpret_cast<bf16*>(&w);
#pragma unroll
            for (int q = 0; q < 8; ++q) e[q] = __float2bfloat16_rn(v[8 * u + q]);
            op[u] = w;
        }
    }
    if (a.out0) {
        float s = a.out0_scale ? (float)*a.out0_scale : 1.0f;
        if (a.out0_mask) s *= a.out0_mask[cell];
        a.out0[cell] = v[0] * s;
    }
}

// The operands the epilogue of a cell reads from global memory (add, gate),
// loaded ahead so that their latency hides behind the wait for the MMAs.
template <int COUT>
struct EpiIn {
    uint4 add[COUT / 8];
    uint4 gate[COUT / 8];
};
template <int COUT>
__device__ __forceinline__ void epi_prefetch(const ConvArgs& a, int cell, EpiIn<COUT>& e) {
    if (a.add) {
        const uint4* ap = reinterpret_cast<const uint4*>(a.add + (size_t)cell * COUT);
#pragma unroll
        for (int u = 0; u < COUT / 8; ++u) e.add[u] = ap[u];
    }
    if (a.gate) {
        const uint4* gp = reinterpret_cast<const uint4*>(a.gate + (size_t)cell * COUT);
#pragma unroll
        for (int u = 0; u < COUT / 8; ++u) e.gate[u] = gp[u];
    }
}
// conv_epilogue with the prefetched operands
template <int COUT>
__device__ __forceinline__ void conv_epilogue_pre(const ConvArgs& a, uint32_t tacc, int cell, const EpiIn<COUT>& e) {
    float v[COUT];
    {
        float h[16];
        tc::tmem_ld16(tacc, h);
#pragma unroll
        for (int q = 0; q < 16; ++q) v[q] = h[q];
        if constexpr (COUT == 32) {
            tc::tmem_ld16(tacc + 16u, h);
#pragma unroll
            for (int q = 0; q < 16; ++q) v[16 + q] = h[q];
        }
    }
    if (a.bias)
#pragma unroll
        for (int q = 0; q < COUT; ++q) v[q] += a.bias[q];
    if (a.add)
#pragma unroll
        for (int u = 0; u < COUT / 8; ++u) {
            const bf16* x = reinterpret_cast<const bf16*>(&e.add[u]);
#pragma unroll
            for (int q = 0; q < 8; ++q) v[8 * u + q] += __bfloat162float(x[q]);
        }
    if (a.relu)
#pragma unroll
        for (int q = 0; q < COUT; ++q) v[q] = fmaxf(v[q], 0.0f);
    if (a.gate)
#pragma unroll
        for (int u = 0; u < COUT / 8; ++u) {
            const bf16* x = reinterpret_cast<const bf16*>(&e.gate[u]);
#pragma unroll
            for (int q = 0; q < 8; ++q)
                if (!(__bfloat162float(x[q]) > 0.0f)) v[8 * u + q] = 0.0f;
        }
    if (a.out) {
        uint4* op = reinterpret_cast<uint4*>(a.out + (size_t)cell * COUT);
#pragma unroll
        for (int u = 0; u < COUT / 8; ++u) {
            uint4 w;
            bf16* x = reinterpret_cast<bf16*>(&w);
#pragma unroll
            for (int q = 0; q < 8; ++q) x[q] = __float2bfloat16_rn(v[8 * u + q]);
            op[u] = w;
        }
    }
    if (a.out0) {
        float sc = a.out0_scale ? (float)*a.out0_scale : 1.0f;
        if (a.out0_mask) sc *= a.out0_mask[cell];
        a.out0[cell] = v[0] * sc;
    }
}

template <int CIN, int COUT>
constexpr size_t conv_smem_weights() { return (size_t)(CIN / 8) * 27 * COUT * 16; }

// out = act(conv(in) + bias + add) * gate, per the flags.
template <int CIN, int COUT>
__global__ void __launch_bounds__(CONV_THREADS) conv_fwd_kernel(ConvArgs a) {
    static_assert(CIN % 16 == 0 && (COUT == 16 || COUT == 32), "CIN multiple of 16, COUT 16 or 32");
    extern __shared__ __align__(128) unsigned char smem[];
    constexpr int NCH = CIN / 8;
    constexpr int WROWS = NCH * 27 * COUT;
    __shared__ uint64_t mbar;
    __shared__ uint32_t tslot;
    const Tiles& T = a.T;
    uint4* sB = reinterpret_cast<uint4*>(smem);
    uint4* sAbuf[2];
    sAbuf[0] = sB + WROWS;
    sAbuf[1] = a.dbuf ? sAbuf[0] + (size_t)NCH * T.np * T.pitch : sAbuf[0];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int i = threadIdx.x; i < WROWS; i += blockDim.x) sB[i] = a.wimg[i];
    if (threadIdx.x == 0) tc::mbar_init(&mbar, 1);
    if (warp == 0) tc::tmem_alloc(&tslot, 32);
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    const uint32_t tmem = tslot;
    const uint32_t idesc = tc::idesc_bf16(COUT, false, false);
    const uint32_t lboA = (uint32_t)(T.np * T.pitch * 16), lboB = 27u * COUT * 16u;
    const uint32_t bBase = tc::smem_u32(sB);
    uint32_t phase = 0;
    bool failed = false;
    const uint4* inp = reinterpret_cast<const uint4*>(a.in);
    int it = 0;
    if (blockIdx.x < T.ntiles) {
        int x0, j0, k;
        tile_origin(T, blockIdx.x, x0, j0, k);
        stage_input<CIN>(T, inp, sAbuf[0], x0, j0, k);
    }
    cp_async_commit();
    for (int tile = blockIdx.x; tile < T.ntiles; tile += gridDim.x, ++it) {
        int x0, j0, k;
        tile_origin(T, tile, x0, j0, k);
        uint4* sA = sAbuf[it & 1];
        const uint32_t aBase = tc::smem_u32(sA);
        const int nxt = tile + gridDim.x;
        if (a.dbuf && nxt < T.ntiles) {
            int x1, j1, k1;
            tile_origin(T, nxt, x1, j1, k1);
            stage_input<CIN>(T, inp, sAbuf[(it + 1) & 1], x1, j1, k1);
            cp_async_commit();
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        tc::fence_async_smem();
        tc::fence_before();
        __syncthreads();
        if (threadIdx.x == 0) {
            tc::fence_after();
#pragma unroll 1
            for (int t = 0; t < 27; ++t) {
                int P, xs;
                tap_plane(T, t, P, xs);
#pragma unroll
                for (int ks = 0; ks < CIN / 16; ++ks) {
                    const uint32_t aa = aBase + (uint32_t)(((2 * ks * T.np + P) * T.pitch + xs) * 16);
                    const uint32_t bb = bBase + (uint32_t)((2 * ks * 27 + t) * COUT * 16);
                    tc::mma_bf16(tmem, tc::sdesc(aa, lboA, 128), tc::sdesc(bb, lboB, 128), idesc,
                                 (t | ks) ? 1u : 0u);
                }
            }
            tc::commit(&mbar);
        }
        const bool ok = tc::mbar_wait(&mbar, phase, WAIT_LIMIT);
        phase ^= 1u;
        if (__syncthreads_or(!ok)) {
            failed = true;
            break;
        }
        tc::fence_after();
        // epilogue: warp w holds tile rows 32w..32w+31 in its TMEM lane quarter
        conv_epilogue<COUT>(a, tmem + ((uint32_t)(warp * 32) << 16), cell_of(T, x0, j0, k, warp * 32 + lane));
        tc::fence_before();
        __syncthreads();
        if (!a.dbuf && nxt < T.ntiles) {
            int x1, j1, k1;
            tile_origin(T, nxt, x1, j1, k1);
            stage_input<CIN>(T, inp, sAbuf[0], x1, j1, k1);
            cp_async_commit();
        }
    }
    cp_async_wait<0>();
    if (failed) {
        if (threadIdx.x == 0) atomicExch(a.err, 1);
        tc::mbar_wait(&mbar, phase ^ 1u, WAIT_LIMIT);   // the outstanding MMAs, bounded
    }
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, 32);
}

// ---------------------------------------------------------------- ring kernel
//
// The forward convolution of x-segment tiles (nx a multiple of 128) as a
// pipeline.  A CTA takes a contiguous range of tiles ordered y fastest
// (tile = (k * tx + xt) * ny + j), so consecutive tiles share two of their
// three y rows: the staged input is a ring of R "entries", an entry being
// one y row of the column's three z planes (dz = -1, 0, +1) with its x halo,
// K-major 16-byte rows (8 channels of a cell) as in stage_input.  A tile
// pushes one entry (row j + 1), or three at the start of a column; tile i's
// rows are the entries q_i - 2, q_i - 1, q_i (q_i the stream index of its
// last entry), held in slots q mod R.  While the tensor core runs the 27
// taps of tile i into one of two TMEM accumulators, the CTA drains tile
// i - 1 from the other and loads the entries of tile i + PF.  An entry
// overwrites the slot of stream index q - R; with at most one column start
// among PF consecutive tiles (ny >= PF + 1), q_{i+PF} - q_i <= PF + 2, so
// R = PF + 5 keeps every slot that tile i reads intact, and tile i - 1's
// slots are reused only after its MMAs completed.
template <int CIN, int COUT, int PF>
struct RingShape {
    static constexpr int NCH = CIN / 8;
    static constexpr int R = PF + 5;
    static constexpr int PITCH = TM + 2;
    static constexpr size_t slot_rows = (size_t)3 * NCH * PITCH;          // 16-byte rows per entry
    static constexpr size_t smem = conv_smem_weights<CIN, COUT>() + (size_t)R * slot_rows * 16;
    static constexpr uint32_t tmem_cols = 2 * COUT < 32 ? 32u : (uint32_t)(2 * COUT);
};

// one entry: row jj of the column (k, x0) for dz = -1, 0, +1, every chunk,
// cells x0 - 1 .. x0 + 128 (periodic in x), zero outside z; consecutive
// threads copy consecutive 16 bytes of the source row
template <int CIN, int COUT, int PF>
__device__ __forceinline__ void ring_load_entry(const Tiles& T, const uint4* __restrict__ in, uint4* sR, int slot,
                                                int k, int x0, int jj) {
    using RS = RingShape<CIN, COUT, PF>;
    constexpr int NCH = RS::NCH, PITCH = RS::PITCH, R = RS::R;
    constexpr int TOTAL = 3 * NCH * PITCH;
    for (int idx = threadIdx.x; idx < TOTAL; idx += blockDim.x) {
        const int c = idx % NCH, rest = idx / NCH;
        const int x = rest % PITCH, d = rest / PITCH;
        const int gz = k + d - 1;
        const bool zin = gz >= 0 && gz < T.nz;
        int gx = x0 - 1 + x;
        gx = gx < 0 ? gx + T.nx : (gx >= T.nx ? gx - T.nx : gx);
        const uint4* src = in + ((size_t)((zin ? gz : 0) * T.ny + jj) * T.nx + gx) * NCH + c;
        cp_async16(sR + ((size_t)((c * R + slot) * 3 + d)) * PITCH + x, src, zin);
    }
}

// The loader / epilogue warps (0-3) and the MMA warp (4) meet only through
// mbarriers, every wait bounded: "tile i's entries landed" (rdy, by the parity
// of i, 128 arrivals) and "the accumulator of tile j is drained" (drn, by the
// parity of j, 128 arrivals) for the MMA warp; the MMA commits for warps 0-3.
// A named barrier joins warps 0-3 among themselves only.
__device__ __forceinline__ void nb_sync_n(int id, int n) { asm volatile("bar.sync %0, %1;" :: "r"(id), "r"(n) : "memory"); }

constexpr int RING_THREADS = 160;

// out = act(conv(in) + bias + add) * gate, per the flags (mode 0 tiles).
// Warps 0-3 load the ring entries and drain the accumulators (a warp reads
// its TMEM lane quarter); warp 4 issues the 27 MMAs of each tile as soon as
// its entries have landed and its accumulator is free, so the MMAs of tile i
// run while warps 0-3 drain tile i-1 and load tile i+PF.
template <int CIN, int COUT, int PF>
__global__ void __launch_bounds__(RING_THREADS) conv_ring_kernel(ConvArgs a) {
    static_assert(CIN % 16 == 0 && (COUT == 16 || COUT == 32), "CIN multiple of 16, COUT 16 or 32");
    static_assert(PF >= 1 && PF <= 4, "prefetch depth 1..4");
    using RS = RingShape<CIN, COUT, PF>;
    constexpr int NCH = RS::NCH, R = RS::R, PITCH = RS::PITCH;
    constexpr int WROWS = NCH * 27 * COUT;
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ uint64_t mbar[2], rdy[2], drn[2];
    __shared__ uint32_t tslot;
    __shared__ int mma_failed;
    const Tiles& T = a.T;
    uint4* sB = reinterpret_cast<uint4*>(smem);
    uint4* sR = sB + WROWS;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int t0 = (int)((long long)T.ntiles * blockIdx.x / gridDim.x);
    const int cnt = (int)((long long)T.ntiles * (blockIdx.x + 1) / gridDim.x) - t0;
    for (int i = threadIdx.x; i < WROWS; i += blockDim.x) sB[i] = a.wimg[i];
    if (threadIdx.x == 0) {
        tc::mbar_init(&mbar[0], 1);
        tc::mbar_init(&mbar[1], 1);
        tc::mbar_init(&rdy[0], 128);
        tc::mbar_init(&rdy[1], 128);
        tc::mbar_init(&drn[0], 128);
        tc::mbar_init(&drn[1], 128);
        mma_failed = 0;
    }
    if (warp == 0) tc::tmem_alloc(&tslot, RS::tmem_cols);
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    const uint32_t tmem = tslot;
    const uint4* inp = reinterpret_cast<const uint4*>(a.in);

    if (warp == 4) {
        // ---- the MMA warp
        const uint32_t idesc = tc::idesc_bf16(COUT, false, false);
        constexpr uint32_t lboA = (uint32_t)(R * 3 * PITCH * 16), lboB = 27u * COUT * 16u;
        const uint64_t descA = tc::sdesc(tc::smem_u32(sR), lboA, 128), descB = tc::sdesc(tc::smem_u32(sB), lboB, 128);
        int qm = -1;
#pragma unroll 1
        for (int i = 0; i < cnt; ++i) {
            const int tau = t0 + i;
            qm += (i == 0 || tau % T.ny == 0) ? 3 : 1;
            bool ok = tc::mbar_wait(&rdy[i & 1], (uint32_t)((i >> 1) & 1), WAIT_LIMIT);          // entries landed
            if (ok && i >= 2) ok = tc::mbar_wait(&drn[i & 1], (uint32_t)(((i - 2) >> 1) & 1), WAIT_LIMIT);  // i-2 drained
            if (!ok) {          // no MMAs on data that may not be there; warps 0-3 time out on the commit
                if (lane == 0) mma_failed = 1;
                __syncwarp();
                continue;
            }
            tc::fence_after();
            if (lane == 0) {
                const uint32_t dacc = tmem + (uint32_t)((i & 1) * COUT);
                int srow[3];
#pragma unroll
                for (int dy = 0; dy < 3; ++dy) srow[dy] = ((qm - 2 + dy) % R) * 3 * PITCH;
#pragma unroll
                for (int t = 0; t < 27; ++t) {
                    const int dz = t / 9, dy = (t / 3) % 3, dx = t % 3;
#pragma unroll
                    for (int ks = 0; ks < CIN / 16; ++ks) {
                        const uint64_t ad = descA + (uint64_t)(2 * ks * R * 3 * PITCH + srow[dy] + dz * PITCH + dx);
                        const uint64_t bd = descB + (uint64_t)((2 * ks * 27 + t) * COUT);
                        tc::mma_bf16(dacc, ad, bd, idesc, (t | ks) ? 1u : 0u);
                    }
                }
                tc::commit(&mbar[i & 1]);
            }
            __syncwarp();
        }
    } else {
        // ---- warps 0-3: loads and epilogues
        const int tid = threadIdx.x;                  // 0 .. 127
        int ql = -1;
        auto load_tile = [&](int iu) {
            const int tau = t0 + iu;
            const int j = tau % T.ny, col = tau / T.ny;
            const int k = col / T.tx, x0 = (col - k * T.tx) * TM;
            const bool fresh = iu == 0 || j == 0;
            for (int dy = fresh ? -1 : 1; dy <= 1; ++dy) {
                int jj = j + dy;
                jj = jj < 0 ? jj + T.ny : (jj >= T.ny ? jj - T.ny : jj);
                ++ql;
                const int slot = ql % R;
                constexpr int TOTAL = 3 * NCH * PITCH;
                for (int idx = tid; idx < TOTAL; idx += 128) {
                    const int c = idx % NCH, rest = idx / NCH;
                    const int x = rest % PITCH, d = rest / PITCH;
                    const int gz = k + d - 1;
                    const bool zin = gz >= 0 && gz < T.nz;
                    int gx = x0 - 1 + x;
                    gx = gx < 0 ? gx + T.nx : (gx >= T.nx ? gx - T.nx : gx);
                    const uint4* src = inp + ((size_t)((zin ? gz : 0) * T.ny + jj) * T.nx + gx) * NCH + c;
                    cp_async16(sR + ((size_t)((c * R + slot) * 3 + d)) * PITCH + x, src, zin);
                }
            }
        };
#pragma unroll 1
        for (int iu = 0; iu < PF; ++iu) {
            if (iu < cnt) load_tile(iu);
            cp_async_commit();
        }
        bool failed = false;
        auto drain = [&](int ip) {
            const int tp = t0 + ip, jp = tp % T.ny, colp = tp / T.ny;
            const int kp = colp / T.tx, x0p = (colp - kp * T.tx) * TM;
            const int cell = (kp * T.ny + jp) * T.nx + x0p + warp * 32 + lane;
            EpiIn<COUT> ein;
            epi_prefetch<COUT>(a, cell, ein);
            const bool ok = !failed && tc::mbar_wait(&mbar[ip & 1], (uint32_t)((ip >> 1) & 1), WAIT_LIMIT);
            if (!ok) {
                failed = true;
            } else {
                tc::fence_after();
                conv_epilogue_pre<COUT>(a, tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)((ip & 1) * COUT), cell,
                                        ein);
            }
            tc::fence_before();
            if (ip + 2 <= cnt - 1) tc::mbar_arrive(&drn[ip & 1]);   // the MMA warp reuses this accumulator for tile ip+2
        };
#pragma unroll 1
        for (int i = 0; i < cnt; ++i) {
            cp_async_wait<PF - 1>();                  // tile i's entries (the group committed PF groups ago)
            tc::fence_async_smem();
            tc::mbar_arrive(&rdy[i & 1]);
            if (i > 0) drain(i - 1);                  // its MMAs done: tile i-1's ring slots are free too
            if (i + PF < cnt && !failed) load_tile(i + PF);
            cp_async_commit();
        }
        if (cnt > 0) drain(cnt - 1);
        cp_async_wait<0>();
        if (failed) {
            if (lane == 0) atomicExch(a.err, 1);
            // the MMAs still in flight, bounded
            for (int u = cnt - 2 < 0 ? 0 : cnt - 2; u < cnt; ++u) tc::mbar_wait(&mbar[u & 1], (uint32_t)((u >> 1) & 1), WAIT_LIMIT);
        }
    }
    tc::fence_before();
    __syncthreads();
    if (threadIdx.x == 0 && mma_failed) atomicExch(a.err, 1);
    if (warp == 0) tc::tmem_dealloc(tmem, RS::tmem_cols);
}

struct WgradArgs {
    Tiles T;
    const bf16* x;         // (n, CIN) layer input
    const bf16* g;         // (n, COUT) gradient of the layer's pre-activation
    float* dW;             // [27][COUT][CIN], accumulated
    float* db;             // [COUT], accumulated
    int* err;
};

template <int CIN> constexpr int wg_mtiles() { return (27 * (CIN / 8) + 15) / 16; }
template <int CIN, int COUT> constexpr uint32_t wg_tmem_cols() {
    return wg_mtiles<CIN>() * COUT <= 32 ? 32u : wg_mtiles<CIN>() * COUT <= 64 ? 64u
         : wg_mtiles<CIN>() * COUT <= 128 ? 128u : 256u;
}

// dW[t][co][ci] += sum over cells of x[nbr_t(cell), ci] g[cell, co] and
// db[co] += sum g[cell, co]: per tile a GEMM D[(t, ci) x co] over K = the
// tile's 128 cells, both operands MN-major, the (t, ci) rows in M-tiles of
// 16 eight-channel planes materialised from the staged input.  Each CTA
// accumulates over its tiles in TMEM and adds its sums to dW at the end.
template <int CIN, int COUT>
__global__ void __launch_bounds__(CONV_THREADS) conv_wgrad_kernel(WgradArgs a) {
    extern __shared__ __align__(128) unsigned char smem[];
    constexpr int NCH = CIN / 8, NCO = COUT / 8, NMT = wg_mtiles<CIN>();
    constexpr uint32_t NCOL = wg_tmem_cols<CIN, COUT>();
    __shared__ uint64_t mbar;
    __shared__ uint32_t tslot;
    const Tiles& T = a.T;
    uint4* sG = reinterpret_cast<uint4*>(smem);          // NCO planes x 128 rows
    uint4* sM = sG + NCO * TM;                           // 16 planes x 128 rows
    uint4* sA = sM + 16 * TM;                            // staged input
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) tc::mbar_init(&mbar, 1);
    if (warp == 0) tc::tmem_alloc(&tslot, NCOL);
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    const uint32_t tmem = tslot;
    const uint32_t idesc = tc::idesc_bf16(COUT, true, true);
    const uint32_t mBase = tc::smem_u32(sM), gBase = tc::smem_u32(sG);
    uint32_t phase = 0;
    bool failed = false, any = false;
    float dbacc = 0.0f;
    for (int tile = blockIdx.x; tile < T.ntiles && !failed; tile += gridDim.x) {
        int x0, j0, k;
        tile_origin(T, tile, x0, j0, k);
        stage_input<CIN>(T, reinterpret_cast<const uint4*>(a.x), sA, x0, j0, k);
        cp_async_commit();
        cp_async_wait<0>();
        for (int it = threadIdx.x; it < NCO * TM; it += blockDim.x) {
            const int c = it / TM, m = it - c * TM;
            sG[it] = reinterpret_cast<const uint4*>(a.g)[(size_t)cell_of(T, x0, j0, k, m) * NCO + c];
        }
        __syncthreads();
        if (threadIdx.x < COUT) {
            const int c = threadIdx.x / 8, e = threadIdx.x % 8;
            const bf16* gp = reinterpret_cast<const bf16*>(sG + c * TM);
            for (int m = 0; m < TM; ++m) dbacc += __bfloat162float(gp[m * 8 + e]);
        }
        for (int mt = 0; mt < NMT; ++mt) {
            for (int it = threadIdx.x; it < 16 * TM; it += blockDim.x) {
                const int gl = it / TM, m = it - gl * TM;
                const int G = mt * 16 + gl;
                uint4 v = make_uint4(0u, 0u, 0u, 0u);
                if (G < 27 * NCH) {
                    const int t = G / NCH, c = G - t * NCH;
                    int P, xs;
                    tap_plane(T, t, P, xs);
                    v = sA[(c * T.np + P) * T.pitch + xs + m];
                }
                sM[it] = v;
            }
            tc::fence_async_smem();
            tc::fence_before();
            __syncthreads();
            if (threadIdx.x == 0) {
                tc::fence_after();
#pragma unroll
                for (int kk = 0; kk < TM / 16; ++kk) {
                    const uint64_t ad = tc::sdesc(mBase + kk * 256u, 128u, (uint32_t)TM * 16u);
                    const uint64_t bd = tc::sdesc(gBase + kk * 256u, 128u, (uint32_t)TM * 16u);
                    tc::mma_bf16(tmem + (uint32_t)(mt * COUT), ad, bd, idesc, (any || kk) ? 1u : 0u);
                }
                tc::commit(&mbar);
            }
            const bool ok = tc::mbar_wait(&mbar, phase, WAIT_LIMIT);
            phase ^= 1u;
            if (__syncthreads_or(!ok)) {
                failed = true;
                break;
            }
        }
        any = true;
    }
    if (failed) {
        if (threadIdx.x == 0) atomicExch(a.err, 1);
        tc::mbar_wait(&mbar, phase ^ 1u, WAIT_LIMIT);
    } else if (any) {
        tc::fence_after();
        if (threadIdx.x < COUT) atomicAdd(&a.db[threadIdx.x], dbacc);
        const int m = warp * 32 + lane;
        for (int mt = 0; mt < NMT; ++mt) {
            float v[COUT];
            float h[16];
            tc::tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(mt * COUT), h);
#pragma unroll
            for (int q = 0; q < 16; ++q) v[q] = h[q];
            if constexpr (COUT == 32) {
                tc::tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(mt * COUT + 16), h);
#pragma unroll
                for (int q = 0; q < 16; ++q) v[16 + q] = h[q];
            }
            const int G = mt * 16 + m / 8;
            if (G < 27 * NCH) {
                const int t = G / NCH, ci = (G % NCH) * 8 + m % 8;
#pragma unroll
                for (int co = 0; co < COUT; ++co) atomicAdd(&a.dW[((size_t)t * COUT + co) * CIN + ci], v[co]);
            }
        }
    }
    tc::fence_before();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, NCOL);
}

// The weight gradient on x-segment tiles as a pipeline (CIN = 16): the input
// rows in the forward kernel's ring (PF = 1, R = 6 entries), the tile's
// output-gradient rows beside it (two buffers), and the (tap, channel) rows of
// each M-tile materialised into one of two shared buffers by warps 0-3 while
// warp 4 multiplies the other: the 8 MMAs (K = 128 cells) of M-tile q run
// while the rows of M-tile q+1 are gathered.  Named barriers 1, 2 "M buffer
// ready" (arrived at by warps 0-3, waited on by warp 4, by the parity of q),
// 5 the loader warps among themselves; the M buffers come back through the
// MMA commits (mbarriers).  Accumulated in TMEM over the CTA's tiles, added
// to dW at the end.
template <int COUT>
struct WgShape {
    static constexpr int CIN = 16, NCH = 2, NCO = COUT / 8, PF = 1;
    static constexpr int NMT = wg_mtiles<16>();
    static constexpr size_t ring_rows = (size_t)RingShape<16, COUT, 1>::R * RingShape<16, COUT, 1>::slot_rows;
    static constexpr size_t g_rows = (size_t)NCO * TM;           // one tile's gradient rows
    static constexpr size_t m_rows = (size_t)16 * TM;            // one M buffer
    static constexpr size_t smem = (ring_rows + 2 * g_rows + 2 * m_rows) * 16;
    static constexpr uint32_t tmem_cols = wg_tmem_cols<16, COUT>();
};

template <int COUT>
__global__ void __launch_bounds__(RING_THREADS) conv_wgrad_ring_kernel(WgradArgs a) {
    using W = WgShape<COUT>;
    using RS = RingShape<16, COUT, 1>;
    constexpr int NCH = W::NCH, NCO = W::NCO, NMT = W::NMT, R = RS::R, PITCH = RS::PITCH;
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ uint64_t mbM[2], rdy[2];
    __shared__ uint32_t tslot;
    __shared__ int mma_failed;
    const Tiles& T = a.T;
    uint4* sR = reinterpret_cast<uint4*>(smem);
    uint4* sG = sR + W::ring_rows;                 // 2 x NCO planes x 128 rows
    uint4* sM = sG + 2 * W::g_rows;                // 2 x 16 planes x 128 rows
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int t0 = (int)((long long)T.ntiles * blockIdx.x / gridDim.x);
    const int cnt = (int)((long long)T.ntiles * (blockIdx.x + 1) / gridDim.x) - t0;
    if (threadIdx.x == 0) {
        tc::mbar_init(&mbM[0], 1);
        tc::mbar_init(&mbM[1], 1);
        tc::mbar_init(&rdy[0], 128);
        tc::mbar_init(&rdy[1], 128);
        mma_failed = 0;
    }
    if (warp == 0) tc::tmem_alloc(&tslot, W::tmem_cols);
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    const uint32_t tmem = tslot;
    const int nq = cnt * NMT;
    bool failed = false;

    if (warp == 4) {
        // ---- the MMA warp: M-tile q of tile i = q / NMT into TMEM columns (q % NMT) * COUT
        const uint32_t idesc = tc::idesc_bf16(COUT, true, true);
#pragma unroll 1
        for (int q = 0; q < nq; ++q) {
            const int i = q / NMT, mt = q - i * NMT;
            if (!tc::mbar_wait(&rdy[q & 1], (uint32_t)((q >> 1) & 1), WAIT_LIMIT)) {
                if (lane == 0) mma_failed = 1;
                __syncwarp();
                continue;
            }
            tc::fence_after();
            if (lane == 0) {
                const uint32_t mBase = tc::smem_u32(sM + (size_t)(q & 1) * W::m_rows);
                const uint32_t gBase = tc::smem_u32(sG + (size_t)(i & 1) * W::g_rows);
#pragma unroll
                for (int kk = 0; kk < TM / 16; ++kk) {
                    const uint64_t ad = tc::sdesc(mBase + kk * 256u, 128u, (uint32_t)TM * 16u);
                    const uint64_t bd = tc::sdesc(gBase + kk * 256u, 128u, (uint32_t)TM * 16u);
                    tc::mma_bf16(tmem + (uint32_t)(mt * COUT), ad, bd, idesc, (i > 0 || kk > 0) ? 1u : 0u);
                }
                tc::commit(&mbM[q & 1]);
            }
            __syncwarp();
        }
    } else {
        // ---- warps 0-3: loads, gradient sums, the M rows
        const int tid = threadIdx.x;
        const uint4* inp = reinterpret_cast<const uint4*>(a.x);
        const uint4* gp = reinterpret_cast<const uint4*>(a.g);
        int ql = -1;
        auto load_tile = [&](int iu) {
            const int tau = t0 + iu;
            const int j = tau % T.ny, col = tau / T.ny;
            const int k = col / T.tx, x0 = (col - k * T.tx) * TM;
            const bool fresh = iu == 0 || j == 0;
            for (int dy = fresh ? -1 : 1; dy <= 1; ++dy) {
                int jj = j + dy;
                jj = jj < 0 ? jj + T.ny : (jj >= T.ny ? jj - T.ny : jj);
                ++ql;
                const int slot = ql % R;
                constexpr int TOTAL = 3 * NCH * PITCH;
                for (int idx = tid; idx < TOTAL; idx += 128) {
                    const int c = idx % NCH, rest = idx / NCH;
                    const int x = rest % PITCH, d = rest / PITCH;
                    const int gz = k + d - 1;
                    const bool zin = gz >= 0 && gz < T.nz;
                    int gx = x0 - 1 + x;
                    gx = gx < 0 ? gx + T.nx : (gx >= T.nx ? gx - T.nx : gx);
                    const uint4* src = inp + ((size_t)((zin ? gz : 0) * T.ny + jj) * T.nx + gx) * NCH + c;
                    cp_async16(sR + ((size_t)((c * R + slot) * 3 + d)) * PITCH + x, src, zin);
                }
            }
            // the tile's gradient rows, N chunk c of cell m at sG[c * 128 + m]
            uint4* dstG = sG + (size_t)(iu & 1) * W::g_rows;
            const size_t cell0 = ((size_t)k * T.ny + j) * T.nx + x0;
            for (int idx = tid; idx < NCO * TM; idx += 128) {
                const int c = idx % NCO, m = idx / NCO;
                cp_async16(dstG + (size_t)c * TM + m, gp + (cell0 + m) * NCO + c, true);
            }
        };
        if (cnt > 0) load_tile(0);
        cp_async_commit();
        float dbacc = 0.0f;
        int qm = -1;
#pragma unroll 1
        for (int i = 0; i < cnt; ++i) {
            const int tau = t0 + i;
            qm += (i == 0 || tau % T.ny == 0) ? 3 : 1;
            cp_async_wait<0>();                        // tile i's rows and gradient landed
            nb_sync_n(5, 128);                         // every loader's copies, before anyone reads them
            if (tid < COUT) {
                const int c = tid / 8, e = tid % 8;
                const bf16* g8 = reinterpret_cast<const bf16*>(sG + (size_t)(i & 1) * W::g_rows + (size_t)c * TM);
                for (int m = 0; m < TM; ++m) dbacc += __bfloat162float(g8[m * 8 + e]);
            }
#pragma unroll 1
            for (int mt = 0; mt < NMT; ++mt) {
                const int q = i * NMT + mt, b = q & 1;
                if (q >= 2)                            // the MMAs of M-tile q-2 read this buffer
                    if (!tc::mbar_wait(&mbM[b], (uint32_t)(((q - 2) >> 1) & 1), WAIT_LIMIT)) failed = true;
                // warp w gathers M chunks 4w .. 4w+3 (one (tap, channel-chunk) row each),
                // its lanes along the cells
                uint4* dM = sM + (size_t)b * W::m_rows;
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int gl = warp * 4 + u, G = mt * 16 + gl;
                    uint4* dst = dM + (size_t)gl * TM;
                    if (G < 27 * NCH) {
                        const int t = G / NCH, c = G - t * NCH;
                        const int dz = t / 9, dy = (t / 3) % 3, dx = t % 3;
                        const uint4* src = sR + ((size_t)((c * R + (qm - 2 + dy) % R) * 3 + dz)) * PITCH + dx;
#pragma unroll
                        for (int m = lane; m < TM; m += 32) dst[m] = src[m];
                    } else {
#pragma unroll
                        for (int m = lane; m < TM; m += 32) dst[m] = make_uint4(0u, 0u, 0u, 0u);
                    }
                }
                tc::fence_async_smem();
                tc::mbar_arrive(&rdy[b]);              // M-tile q ready
            }
            // every loader is done with tile i-1's ring slots and (its MMAs having
            // completed, M-tile i*NMT-1 was waited for above) its gradient rows
            nb_sync_n(5, 128);
            if (i + 1 < cnt) load_tile(i + 1);
            cp_async_commit();
        }
        cp_async_wait<0>();
        // the last two M-tiles' MMAs (the accumulators complete), bounded
        for (int q = nq - 2 < 0 ? 0 : nq - 2; q < nq; ++q)
            if (!tc::mbar_wait(&mbM[q & 1], (uint32_t)((q >> 1) & 1), WAIT_LIMIT)) failed = true;
        if (tid < COUT && cnt > 0) atomicAdd(&a.db[tid], dbacc);
        if (failed) {
            if (tid == 0) atomicExch(a.err, 1);
        } else if (cnt > 0) {
            tc::fence_after();
            const int m = warp * 32 + lane;
            for (int mt = 0; mt < NMT; ++mt) {
                float v[COUT];
                float h[16];
                tc::tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(mt * COUT), h);
#pragma unroll
                for (int r = 0; r < 16; ++r) v[r] = h[r];
                if constexpr (COUT == 32) {
                    tc::tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(mt * COUT + 16), h);
#pragma unroll
                    for (int r = 0; r < 16; ++r) v[16 + r] = h[r];
                }
                const int G = mt * 16 + m / 8;
                if (G < 27 * NCH) {
                    const int t = G / NCH, ci = (G % NCH) * 8 + m % 8;
#pragma unroll
                    for (int co = 0; co < COUT; ++co) atomicAdd(&a.dW[((size_t)t * COUT + co) * 16 + ci], v[co]);
                }
            }
        }
    }
    tc::fence_before();
    __syncthreads();
    if (threadIdx.x == 0 && mma_failed) atomicExch(a.err, 1);
    if (warp == 0) tc::tmem_dealloc(tmem, W::tmem_cols);
}

// ---------------------------------------------------------------- helpers

#define GS(i, n) for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < (long long)(n); \
                      i += (long long)gridDim.x * blockDim.x)

// Forward image [c][t][co][8] of W[t][co][ci] (FP32 master) in BF16; with
// `transpose` the image of the transposed, flipped convolution that maps an
// output gradient back to the input: W'[t'][ci][co] = W[26 - t'][co][ci].
__global__ void weight_image_kernel(const float* __restrict__ W, bf16* __restrict__ img, int cin, int cout,
                                    int transpose) {
    const int ci_img = transpose ? cout : cin, co_img = transpose ? cin : cout;
    const int n = 27 * ci_img * co_img;
    GS(q, n) {
        // img index: ((c * 27 + t) * co_img + o) * 8 + e, input channel i = 8c + e
        const int e = (int)(q % 8);
        long long r = q / 8;
        const int o = (int)(r % co_img);
        r /= co_img;
        const int t = (int)(r % 27);
        const int c = (int)(r / 27);
        const int i = 8 * c + e;
        float w = transpose ? W[((size_t)(26 - t) * cout + i) * cin + o] : W[((size_t)t * cout + o) * cin + i];
        img[q] = __float2bfloat16_rn(w);
    }
}

// network input: channel 0 = r * s (s = sqrt(n_fluid)/|r| from *scale), 1 = fluid mask
__global__ void input_kernel(const double* __restrict__ r, const float* __restrict__ mask, const double* scale,
                             bf16* __restrict__ x, long long n) {
    const float s = (float)*scale;
    GS(q, n) {
        uint4 w0 = make_uint4(0u, 0u, 0u, 0u), w1 = w0;
        bf16* e = reinterpret_cast<bf16*>(&w0);
        e[0] = __float2bfloat16_rn((float)r[q] * s);
        e[1] = __float2bfloat16_rn(mask[q]);
        uint4* xp = reinterpret_cast<uint4*>(x + q * 16);
        xp[0] = w0;
        xp[1] = w1;
    }
}

// coarse = mean of the 8 fine children (2x2x2 pooling), C channels
__global__ void pool_kernel(const bf16* __restrict__ f, bf16* __restrict__ c, int nx, int ny, int nz, int C) {
    const int cx = nx / 2, cy = ny / 2, cz = nz / 2;
    const long long n = (long long)cx * cy * cz * C;
    GS(q, n) {
        const int ch = (int)(q % C);
        long long cell = q / C;
        const int I = (int)(cell % cx), J = (int)((cell / cx) % cy), K = (int)(cell / ((long long)cx * cy));
        float s = 0.0f;
#pragma unroll
        for (int d = 0; d < 8; ++d) {
            const int i = 2 * I + (d & 1), j = 2 * J + ((d >> 1) & 1), k = 2 * K + (d >> 2);
            s += __bfloat162float(f[(((size_t)k * ny + j) * nx + i) * C + ch]);
        }
        c[q] = __float2bfloat16_rn(s * 0.125f);
    }
}

// fine = coarse[parent] + skip (nearest upsampling with an additive skip)
__global__ void up_add_kernel(const bf16* __restrict__ c, const bf16* __restrict__ skip, bf16* __restrict__ f, int nx,
                              int ny, int nz, int C) {
    const long long n = (long long)nx * ny * nz * C;
    GS(q, n) {
        const int ch = (int)(q % C);
        long long cell = q / C;
        const int i = (int)(cell % nx), j = (int)((cell / nx) % ny), k = (int)(cell / ((long long)nx * ny));
        const size_t p = (((size_t)(k / 2) * (ny / 2) + j / 2) * (nx / 2) + i / 2) * C + ch;
        f[q] = __float2bfloat16_rn(__bfloat162float(c[p]) + __bfloat162float(skip[q]));
    }
}

// coarse gradient of nearest upsampling (sum of the 8 children), times (act > 0)
__global__ void up_back_gate_kernel(const bf16* __restrict__ gf, const bf16* __restrict__ act, bf16* __restrict__ gc,
                                    int nx, int ny, int nz, int C) {
    const int cx = nx / 2, cy = ny / 2, cz = nz / 2;
    const long long n = (long long)cx * cy * cz * C;
    GS(q, n) {
        const int ch = (int)(q % C);
        long long cell = q / C;
        const int I = (int)(cell % cx), J = (int)((cell / cx) % cy), K = (int)(cell / ((long long)cx * cy));
        float s = 0.0f;
#pragma unroll
        for (int d = 0; d < 8; ++d) {
            const int i = 2 * I + (d & 1), j = 2 * J + ((d >> 1) & 1), k = 2 * K + (d >> 2);
            s += __bfloat162float(gf[(((size_t)k * ny + j) * nx + i) * C + ch]);
        }
        gc[q] = __bfloat162float(act[q]) > 0.0f ? __float2bfloat16_rn(s) : __float2bfloat16_rn(0.0f);
    }
}

// fine gradient = (skip gradient + pooled-coarse gradient / 8) * (act > 0)
__global__ void pool_back_add_gate_kernel(const bf16* __restrict__ gskip, const bf16* __restrict__ gc,
                                          const bf16* __restrict__ act, bf16* __restrict__ gf, int nx, int ny, int nz,
                                          int C) {
    const long long n = (long long)nx * ny * nz * C;
    GS(q, n) {
        const int ch = (int)(q % C);
        long long cell = q / C;
        const int i = (int)(cell % nx), j = (int)((cell / nx) % ny), k = (int)(cell / ((long long)nx * ny));
        const size_t p = (((size_t)(k / 2) * (ny / 2) + j / 2) * (nx / 2) + i / 2) * C + ch;
        const float v = __bfloat162float(gskip[q]) + 0.125f * __bfloat162float(gc[p]);
        gf[q] = __bfloat162float(act[q]) > 0.0f ? __float2bfloat16_rn(v) : __float2bfloat16_rn(0.0f);
    }
}

// the output-layer gradient image: channel 0 = g (FP32 field), the rest 0
__global__ void grad_out_kernel(const float* __restrict__ g, bf16* __restrict__ gimg, long long n) {
    GS(q, n) {
        uint4 w0 = make_uint4(0u, 0u, 0u, 0u), w1 = w0;
        reinterpret_cast<bf16*>(&w0)[0] = __float2bfloat16_rn(g[q]);
        uint4* p = reinterpret_cast<uint4*>(gimg + q * 16);
        p[0] = w0;
        p[1] = w1;
    }
}

// Sums over fluid cells: z in network units (z * zs, zs = *tscale), the raw
// error e, the count and e^2.  The loss compares the mean-free network
// output with the mean-free error scaled to unit RMS on the fluid: flexible
// CG is invariant to the scale of each preconditioner application, so only
// the error's shape is learned, whatever its magnitude.
__global__ void loss_sums_kernel(const float* __restrict__ z, const double* __restrict__ e, const float* __restrict__ mask,
                                 const double* tscale, double* sums, long long n) {
    double sz = 0.0, se = 0.0, sn = 0.0, see = 0.0;
    const double zs = *tscale;
    GS(q, n) {
        if (mask[q] > 0.0f) {
            sz += z[q] * zs;
            se += e[q];
            see += e[q] * e[q];
            sn += 1.0;
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        sz += __shfl_down_sync(0xffffffffu, sz, o);
        se += __shfl_down_sync(0xffffffffu, se, o);
        sn += __shfl_down_sync(0xffffffffu, sn, o);
        see += __shfl_down_sync(0xffffffffu, see, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&sums[0], sz);
        atomicAdd(&sums[1], se);
        atomicAdd(&sums[2], sn);
        atomicAdd(&sums[3], see);
    }
}

// d = (z' - mean z') - (e' - mean e') on fluid cells, z' = z tscale, e' = e
// scaled to unit RMS; loss += d^2 / n_f; g = dloss/dz' = 2 d / n_f
__global__ void loss_grad_kernel(const float* __restrict__ z, const double* __restrict__ e,
                                 const float* __restrict__ mask, const double* tscale, double* sums,
                                 float* __restrict__ g, long long n) {
    const double nf = sums[2] > 0.0 ? sums[2] : 1.0;
    const double es = sums[3] > 0.0 ? sqrt(nf / sums[3]) : 1.0;
    const double mz = sums[0] / nf, me = sums[1] * es / nf, zs = *tscale;
    double l = 0.0;
    GS(q, n) {
        float gv = 0.0f;
        if (mask[q] > 0.0f) {
            const double d = (z[q] * zs - mz) - (e[q] * es - me);
            l += d * d;
            gv = (float)(2.0 * d / nf);
        }
        g[q] = gv;
    }
    for (int o = 16; o > 0; o >>= 1) l += __shfl_down_sync(0xffffffffu, l, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(&sums[4], l / nf);
}

// Adam on the FP32 master parameters (Kingma & Ba 2015), gradients zeroed after use
__global__ void adam_kernel(float* __restrict__ p, float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                            long long n, float lr, float b1, float b2, float eps, float c1, float c2) {
    GS(q, n) {
        const float gq = g[q];
        const float mq = b1 * m[q] + (1.0f - b1) * gq;
        const float vq = b2 * v[q] + (1.0f - b2) * gq * gq;
        m[q] = mq;
        v[q] = vq;
        p[q] -= lr * (mq / c1) / (sqrtf(vq / c2) + eps);
        g[q] = 0.0f;
    }
}

// s = sqrt(n_fluid) / |r|, from a reduction of r^2 over fluid cells
__global__ void rscale_kernel(const double* __restrict__ r, const float* __restrict__ mask, double* acc, long long n) {
    double s = 0.0, c = 0.0;
    GS(q, n) {
        if (mask[q] > 0.0f) {
            s += r[q] * r[q];
            c += 1.0;
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        s += __shfl_down_sync(0xffffffffu, s, o);
        c += __shfl_down_sync(0xffffffffu, c, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&acc[0], s);
        atomicAdd(&acc[1], c);
    }
}

// scale[0] = sqrt(n_f / sum r^2) (network input scale); scale[1] = out_scale / scale[0]
// (network output -> error); scale[2] = 1 / scale[1] (error -> training target)
__global__ void rscale_final_kernel(const double* acc, double* scale, const double* out_scale) {
    const double s = acc[0] > 0.0 ? sqrt(acc[1] / acc[0]) : 1.0;
    scale[0] = s;
    scale[1] = *out_scale / s;
    scale[2] = s / *out_scale;
}

#undef GS

}  // namespace un
