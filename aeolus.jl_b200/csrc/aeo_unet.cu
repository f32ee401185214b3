// aeo_unet.cu -- the learned U-Net preconditioner: parameters, forward,
// backward (tcgen05 implicit-GEMM convolutions, tcgen05 weight gradients),
// Adam, and the C ABI of include/aeolus_b200_unet.h.
//
// Network (levels 16 / 32 / 32 channels, BF16 activations and weights, FP32
// accumulation and FP32 master weights):
//   x (r scaled to unit RMS over the fluid, the fluid mask; 16 channels)
//   e1a = relu(conv 16->16), e1 = relu(conv 16->16)           level 1
//   e2a = relu(conv(pool e1) 16->32), e2 = relu(conv 32->32)  level 2
//   e3a = relu(conv(pool e2) 32->32), e3 = relu(conv 32->32)  level 3
//   d2 = relu(conv(up e3 + e2) 32->16)                        level 2
//   d1 = relu(conv(up d2 + e1) 16->16)                        level 1
//   z  = out_scale / s * conv(d1)[channel 0] * fluid mask
// 3x3x3 convolutions periodic in x and y, zero outside z; 2x2x2 mean
// pooling; nearest upsampling.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <new>
#include <random>
#include <string>
#include <vector>

#include "../../include/aeolus_b200_unet.h"
#include "aeo_unet_kernels.cuh"

namespace {

using un::bf16;
using un::Tiles;

struct LayerDef {
    const char* name;
    int cin, cout, level;
};

const LayerDef LAYERS[] = {{"e1a", 16, 16, 0}, {"e1", 16, 16, 0},  {"e2a", 16, 32, 1},
                           {"e2", 32, 32, 1},  {"e3a", 32, 32, 2}, {"e3", 32, 32, 2},
                           {"d2", 32, 16, 1},  {"d1", 16, 16, 0},  {"out", 16, 16, 0}};
constexpr int NLAYERS = 9;
enum { L_E1A, L_E1, L_E2A, L_E2, L_E3A, L_E3, L_D2, L_D1, L_OUT };

size_t layer_params(int l) { return (size_t)27 * LAYERS[l].cin * LAYERS[l].cout + LAYERS[l].cout; }

std::string g_unet_error;

#define CK(call)                                                                         \
    do {                                                                                 \
        cudaError_t e_ = (call);                                                         \
        if (e_ != cudaSuccess) {                                                         \
            err = std::string(#call) + ": " + cudaGetErrorString(e_);                    \
            return AEO_ERR_CUDA;                                                         \
        }                                                                                \
    } while (0)

#define CKL()                                                                            \
    do {                                                                                 \
        cudaError_t e_ = cudaGetLastError();                                             \
        if (e_ != cudaSuccess) {                                                         \
            err = std::string("kernel launch: ") + cudaGetErrorString(e_);               \
            return AEO_ERR_CUDA;                                                         \
        }                                                                                \
    } while (0)

int grid_for(long long n, int tpb = 256) {
    long long b = (n + tpb - 1) / tpb;
    return (int)(b < 148 * 16 ? (b < 1 ? 1 : b) : 148 * 16);
}

constexpr size_t SMEM_CAP = 227 * 1024;

template <int CIN>
size_t stage_bytes(const Tiles& T) { return (size_t)(CIN / 8) * T.np * T.pitch * 16; }
// two staging buffers when they fit, else one
template <int CIN, int COUT>
bool fwd_dbuf(const Tiles& T) { return un::conv_smem_weights<CIN, COUT>() + 2 * stage_bytes<CIN>(T) <= SMEM_CAP; }
template <int CIN, int COUT>
size_t fwd_smem(const Tiles& T) {
    return un::conv_smem_weights<CIN, COUT>() + (fwd_dbuf<CIN, COUT>(T) ? 2 : 1) * stage_bytes<CIN>(T);
}
template <int CIN, int COUT>
size_t wg_smem(const Tiles& T) {
    return ((size_t)(COUT / 8) * un::TM + 16 * un::TM + (size_t)(CIN / 8) * T.np * T.pitch) * 16;
}

}  // namespace

struct aeo_unet {
    int nx = 0, ny = 0, nz = 0, device = 0;
    long long n[3] = {0, 0, 0};
    Tiles T[3];
    std::string err;
    cudaStream_t st = nullptr;
    int sms = 148;
    std::vector<void*> allocs;
    // parameters: one flat FP32 buffer per role, per-layer offsets
    size_t off[NLAYERS + 1];
    float *P = nullptr, *G = nullptr, *M = nullptr, *V = nullptr;
    bf16* wf[NLAYERS];                  // forward weight images
    bf16* wb[NLAYERS];                  // transposed (backward-data) weight images
    int adam_step = 0;
    // activations
    bf16 *x, *e1a, *e1, *p1, *e2a, *e2, *p2, *e3a, *e3, *u2, *d2, *u1, *d1;
    float* z = nullptr;                 // the network's output field (scaled, masked)
    float* mask = nullptr;
    double* scale = nullptr;            // [0] input scale, [1] output scale, [2] target scale, [3] out_scale
    double* acc = nullptr;              // reductions
    // gradients
    float* gz = nullptr;
    bf16 *gimg, *g_d1, *g_u1, *g_e1, *g_e1a, *g_d2, *g_u2, *g_e2, *g_e2a, *g_p1, *g_e3, *g_e3a, *g_p2;
    double* rbuf = nullptr;             // device residual / target for host-array calls
    double* ebuf = nullptr;
    int* derr = nullptr;

    template <typename T_>
    aeo_status dalloc(T_** p, size_t count) {
        void* a = nullptr;
        CK(cudaMalloc(&a, sizeof(T_) * (count ? count : 1)));
        allocs.push_back(a);
        *p = reinterpret_cast<T_*>(a);
        return AEO_OK;
    }

    ~aeo_unet() {
        if (st) cudaStreamSynchronize(st);
        for (void* a : allocs) cudaFree(a);
        if (st) cudaStreamDestroy(st);
    }

    aeo_status init(uint64_t seed) {
        CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
        for (int l = 0; l < 3; ++l) {
            const int f = 1 << l;
            T[l] = un::make_tiles(nx / f, ny / f, nz / f);
            n[l] = (long long)(nx / f) * (ny / f) * (nz / f);
        }
        off[0] = 0;
        for (int l = 0; l < NLAYERS; ++l) off[l + 1] = off[l] + layer_params(l);
        const size_t np = off[NLAYERS];
        if (aeo_status s = dalloc(&P, np)) return s;
        if (aeo_status s = dalloc(&G, np)) return s;
        if (aeo_status s = dalloc(&M, np)) return s;
        if (aeo_status s = dalloc(&V, np)) return s;
        CK(cudaMemset(G, 0, sizeof(float) * np));
        CK(cudaMemset(M, 0, sizeof(float) * np));
        CK(cudaMemset(V, 0, sizeof(float) * np));
        for (int l = 0; l < NLAYERS; ++l) {
            const size_t w = (size_t)27 * LAYERS[l].cin * LAYERS[l].cout;
            if (aeo_status s = dalloc(&wf[l], w)) return s;
            if (aeo_status s = dalloc(&wb[l], w)) return s;
        }
        // He-normal initial weights, zero biases; the padded input channels of
        // the first layer and the padded outputs of the last are zero
        std::vector<float> h(np, 0.0f);
        std::mt19937_64 rng(seed);
        std::normal_distribution<float> nd(0.0f, 1.0f);
        for (int l = 0; l < NLAYERS; ++l) {
            const int ci = LAYERS[l].cin, co = LAYERS[l].cout;
            const float sd = std::sqrt(2.0f / (27.0f * ci)) * (l == L_OUT ? 0.1f : 1.0f);
            for (int t = 0; t < 27; ++t)
                for (int o = 0; o < co; ++o)
                    for (int i = 0; i < ci; ++i) {
                        float w = nd(rng) * sd;
                        if ((l == L_E1A && i >= 2) || (l == L_OUT && o >= 1)) w = 0.0f;
                        h[off[l] + ((size_t)t * co + o) * ci + i] = w;
                    }
        }
        CK(cudaMemcpy(P, h.data(), sizeof(float) * np, cudaMemcpyHostToDevice));
        const long long n0 = n[0], n1 = n[1], n2 = n[2];
        bf16** a16_0[] = {&x, &e1a, &e1, &u1, &d1, &gimg, &g_d1, &g_u1, &g_e1, &g_e1a};
        for (bf16** p : a16_0)
            if (aeo_status s = dalloc(p, (size_t)n0 * 16)) return s;
        bf16** a16_1[] = {&p1, &d2, &g_d2, &g_p1};
        for (bf16** p : a16_1)
            if (aeo_status s = dalloc(p, (size_t)n1 * 16)) return s;
        bf16** a32_1[] = {&e2a, &e2, &u2, &g_u2, &g_e2, &g_e2a};
        for (bf16** p : a32_1)
            if (aeo_status s = dalloc(p, (size_t)n1 * 32)) return s;
        bf16** a32_2[] = {&p2, &e3a, &e3, &g_e3, &g_e3a, &g_p2};
        for (bf16** p : a32_2)
            if (aeo_status s = dalloc(p, (size_t)n2 * 32)) return s;
        if (aeo_status s = dalloc(&z, n0)) return s;
        if (aeo_status s = dalloc(&gz, n0)) return s;
        if (aeo_status s = dalloc(&mask, n0)) return s;
        if (aeo_status s = dalloc(&rbuf, n0)) return s;
        if (aeo_status s = dalloc(&ebuf, n0)) return s;
        if (aeo_status s = dalloc(&scale, 4)) return s;
        if (aeo_status s = dalloc(&acc, 10)) return s;
        if (aeo_status s = dalloc(&derr, 1)) return s;
        CK(cudaMemset(derr, 0, sizeof(int)));
        std::vector<float> ones((size_t)n0, 1.0f);
        CK(cudaMemcpy(mask, ones.data(), sizeof(float) * n0, cudaMemcpyHostToDevice));
        double sc[4] = {1.0, 1.0, 1.0, 1.0};
        CK(cudaMemcpy(scale, sc, sizeof(sc), cudaMemcpyHostToDevice));
        if (aeo_status s = set_smem_limits()) return s;
        return refresh_images();
    }

    aeo_status set_smem_limits() {
        size_t f1616 = 0, f1632 = 0, f3232 = 0, f3216 = 0, w1616 = 0, w1632 = 0, w3232 = 0, w3216 = 0;
        for (int l = 0; l < 3; ++l) {
            f1616 = std::max(f1616, fwd_smem<16, 16>(T[l]));
            f1632 = std::max(f1632, fwd_smem<16, 32>(T[l]));
            f3232 = std::max(f3232, fwd_smem<32, 32>(T[l]));
            f3216 = std::max(f3216, fwd_smem<32, 16>(T[l]));
            w1616 = std::max(w1616, wg_smem<16, 16>(T[l]));
            w1632 = std::max(w1632, wg_smem<16, 32>(T[l]));
            w3232 = std::max(w3232, wg_smem<32, 32>(T[l]));
            w3216 = std::max(w3216, wg_smem<32, 16>(T[l]));
        }
        const size_t cap = SMEM_CAP;
        for (size_t v : {f1616, f1632, f3232, f3216, w1616, w1632, w3232, w3216})
            if (v > cap) {
                err = "U-Net tile needs more shared memory than a block has";
                return AEO_ERR_ARGUMENT;
            }
        CK(cudaFuncSetAttribute(un::conv_fwd_kernel<16, 16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)f1616));
        CK(cudaFuncSetAttribute(un::conv_fwd_kernel<16, 32>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)f1632));
        CK(cudaFuncSetAttribute(un::conv_fwd_kernel<32, 32>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)f3232));
        CK(cudaFuncSetAttribute(un::conv_fwd_kernel<32, 16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)f3216));
        CK(cudaFuncSetAttribute(un::conv_ring_kernel<16, 16, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)un::RingShape<16, 16, 2>::smem));
        CK(cudaFuncSetAttribute(un::conv_ring_kernel<16, 32, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)un::RingShape<16, 32, 1>::smem));
        CK(cudaFuncSetAttribute(un::conv_ring_kernel<32, 32, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)un::RingShape<32, 32, 1>::smem));
        CK(cudaFuncSetAttribute(un::conv_ring_kernel<32, 16, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)un::RingShape<32, 16, 1>::smem));
        CK(cudaFuncSetAttribute(un::conv_wgrad_ring_kernel<16>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)un::WgShape<16>::smem));
        CK(cudaFuncSetAttribute(un::conv_wgrad_ring_kernel<32>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)un::WgShape<32>::smem));
        CK(cudaFuncSetAttribute(un::conv_wgrad_kernel<16, 16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)w1616));
        CK(cudaFuncSetAttribute(un::conv_wgrad_kernel<16, 32>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)w1632));
        CK(cudaFuncSetAttribute(un::conv_wgrad_kernel<32, 32>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)w3232));
        CK(cudaFuncSetAttribute(un::conv_wgrad_kernel<32, 16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)w3216));
        return AEO_OK;
    }

    // BF16 images of the FP32 master weights (forward and transposed)
    aeo_status refresh_images() {
        for (int l = 0; l < NLAYERS; ++l) {
            const int ci = LAYERS[l].cin, co = LAYERS[l].cout;
            const long long w = 27LL * ci * co;
            un::weight_image_kernel<<<grid_for(w), 256, 0, st>>>(P + off[l], wf[l], ci, co, 0);
            CKL();
            un::weight_image_kernel<<<grid_for(w), 256, 0, st>>>(P + off[l], wb[l], ci, co, 1);
            CKL();
        }
        return AEO_OK;
    }

    const float* bias(int l) const { return P + off[l] + (size_t)27 * LAYERS[l].cin * LAYERS[l].cout; }
    float* dW(int l) { return G + off[l]; }
    float* db(int l) { return G + off[l] + (size_t)27 * LAYERS[l].cin * LAYERS[l].cout; }

    int conv_grid(const Tiles& Tl) const {
        int g = sms * 2;
        return Tl.ntiles < g ? Tl.ntiles : g;
    }

    // the ring kernel on x-segment tiles: two CTAs an SM where the ring and
    // the weights fit twice, contiguous tile ranges of equal length
    template <int CIN, int COUT, int PF>
    void ring(const Tiles& Tl, const un::ConvArgs& a) {
        constexpr size_t sm = un::RingShape<CIN, COUT, PF>::smem;
        const int per_sm = sm <= 113 * 1024 ? 2 : 1;
        const int g = Tl.ntiles < sms * per_sm ? Tl.ntiles : sms * per_sm;
        un::conv_ring_kernel<CIN, COUT, PF><<<g, un::RING_THREADS, sm, st>>>(a);
    }

    // one convolution (forward, or transposed with the backward image)
    aeo_status conv(int l, bool transposed, const bf16* in, bf16* out, const float* b, const bf16* add,
                    const bf16* gate, int relu, float* out0 = nullptr, const float* out0_mask = nullptr,
                    const double* out0_scale = nullptr) {
        const int ci = transposed ? LAYERS[l].cout : LAYERS[l].cin;
        const int co = transposed ? LAYERS[l].cin : LAYERS[l].cout;
        const Tiles& Tl = T[LAYERS[l].level];
        un::ConvArgs a{};
        a.T = Tl;
        a.in = in;
        a.wimg = reinterpret_cast<const uint4*>(transposed ? wb[l] : wf[l]);
        a.bias = b;
        a.add = add;
        a.gate = gate;
        a.out = out;
        a.out0 = out0;
        a.out0_mask = out0_mask;
        a.out0_scale = out0_scale;
        a.relu = relu;
        a.err = derr;
        if (Tl.mode == 0 && Tl.ny >= 3) {   // x-segment tiles, ny >= prefetch + 1: the pipelined ring kernel
            if (ci == 16 && co == 16) ring<16, 16, 2>(Tl, a);
            else if (ci == 16 && co == 32) ring<16, 32, 1>(Tl, a);
            else if (ci == 32 && co == 32) ring<32, 32, 1>(Tl, a);
            else ring<32, 16, 1>(Tl, a);
            CKL();
            return AEO_OK;
        }
        if (ci == 16 && co == 16) a.dbuf = fwd_dbuf<16, 16>(Tl);
        else if (ci == 16 && co == 32) a.dbuf = fwd_dbuf<16, 32>(Tl);
        else if (ci == 32 && co == 32) a.dbuf = fwd_dbuf<32, 32>(Tl);
        else a.dbuf = fwd_dbuf<32, 16>(Tl);
        const int gsz = conv_grid(Tl);
        if (ci == 16 && co == 16) un::conv_fwd_kernel<16, 16><<<gsz, un::CONV_THREADS, fwd_smem<16, 16>(Tl), st>>>(a);
        else if (ci == 16 && co == 32) un::conv_fwd_kernel<16, 32><<<gsz, un::CONV_THREADS, fwd_smem<16, 32>(Tl), st>>>(a);
        else if (ci == 32 && co == 32) un::conv_fwd_kernel<32, 32><<<gsz, un::CONV_THREADS, fwd_smem<32, 32>(Tl), st>>>(a);
        else un::conv_fwd_kernel<32, 16><<<gsz, un::CONV_THREADS, fwd_smem<32, 16>(Tl), st>>>(a);
        CKL();
        return AEO_OK;
    }

    aeo_status wgrad(int l, const bf16* xin, const bf16* g) {
        const int ci = LAYERS[l].cin, co = LAYERS[l].cout;
        const Tiles& Tl = T[LAYERS[l].level];
        un::WgradArgs a{};
        a.T = Tl;
        a.x = xin;
        a.g = g;
        a.dW = dW(l);
        a.db = db(l);
        a.err = derr;
        if (ci == 16 && Tl.mode == 0 && Tl.ny >= 3) {   // x-segment tiles: the pipelined ring kernel, one CTA an SM
            const int g1 = Tl.ntiles < sms ? Tl.ntiles : sms;
            if (co == 16) un::conv_wgrad_ring_kernel<16><<<g1, un::RING_THREADS, un::WgShape<16>::smem, st>>>(a);
            else un::conv_wgrad_ring_kernel<32><<<g1, un::RING_THREADS, un::WgShape<32>::smem, st>>>(a);
            CKL();
            return AEO_OK;
        }
        const int gsz = conv_grid(Tl);
        if (ci == 16 && co == 16) un::conv_wgrad_kernel<16, 16><<<gsz, un::CONV_THREADS, wg_smem<16, 16>(Tl), st>>>(a);
        else if (ci == 16 && co == 32) un::conv_wgrad_kernel<16, 32><<<gsz, un::CONV_THREADS, wg_smem<16, 32>(Tl), st>>>(a);
        else if (ci == 32 && co == 32) un::conv_wgrad_kernel<32, 32><<<gsz, un::CONV_THREADS, wg_smem<32, 32>(Tl), st>>>(a);
        else un::conv_wgrad_kernel<32, 16><<<gsz, un::CONV_THREADS, wg_smem<32, 16>(Tl), st>>>(a);
        CKL();
        return AEO_OK;
    }

    // the network on the device residual r (FP64); z = the scaled, masked output
    aeo_status forward(const double* r, cudaStream_t s) {
        cudaStream_t keep = st;
        st = s;
        aeo_status q = forward_(r);
        st = keep;
        return q;
    }

    aeo_status forward_(const double* r) {
        const int nx1 = nx / 2, ny1 = ny / 2, nz1 = nz / 2;
        CK(cudaMemsetAsync(acc, 0, sizeof(double) * 2, st));
        un::rscale_kernel<<<grid_for(n[0]), 256, 0, st>>>(r, mask, acc, n[0]);
        CKL();
        un::rscale_final_kernel<<<1, 1, 0, st>>>(acc, scale, scale + 3);
        CKL();
        un::input_kernel<<<grid_for(n[0]), 256, 0, st>>>(r, mask, scale, x, n[0]);
        CKL();
        if (aeo_status q = conv(L_E1A, false, x, e1a, bias(L_E1A), nullptr, nullptr, 1)) return q;
        if (aeo_status q = conv(L_E1, false, e1a, e1, bias(L_E1), nullptr, nullptr, 1)) return q;
        un::pool_kernel<<<grid_for(n[1] * 16), 256, 0, st>>>(e1, p1, nx, ny, nz, 16);
        CKL();
        if (aeo_status q = conv(L_E2A, false, p1, e2a, bias(L_E2A), nullptr, nullptr, 1)) return q;
        if (aeo_status q = conv(L_E2, false, e2a, e2, bias(L_E2), nullptr, nullptr, 1)) return q;
        un::pool_kernel<<<grid_for(n[2] * 32), 256, 0, st>>>(e2, p2, nx1, ny1, nz1, 32);
        CKL();
        if (aeo_status q = conv(L_E3A, false, p2, e3a, bias(L_E3A), nullptr, nullptr, 1)) return q;
        if (aeo_status q = conv(L_E3, false, e3a, e3, bias(L_E3), nullptr, nullptr, 1)) return q;
        un::up_add_kernel<<<grid_for(n[1] * 32), 256, 0, st>>>(e3, e2, u2, nx1, ny1, nz1, 32);
        CKL();
        if (aeo_status q = conv(L_D2, false, u2, d2, bias(L_D2), nullptr, nullptr, 1)) return q;
        un::up_add_kernel<<<grid_for(n[0] * 16), 256, 0, st>>>(d2, e1, u1, nx, ny, nz, 16);
        CKL();
        if (aeo_status q = conv(L_D1, false, u1, d1, bias(L_D1), nullptr, nullptr, 1)) return q;
        return conv(L_OUT, false, d1, nullptr, bias(L_OUT), nullptr, nullptr, 0, z, mask, scale + 1);
    }

    // gradients of the loss against the error e (FP64 field) into G
    aeo_status backward(const double* e) {
        const int nx1 = nx / 2, ny1 = ny / 2, nz1 = nz / 2;
        CK(cudaMemsetAsync(acc + 4, 0, sizeof(double) * 5, st));
        un::loss_sums_kernel<<<grid_for(n[0]), 256, 0, st>>>(z, e, mask, scale + 2, acc + 4, n[0]);
        CKL();
        // the loss is on the network's raw output: undo the output scale in z
        un::loss_grad_kernel<<<grid_for(n[0]), 256, 0, st>>>(z, e, mask, scale + 2, acc + 4, gz, n[0]);
        CKL();
        un::grad_out_kernel<<<grid_for(n[0]), 256, 0, st>>>(gz, gimg, n[0]);
        CKL();
        if (aeo_status q = wgrad(L_OUT, d1, gimg)) return q;
        if (aeo_status q = conv(L_OUT, true, gimg, g_d1, nullptr, nullptr, d1, 0)) return q;
        if (aeo_status q = wgrad(L_D1, u1, g_d1)) return q;
        if (aeo_status q = conv(L_D1, true, g_d1, g_u1, nullptr, nullptr, nullptr, 0)) return q;
        un::up_back_gate_kernel<<<grid_for(n[1] * 16), 256, 0, st>>>(g_u1, d2, g_d2, nx, ny, nz, 16);
        CKL();
        if (aeo_status q = wgrad(L_D2, u2, g_d2)) return q;
        if (aeo_status q = conv(L_D2, true, g_d2, g_u2, nullptr, nullptr, nullptr, 0)) return q;
        un::up_back_gate_kernel<<<grid_for(n[2] * 32), 256, 0, st>>>(g_u2, e3, g_e3, nx1, ny1, nz1, 32);
        CKL();
        if (aeo_status q = wgrad(L_E3, e3a, g_e3)) return q;
        if (aeo_status q = conv(L_E3, true, g_e3, g_e3a, nullptr, nullptr, e3a, 0)) return q;
        if (aeo_status q = wgrad(L_E3A, p2, g_e3a)) return q;
        if (aeo_status q = conv(L_E3A, true, g_e3a, g_p2, nullptr, nullptr, nullptr, 0)) return q;
        un::pool_back_add_gate_kernel<<<grid_for(n[1] * 32), 256, 0, st>>>(g_u2, g_p2, e2, g_e2, nx1, ny1, nz1, 32);
        CKL();
        if (aeo_status q = wgrad(L_E2, e2a, g_e2)) return q;
        if (aeo_status q = conv(L_E2, true, g_e2, g_e2a, nullptr, nullptr, e2a, 0)) return q;
        if (aeo_status q = wgrad(L_E2A, p1, g_e2a)) return q;
        if (aeo_status q = conv(L_E2A, true, g_e2a, g_p1, nullptr, nullptr, nullptr, 0)) return q;
        un::pool_back_add_gate_kernel<<<grid_for(n[0] * 16), 256, 0, st>>>(g_u1, g_p1, e1, g_e1, nx, ny, nz, 16);
        CKL();
        if (aeo_status q = wgrad(L_E1, e1a, g_e1)) return q;
        if (aeo_status q = conv(L_E1, true, g_e1, g_e1a, nullptr, nullptr, e1a, 0)) return q;
        return wgrad(L_E1A, x, g_e1a);
    }

    aeo_status adam(double lr) {
        ++adam_step;
        const float b1 = 0.9f, b2 = 0.999f;
        const float c1 = 1.0f - std::pow(b1, (float)adam_step), c2 = 1.0f - std::pow(b2, (float)adam_step);
        const long long np = (long long)off[NLAYERS];
        un::adam_kernel<<<grid_for(np), 256, 0, st>>>(P, G, M, V, np, (float)lr, b1, b2, 1e-8f, c1, c2);
        CKL();
        return refresh_images();
    }

    aeo_status check_err() {
        int h = 0;
        CK(cudaMemcpyAsync(&h, derr, sizeof(int), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        if (h) {
            err = "a tensor-core kernel timed out waiting for its MMAs";
            return AEO_ERR_NUMERICAL;
        }
        return AEO_OK;
    }
};

extern "C" {

int64_t aeo_unet_param_count(void) {
    size_t s = 0;
    for (int l = 0; l < NLAYERS; ++l) s += layer_params(l);
    return (int64_t)s;
}

aeo_status aeo_unet_create(int32_t nx, int32_t ny, int32_t nz, uint64_t seed, int32_t device, aeo_unet** out) {
    if (!out) { g_unet_error = "out is NULL"; return AEO_ERR_ARGUMENT; }
    *out = nullptr;
    auto level_ok = [](int a) { return a >= 1 && (a % un::TM == 0 || un::TM % a == 0); };
    if (nx % 4 || ny % 4 || nz % 4 || !level_ok(nx) || !level_ok(nx / 2) || !level_ok(nx / 4) ||
        (nx / 4 < un::TM && (ny / 4) % (un::TM / (nx / 4)) != 0) ||
        (nx / 2 < un::TM && (ny / 2) % (un::TM / (nx / 2)) != 0) || (nx < un::TM && ny % (un::TM / nx) != 0)) {
        g_unet_error = "U-Net grid: nx, ny, nz multiples of 4; at every level nx a multiple or divisor of 128 "
                       "and ny a multiple of the rows a 128-cell tile spans";
        return AEO_ERR_ARGUMENT;
    }
    if ((long long)nx * ny * nz >= (1LL << 30)) { g_unet_error = "grid at or above 2^30 cells"; return AEO_ERR_ARGUMENT; }
    if (cudaSetDevice(device) != cudaSuccess) { g_unet_error = "cudaSetDevice failed"; return AEO_ERR_CUDA; }
    aeo_unet* h = new (std::nothrow) aeo_unet;
    if (!h) { g_unet_error = "out of host memory"; return AEO_ERR_CUDA; }
    h->nx = nx; h->ny = ny; h->nz = nz; h->device = device;
    if (aeo_status s = h->init(seed)) {
        g_unet_error = h->err;
        delete h;
        return s;
    }
    *out = h;
    return AEO_OK;
}

aeo_status aeo_unet_destroy(aeo_unet* h) {
    if (!h) return AEO_OK;
    cudaSetDevice(h->device);
    delete h;
    return AEO_OK;
}

#define UN_ENTER(h)                                                    \
    if (!h) return AEO_ERR_ARGUMENT;                                   \
    if (cudaSetDevice(h->device) != cudaSuccess) {                     \
        h->err = "cudaSetDevice failed";                               \
        return AEO_ERR_CUDA;                                           \
    }

aeo_status aeo_unet_set_params(aeo_unet* h, const float* p) {
    UN_ENTER(h);
    if (!p) { h->err = "params NULL"; return AEO_ERR_ARGUMENT; }
    std::string& err = h->err;
    CK(cudaMemcpyAsync(h->P, p, sizeof(float) * h->off[NLAYERS], cudaMemcpyHostToDevice, h->st));
    if (aeo_status s = h->refresh_images()) return s;
    CK(cudaStreamSynchronize(h->st));
    return AEO_OK;
}

aeo_status aeo_unet_get_params(aeo_unet* h, float* p, float* grads) {
    UN_ENTER(h);
    std::string& err = h->err;
    if (p) CK(cudaMemcpyAsync(p, h->P, sizeof(float) * h->off[NLAYERS], cudaMemcpyDeviceToHost, h->st));
    if (grads) CK(cudaMemcpyAsync(grads, h->G, sizeof(float) * h->off[NLAYERS], cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
    return AEO_OK;
}

aeo_status aeo_unet_set_mask(aeo_unet* h, const float* fluid) {
    UN_ENTER(h);
    if (!fluid) { h->err = "mask NULL"; return AEO_ERR_ARGUMENT; }
    std::string& err = h->err;
    CK(cudaMemcpyAsync(h->mask, fluid, sizeof(float) * h->n[0], cudaMemcpyHostToDevice, h->st));
    CK(cudaStreamSynchronize(h->st));
    return AEO_OK;
}

aeo_status aeo_unet_set_out_scale(aeo_unet* h, double s) {
    UN_ENTER(h);
    if (!(s > 0)) { h->err = "out_scale must be positive"; return AEO_ERR_ARGUMENT; }
    std::string& err = h->err;
    CK(cudaMemcpyAsync(h->scale + 3, &s, sizeof(double), cudaMemcpyHostToDevice, h->st));
    CK(cudaStreamSynchronize(h->st));
    return AEO_OK;
}

aeo_status aeo_unet_apply(aeo_unet* h, const double* r, double* z) {
    UN_ENTER(h);
    if (!r || !z) { h->err = "r and z must not be NULL"; return AEO_ERR_ARGUMENT; }
    std::string& err = h->err;
    CK(cudaMemcpyAsync(h->rbuf, r, sizeof(double) * h->n[0], cudaMemcpyHostToDevice, h->st));
    if (aeo_status s = h->forward_(h->rbuf)) return s;
    std::vector<float> zf((size_t)h->n[0]);
    CK(cudaMemcpyAsync(zf.data(), h->z, sizeof(float) * h->n[0], cudaMemcpyDeviceToHost, h->st));
    if (aeo_status s = h->check_err()) return s;
    for (long long q = 0; q < h->n[0]; ++q) z[q] = zf[q];
    return AEO_OK;
}

aeo_status aeo_unet_gradients(aeo_unet* h, const double* r, const double* e, double* loss) {
    UN_ENTER(h);
    if (!r || !e) { h->err = "r and e must not be NULL"; return AEO_ERR_ARGUMENT; }
    std::string& err = h->err;
    CK(cudaMemsetAsync(h->G, 0, sizeof(float) * h->off[NLAYERS], h->st));
    CK(cudaMemcpyAsync(h->rbuf, r, sizeof(double) * h->n[0], cudaMemcpyHostToDevice, h->st));
    CK(cudaMemcpyAsync(h->ebuf, e, sizeof(double) * h->n[0], cudaMemcpyHostToDevice, h->st));
    if (aeo_status s = h->forward_(h->rbuf)) return s;
    if (aeo_status s = h->backward(h->ebuf)) return s;
    double hl[5];
    CK(cudaMemcpyAsync(hl, h->acc + 4, sizeof(hl), cudaMemcpyDeviceToHost, h->st));
    if (aeo_status s = h->check_err()) return s;
    if (loss) *loss = hl[4];
    return AEO_OK;
}

aeo_status aeo_unet_train_step(aeo_unet* h, const double* r, const double* e, double lr, double* loss) {
    if (aeo_status s = aeo_unet_gradients(h, r, e, loss)) return s;
    std::string& err = h->err;
    if (aeo_status s = h->adam(lr)) return s;
    CK(cudaStreamSynchronize(h->st));
    return AEO_OK;
}

aeo_status aeo_unet_activation(aeo_unet* h, int32_t which, float* out) {
    UN_ENTER(h);
    if (!out) { h->err = "out NULL"; return AEO_ERR_ARGUMENT; }
    std::string& err = h->err;
    struct A { bf16* p; int level, c; };
    const A acts[] = {{h->x, 0, 16},  {h->e1a, 0, 16}, {h->e1, 0, 16}, {h->p1, 1, 16}, {h->e2a, 1, 32},
                      {h->e2, 1, 32}, {h->p2, 2, 32},  {h->e3a, 2, 32}, {h->e3, 2, 32}, {h->u2, 1, 32},
                      {h->d2, 1, 16}, {h->u1, 0, 16},  {h->d1, 0, 16}};
    if (which < 0 || which > 13) { h->err = "activation index 0..13"; return AEO_ERR_ARGUMENT; }
    if (which == 13) {
        CK(cudaMemcpyAsync(out, h->z, sizeof(float) * h->n[0], cudaMemcpyDeviceToHost, h->st));
        CK(cudaStreamSynchronize(h->st));
        return AEO_OK;
    }
    const A& a = acts[which];
    const size_t cnt = (size_t)h->n[a.level] * a.c;
    std::vector<uint16_t> tmp(cnt);
    CK(cudaMemcpyAsync(tmp.data(), a.p, sizeof(uint16_t) * cnt, cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
    for (size_t q = 0; q < cnt; ++q) {
        uint32_t u = (uint32_t)tmp[q] << 16;
        std::memcpy(&out[q], &u, 4);
    }
    return AEO_OK;
}

aeo_status aeo_unet_profile(aeo_unet* h, int32_t what, int32_t reps, double* ms) {
    UN_ENTER(h);
    if (!ms || reps < 1) { h->err = "profile: ms NULL or reps < 1"; return AEO_ERR_ARGUMENT; }
    std::string& err = h->err;
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    auto run = [&]() -> aeo_status {
        switch (what) {
        case 0: return h->forward_(h->rbuf);
        case 1: {
            if (aeo_status s = h->forward_(h->rbuf)) return s;
            return h->backward(h->ebuf);
        }
        case 2: return h->conv(L_E1, false, h->e1a, h->e1, h->bias(L_E1), nullptr, nullptr, 1);
        case 3: return h->wgrad(L_E1, h->e1a, h->g_e1);
        default: h->err = "profile: unknown part"; return AEO_ERR_ARGUMENT;
        }
    };
    for (int w = 0; w < 2; ++w)
        if (aeo_status s = run()) return s;
    CK(cudaEventRecord(e0, h->st));
    for (int i = 0; i < reps; ++i)
        if (aeo_status s = run()) return s;
    CK(cudaEventRecord(e1, h->st));
    CK(cudaEventSynchronize(e1));
    float t = 0;
    CK(cudaEventElapsedTime(&t, e0, e1));
    *ms = double(t) / reps;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (what == 1 || what == 3) CK(cudaMemsetAsync(h->G, 0, sizeof(float) * h->off[NLAYERS], h->st));
    return h->check_err();
}

const char* aeo_unet_last_error(const aeo_unet* h) { return h ? h->err.c_str() : g_unet_error.c_str(); }

}  // extern "C"

// ----------------------------------------------------------------- internal
// used by the MG-PCG solve graph (aeo_mgpcg.cu): the forward pass on a
// device residual, launched on the solver's stream, result in unet_output().
aeo_status aeo_unet_forward_on(aeo_unet* h, const double* r_dev, cudaStream_t s) { return h->forward(r_dev, s); }
const float* aeo_unet_output(const aeo_unet* h) { return h->z; }
long long aeo_unet_cells(const aeo_unet* h) { return h->n[0]; }
