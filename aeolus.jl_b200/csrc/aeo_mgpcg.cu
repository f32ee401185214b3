// aeo_mgpcg.cu -- multigrid-preconditioned conjugate gradients for
// div(c grad phi) = b on a uniform grid (the cut-cell pressure solve).
//
// The algorithm is the reference's MGPreconditionedCG (src/Multigrid.jl:
// 551-967, pcg! in src/Backends.jl:1511-1589): CG on the FP64 operator with
// face coefficients, deflated for a singular operator (periodic / Neumann
// axes), preconditioned by one V-cycle of red-black Gauss-Seidel (nu1 / nu2
// sweeps), full-weighting restriction, trilinear prolongation and face
// coefficients coarsened by four-face means, with a long RB-GS smoothing on
// the coarsest level.
//
// GPU design:
//   * the whole solve is one CUDA graph: a prologue, a conditional WHILE node
//     whose body is one CG iteration (operator, update, V-cycle, reductions,
//     direction), and the final mean shift.  The loop condition is set on the
//     device by the last kernel of each iteration (converged, breakdown, or
//     the iteration cap), so no host round trip happens between iterations
//     and the loop always ends by the cap;
//   * every reduction is FP64 and deterministic: fixed grids, per-block
//     partials, and the last block to finish folds the partials in a fixed
//     order and computes the scalars (alpha, beta, the means, the status) in
//     device memory;
//   * levels are interior-only arrays; halos are index maps (periodic wrap,
//     Neumann mirror), exact for the even dimensions of every level that is
//     not the coarsest;
//   * the coarsest level runs all its sweeps in one thread block with its
//     arrays in shared memory (threads own columns; colour passes in place,
//     or double-buffered where a periodic axis of odd length would join two
//     cells of one colour), the reference's halo-copy semantics at any parity;
//   * face coefficients with at most 256 distinct values (the sampled
//     apertures of a cut-cell geometry) are stored as one-byte codes into a
//     table of the values themselves: the same operator at 3 bytes per cell
//     instead of 12 (FP32) or 24 (FP64);
//   * the first half-sweep of a level that starts from zero is pointwise
//     (every neighbour is zero), so it is fused with the zeroing and with
//     the mean projection of the level's right-hand side;
//   * the coarsest solve (nu sweeps of RB-GS from zero, a linear map of its
//     right-hand side) is precomputed once per coefficient field as a dense
//     matrix, built by running the sweeps on every unit vector, and applied
//     as one L2-resident matrix-vector product on all SMs;
//   * the mean projections the reference applies to phi after smoothing and
//     prolongation shift phi by a constant; RB-GS, the residual and the
//     prolongation commute with constant shifts and the CG deflation removes
//     the mean of z, so they are omitted; the projections of every
//     right-hand side are kept.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdlib>
#include <cstdint>
#include <cstring>
#include <new>
#include <string>
#include <type_traits>
#include <unordered_map>
#include <vector>

#include "../../include/aeolus_b200_mgpcg.h"
#include "../../include/aeolus_b200_unet.h"
#include "aeo_mg_kernels.cuh"

// Launch with programmatic stream serialisation (the kernel may start while
// the one before it drains, and waits in pdl_wait for its completion), unless
// the handle turned it off.
#define AEO_PDL_LAUNCH(KERN, GRID, BLOCK, SMEM, STREAM, ...)                                        \
    do {                                                                                          \
        cudaLaunchConfig_t lc_{};                                                                 \
        lc_.gridDim = dim3(GRID);                                                                 \
        lc_.blockDim = dim3(BLOCK);                                                               \
        lc_.dynamicSmemBytes = (size_t)(SMEM);                                                    \
        lc_.stream = (STREAM);                                                                    \
        cudaLaunchAttribute la_[1];                                                               \
        la_[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;                           \
        la_[0].val.programmaticStreamSerializationAllowed = pdl_on ? 1 : 0;                       \
        lc_.attrs = la_;                                                                          \
        lc_.numAttrs = 1;                                                                         \
        cudaLaunchKernelEx(&lc_, KERN, __VA_ARGS__);                                              \
    } while (0)

// the learned preconditioner's forward pass on a device residual (aeo_unet.cu)
aeo_status aeo_unet_forward_on(aeo_unet* h, const double* r_dev, cudaStream_t s);
const float* aeo_unet_output(const aeo_unet* h);
long long aeo_unet_cells(const aeo_unet* h);

namespace {

using namespace mgk;

constexpr int MAX_LEVELS = 24;

struct MgBase {
    aeo_mg_config cfg{};
    std::string err;
    virtual ~MgBase() {}
    void fail(const std::string& m) { err = m; }
    virtual aeo_status init(const double* cx, const double* cy, const double* cz) = 0;
    virtual aeo_status solve(const double* b, double* x, bool device, aeo_mg_stats* st) = 0;
    virtual aeo_status cycles(const double* b, double* x, aeo_mg_stats* st) = 0;
    virtual aeo_status apply(const double* x, double* out) = 0;
    virtual aeo_status precondition(const double* r, double* z) = 0;
    virtual aeo_status profile(int what, int reps, double* ms) = 0;
    virtual int nlevels() const = 0;
    virtual void level_dims(int l, int32_t* d) const = 0;
    virtual int launches_per_iteration() const = 0;
    virtual int launches_per_solve(int iterations) const = 0;
    virtual aeo_status set_learned(aeo_unet* net, double stag) = 0;
    virtual aeo_status harvest(const double* b, double* x, aeo_mg_stats* st, double* rh, double* xh, int cap,
                               int* count) = 0;
    // the stepping engine's use: the device right-hand side and solution
    // buffers, the solve enqueued on the caller's stream, the last statistics
    virtual void buffers(double** b, double** x) = 0;
    virtual aeo_status launch_on(cudaStream_t s) = 0;
    virtual aeo_status enqueue_on(cudaStream_t s) = 0;
    virtual aeo_status order_before(cudaStream_t s) = 0;
    virtual aeo_status last_stats(aeo_mg_stats* o) = 0;
};

#define CK(call)                                                                         \
    do {                                                                                 \
        cudaError_t e_ = (call);                                                         \
        if (e_ != cudaSuccess) {                                                         \
            fail(std::string(#call) + ": " + cudaGetErrorString(e_));                    \
            return AEO_ERR_CUDA;                                                         \
        }                                                                                \
    } while (0)

#define CKL()                                                                            \
    do {                                                                                 \
        cudaError_t e_ = cudaGetLastError();                                             \
        if (e_ != cudaSuccess) {                                                         \
            fail(std::string("kernel launch: ") + cudaGetErrorString(e_));               \
            return AEO_ERR_CUDA;                                                         \
        }                                                                                \
    } while (0)

// Four-face means of the face coefficients (_restrict_coeff,
// src/Multigrid.jl:465-496), on the host in FP64 at set-up.
void restrict_coeff(int nx, int ny, int nz, const std::vector<double>& cx, const std::vector<double>& cy,
                    const std::vector<double>& cz, int cnx, int cny, int cnz, std::vector<double>& Cx,
                    std::vector<double>& Cy, std::vector<double>& Cz) {
    auto mn = [](int a, int b) { return a < b ? a : b; };
    const int sx1 = nx + 1, sx2 = ny, sx3 = nz, sy1 = nx, sy2 = ny + 1, sy3 = nz, sz1 = nx, sz2 = ny, sz3 = nz + 1;
    Cx.assign((size_t)(cnx + 1) * cny * cnz, 0.0);
    Cy.assign((size_t)cnx * (cny + 1) * cnz, 0.0);
    Cz.assign((size_t)cnx * cny * (cnz + 1), 0.0);
    auto fx = [&](int i, int j, int k) { return cx[(size_t)(i - 1) + (size_t)sx1 * ((size_t)(j - 1) + (size_t)sx2 * (k - 1))]; };
    auto fy = [&](int i, int j, int k) { return cy[(size_t)(i - 1) + (size_t)sy1 * ((size_t)(j - 1) + (size_t)sy2 * (k - 1))]; };
    auto fz = [&](int i, int j, int k) { return cz[(size_t)(i - 1) + (size_t)sz1 * ((size_t)(j - 1) + (size_t)sz2 * (k - 1))]; };
    for (int K = 1; K <= cnz; ++K)
        for (int J = 1; J <= cny; ++J)
            for (int I = 1; I <= cnx + 1; ++I) {
                int i = 2 * I - 1;
                double s = 0;
                for (int dk = 0; dk <= 1; ++dk)
                    for (int dj = 0; dj <= 1; ++dj) s += fx(mn(i, sx1), mn(2 * J - 1 + dj, sx2), mn(2 * K - 1 + dk, sx3));
                Cx[(size_t)(I - 1) + (size_t)(cnx + 1) * ((size_t)(J - 1) + (size_t)cny * (K - 1))] = s * 0.25;
            }
    for (int K = 1; K <= cnz; ++K)
        for (int J = 1; J <= cny + 1; ++J)
            for (int I = 1; I <= cnx; ++I) {
                int j = 2 * J - 1;
                double s = 0;
                for (int dk = 0; dk <= 1; ++dk)
                    for (int di = 0; di <= 1; ++di) s += fy(mn(2 * I - 1 + di, sy1), mn(j, sy2), mn(2 * K - 1 + dk, sy3));
                Cy[(size_t)(I - 1) + (size_t)cnx * ((size_t)(J - 1) + (size_t)(cny + 1) * (K - 1))] = s * 0.25;
            }
    for (int K = 1; K <= cnz + 1; ++K)
        for (int J = 1; J <= cny; ++J)
            for (int I = 1; I <= cnx; ++I) {
                int k = 2 * K - 1;
                double s = 0;
                for (int dj = 0; dj <= 1; ++dj)
                    for (int di = 0; di <= 1; ++di) s += fz(mn(2 * I - 1 + di, sz1), mn(2 * J - 1 + dj, sz2), mn(k, sz3));
                Cz[(size_t)(I - 1) + (size_t)cnx * ((size_t)(J - 1) + (size_t)cny * (K - 1))] = s * 0.25;
            }
}

// One-byte codes of a level's face coefficients when it holds at most 256
// distinct values (the sampled apertures of a cut-cell geometry hold at most
// nsub^2 + 1): tab[code] is the value itself, so the coded operator is
// exactly the given one.
bool encode(const std::vector<double>& x, const std::vector<double>& y, const std::vector<double>& z,
            std::vector<double>& tab, std::vector<uint8_t>& kx, std::vector<uint8_t>& ky, std::vector<uint8_t>& kz) {
    std::unordered_map<uint64_t, uint8_t> code;
    tab.clear();
    auto key = [](double v) {
        uint64_t u;
        std::memcpy(&u, &v, 8);
        return u;
    };
    for (const std::vector<double>* a : {&x, &y, &z})
        for (double v : *a) {
            uint64_t u = key(v);
            if (code.find(u) != code.end()) continue;
            if (tab.size() == 256) return false;
            code.emplace(u, (uint8_t)tab.size());
            tab.push_back(v);
        }
    auto fill = [&](const std::vector<double>& a, std::vector<uint8_t>& k) {
        k.resize(a.size());
        for (size_t q = 0; q < a.size(); ++q) k[q] = code[key(a[q])];
    };
    fill(x, kx);
    fill(y, ky);
    fill(z, kz);
    return true;
}

template <typename R>
struct Mg : MgBase {
    cudaStream_t st = nullptr, st_body = nullptr, st_br[2] = {nullptr, nullptr};
    aeo_unet* net = nullptr;       // the learned preconditioner (AEO_PC_LEARNED)
    double* invd = nullptr;        // AEO_PC_JACOBI: 1 / the operator's diagonal (0 on a fully blocked cell)
    double* zj = nullptr;          // ... and z = r / diag
    std::vector<double> h_invd;
    double* hist_x = nullptr;      // harvest history, `hist_cap` slots of n
    double* hist_r = nullptr;
    int hist_cap = 0;
    cudaGraphExec_t g_harvest = nullptr;
    Bc bc{0, 0, 0};
    int nl = 0;
    int n = 0;
    Level<R> L[MAX_LEVELS];
    std::vector<void*> allocs;
    Coef<double> opd;              // the operator's coefficients, FP64 values or codes
    Coef<float> opf;               // ... or FP32 values when every one is exact in FP32
    bool op_f32 = false;
    int coded_levels = 0;
    double *b = nullptr, *x = nullptr, *r = nullptr, *p = nullptr, *Ap = nullptr;
    double* part = nullptr;
    size_t part_cap = 0;           // doubles in `part`
    double* bmeans = nullptr;      // one device scalar per level
    PcgState* S = nullptr;
    PcgState* hS = nullptr;        // pinned host copy
    cudaEvent_t ev_own = nullptr;  // orders this handle's stream before a launch on another
    int* dzero = nullptr;          // a device flag that stays 0 (kernels run outside a solve)
    int coarse_staged = 0;
    int coarse_inplace = 1;        // 0 when a periodic axis of the coarsest level has an odd length
    size_t coarse_smem = 0;
    R* coarse_spare = nullptr;     // the coarsest level's second buffer when not staged
    R* coarse_mat = nullptr;       // the coarsest solve as a dense n x n matrix (nullptr: run the sweeps)
    int coarse_col = 0;            // the register-column coarsest kernel applies
    bool pdl_on = true;            // programmatic launches of the cycle and CG kernels
    int coarse_col_threads = 0;
    size_t coarse_col_smem = 0;
    cudaGraphExec_t g_solve = nullptr, g_cycles = nullptr;
    int body_launches = 0;
    int prologue_launches = 0;

    ~Mg() override {
        if (st) cudaStreamSynchronize(st);
        if (g_solve) cudaGraphExecDestroy(g_solve);
        if (g_cycles) cudaGraphExecDestroy(g_cycles);
        if (g_harvest) cudaGraphExecDestroy(g_harvest);
        for (void* a : allocs) cudaFree(a);
        if (hist_x) cudaFree(hist_x);
        if (hist_r) cudaFree(hist_r);
        if (hS) cudaFreeHost(hS);
        if (ev_own) cudaEventDestroy(ev_own);
        if (st) cudaStreamDestroy(st);
        if (st_body) cudaStreamDestroy(st_body);
        for (cudaStream_t b_ : st_br)
            if (b_) cudaStreamDestroy(b_);
    }

    template <typename T>
    aeo_status dalloc(T** ptr, size_t count) {
        void* a = nullptr;
        CK(cudaMalloc(&a, sizeof(T) * (count ? count : 1)));
        allocs.push_back(a);
        *ptr = reinterpret_cast<T*>(a);
        return AEO_OK;
    }

    template <typename T, typename S_>
    aeo_status upload(const T** out, const std::vector<S_>& h) {
        T* d;
        if (aeo_status s = dalloc(&d, h.size())) return s;
        std::vector<T> t(h.begin(), h.end());
        CK(cudaMemcpy(d, t.data(), sizeof(T) * t.size(), cudaMemcpyHostToDevice));
        *out = d;
        return AEO_OK;
    }

    int nlevels() const override { return nl; }
    void level_dims(int l, int32_t* d) const override {
        d[0] = L[l].nx;
        d[1] = L[l].ny;
        d[2] = L[l].nz;
    }
    int launches_per_iteration() const override { return body_launches; }
    // kernels of one solve graph launch of `iterations` CG iterations: the
    // prologue, the loop bodies and the two of the mean shift (the U-Net's own
    // kernels in a learned prologue are not counted)
    int launches_per_solve(int iterations) const override {
        return prologue_launches + iterations * body_launches + 2;
    }

    static dim3 half_grid(const Level<R>& F) {
        return dim3((unsigned)((F.nx / 2 + RB_X - 1) / RB_X), (unsigned)((F.ny + RB_Y - 1) / RB_Y), (unsigned)F.nz);
    }
    static dim3 cell_grid(const Level<R>& F) {
        return dim3((unsigned)((F.nx + RB_X - 1) / RB_X), (unsigned)((F.ny + RB_Y - 1) / RB_Y), (unsigned)F.nz);
    }
    static dim3 restrict_grid(const Level<R>& Cl) { return cell_grid(Cl); }
    static int row_blocks(int rows) {
        int b = (rows + RB_Y - 1) / RB_Y;
        return b < RED_BLOCKS ? b : RED_BLOCKS;
    }

    aeo_status init(const double* cx, const double* cy, const double* cz) override {
        bc = {cfg.bc_x, cfg.bc_y, cfg.bc_z};
        CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        CK(cudaStreamCreateWithFlags(&st_body, cudaStreamNonBlocking));
        CK(cudaStreamCreateWithFlags(&st_br[0], cudaStreamNonBlocking));
        CK(cudaStreamCreateWithFlags(&st_br[1], cudaStreamNonBlocking));
        const bool coeff = cx != nullptr;
        int nx = cfg.nx, ny = cfg.ny, nz = cfg.nz;
        double dx = cfg.dx, dy = cfg.dy, dz = cfg.dz;
        n = nx * ny * nz;
        if (cfg.precond == AEO_PC_JACOBI) {
            // the diagonal of the fine operator: -sum over the faces of c / h^2,
            // a Neumann boundary face (whose mirror neighbour is the cell itself)
            // contributing nothing
            h_invd.assign((size_t)n, 0.0);
            const double ix2 = 1.0 / (dx * dx), iy2 = 1.0 / (dy * dy), iz2 = 1.0 / (dz * dz);
            auto C3 = [&](const double* c, size_t f) { return c ? c[f] : 1.0; };
            for (int k = 0; k < nz; ++k)
                for (int j = 0; j < ny; ++j)
                    for (int i = 0; i < nx; ++i) {
                        const size_t q = (size_t)i + (size_t)nx * (j + (size_t)ny * k);
                        const size_t xr = (size_t)(nx + 1) * (j + (size_t)ny * k) + i;
                        const size_t yr = (size_t)nx * (j + (size_t)(ny + 1) * k) + i;
                        double sum = 0.0;
                        if (!(i == 0 && cfg.bc_x == AEO_MG_NEUMANN)) sum += C3(cx, xr) * ix2;
                        if (!(i == nx - 1 && cfg.bc_x == AEO_MG_NEUMANN)) sum += C3(cx, xr + 1) * ix2;
                        if (!(j == 0 && cfg.bc_y == AEO_MG_NEUMANN)) sum += C3(cy, yr) * iy2;
                        if (!(j == ny - 1 && cfg.bc_y == AEO_MG_NEUMANN)) sum += C3(cy, yr + nx) * iy2;
                        if (!(k == 0 && cfg.bc_z == AEO_MG_NEUMANN)) sum += C3(cz, q) * iz2;
                        if (!(k == nz - 1 && cfg.bc_z == AEO_MG_NEUMANN)) sum += C3(cz, q + (size_t)nx * ny) * iz2;
                        h_invd[q] = sum > 0.0 ? -1.0 / sum : 0.0;
                    }
        }
        std::vector<double> hx, hy, hz;
        if (coeff) {
            hx.assign(cx, cx + (size_t)(nx + 1) * ny * nz);
            hy.assign(cy, cy + (size_t)nx * (ny + 1) * nz);
            hz.assign(cz, cz + (size_t)nx * ny * (nz + 1));
        }
        if (aeo_status s = dalloc(&bmeans, MAX_LEVELS)) return s;
        CK(cudaMemset(bmeans, 0, sizeof(double) * MAX_LEVELS));
        std::vector<double> Cx, Cy, Cz, tab;
        std::vector<uint8_t> kx, ky, kz;
        // the hierarchy (src/Multigrid.jl:572-591)
        while (true) {
            Level<R>& V = L[nl];
            V.nx = nx; V.ny = ny; V.nz = nz;
            V.n = nx * ny * nz;
            V.ix2 = R(1) / (R(dx) * R(dx));   // one(T) / dx^2 (src/Multigrid.jl:162-164)
            V.iy2 = R(1) / (R(dy) * R(dy));
            V.iz2 = R(1) / (R(dz) * R(dz));
            if (aeo_status s = dalloc(&V.phi, V.n)) return s;
            if (aeo_status s = dalloc(&V.b, V.n)) return s;
            V.r = nullptr;
            V.bmean = bmeans + nl;
            V.c = Coef<R>();
            if (coeff) {
                if (encode(hx, hy, hz, tab, kx, ky, kz)) {
                    if (aeo_status s = upload(&V.c.kx, kx)) return s;
                    if (aeo_status s = upload(&V.c.ky, ky)) return s;
                    if (aeo_status s = upload(&V.c.kz, kz)) return s;
                    std::vector<double> tab256(tab);
                    tab256.resize(256, 0.0);   // the smoothers stage all 256 entries in shared memory
                    if (aeo_status s = upload(&V.c.tab, tab256)) return s;
                    ++coded_levels;
                    if (nl == 0) {
                        opd.kx = V.c.kx; opd.ky = V.c.ky; opd.kz = V.c.kz;
                        if (aeo_status s = upload(&opd.tab, tab256)) return s;
                    }
                } else {
                    if (aeo_status s = upload(&V.c.cx, hx)) return s;
                    if (aeo_status s = upload(&V.c.cy, hy)) return s;
                    if (aeo_status s = upload(&V.c.cz, hz)) return s;
                    if (nl == 0) {
                        bool exact = std::is_same<R, float>::value;
                        for (const std::vector<double>* v : {&hx, &hy, &hz})
                            for (size_t q = 0; exact && q < v->size(); ++q) exact = double(float((*v)[q])) == (*v)[q];
                        if (exact) {
                            op_f32 = true;
                            opf.cx = reinterpret_cast<const float*>(V.c.cx);
                            opf.cy = reinterpret_cast<const float*>(V.c.cy);
                            opf.cz = reinterpret_cast<const float*>(V.c.cz);
                        } else if (std::is_same<R, double>::value) {
                            opd.cx = reinterpret_cast<const double*>(V.c.cx);
                            opd.cy = reinterpret_cast<const double*>(V.c.cy);
                            opd.cz = reinterpret_cast<const double*>(V.c.cz);
                        } else {
                            if (aeo_status s = upload(&opd.cx, hx)) return s;
                            if (aeo_status s = upload(&opd.cy, hy)) return s;
                            if (aeo_status s = upload(&opd.cz, hz)) return s;
                        }
                    }
                }
            }
            ++nl;
            bool cxo = nx % 2 == 0 && nx / 2 >= cfg.min_size;
            bool cyo = ny % 2 == 0 && ny / 2 >= cfg.min_size;
            bool czo = nz % 2 == 0 && nz / 2 >= cfg.min_size;
            if (!(cxo && cyo && czo) || nl == MAX_LEVELS) break;
            int cnx = nx / 2, cny = ny / 2, cnz = nz / 2;
            if (coeff) {
                restrict_coeff(nx, ny, nz, hx, hy, hz, cnx, cny, cnz, Cx, Cy, Cz);
                hx.swap(Cx); hy.swap(Cy); hz.swap(Cz);
            }
            if (aeo_status s = dalloc(&V.r, V.n)) return s;
            nx = cnx; ny = cny; nz = cnz;
            dx *= 2; dy *= 2; dz *= 2;
        }
        const Level<R>& C = L[nl - 1];
        if (C.n > COARSE_MAX_CELLS) {
            fail("coarsest multigrid level has " + std::to_string(C.n) + " cells, above the " +
                 std::to_string(COARSE_MAX_CELLS) + " one block solves: give nx, ny, nz more factors of two");
            return AEO_ERR_ARGUMENT;
        }
        size_t cb = sizeof(R) * (3 * (size_t)C.n + (coeff ? (size_t)(C.nx + 1) * C.ny * C.nz +
                                                          (size_t)C.nx * (C.ny + 1) * C.nz +
                                                          (size_t)C.nx * C.ny * (C.nz + 1) : 0));
        coarse_staged = cb <= 200 * 1024;
        coarse_inplace = !((cfg.bc_x == AEO_MG_PERIODIC && C.nx % 2) || (cfg.bc_y == AEO_MG_PERIODIC && C.ny % 2) ||
                           (cfg.bc_z == AEO_MG_PERIODIC && C.nz % 2));
        coarse_smem = coarse_staged ? cb : 0;
        coarse_col_smem = sizeof(R) * (2 * (size_t)C.n + (coeff ? (size_t)(C.nx + 1) * C.ny * C.nz +
                                                             (size_t)C.nx * (C.ny + 1) * C.nz +
                                                             (size_t)C.nx * C.ny * (C.nz + 1) : 0));
        coarse_col = coarse_inplace && C.nz <= COL_NZ && C.nx * C.ny <= COARSE_THREADS && coarse_col_smem <= 225 * 1024;
        coarse_col_threads = ((C.nx * C.ny + 31) / 32) * 32;
        if (coarse_col && coarse_col_smem > 48 * 1024) {
            CK(cudaFuncSetAttribute(mg_coarsest_col_kernel<R, 256>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)coarse_col_smem));
            CK(cudaFuncSetAttribute(mg_coarsest_col_kernel<R, COARSE_THREADS>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, (int)coarse_col_smem));
        }
        if (coarse_smem > 48 * 1024)
            CK(cudaFuncSetAttribute(mg_coarsest_kernel<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)coarse_smem));
        if (aeo_status s = dalloc(&coarse_spare, C.n)) return s;
        // the coarsest solve as a matrix, when its sweeps fit shared memory and
        // the matrix is modest: one block per unit right-hand side
        if (coarse_staged && (size_t)C.n * C.n * sizeof(R) <= (size_t(512) << 20) && cfg.coarse_sweeps > 0) {
            if (aeo_status s = dalloc(&coarse_mat, (size_t)C.n * C.n)) return s;
            int* dz = nullptr;
            if (aeo_status s = dalloc(&dz, 1)) return s;
            CK(cudaMemset(dz, 0, sizeof(int)));
            mg_coarsest_kernel<R><<<C.n, COARSE_THREADS, coarse_smem, st>>>(L[nl - 1], coarse_spare, bc,
                                                                            cfg.coarse_sweeps, 1, coarse_inplace,
                                                                            nullptr, nullptr, dz, coarse_mat);
            CKL();
            CK(cudaStreamSynchronize(st));
        }
        if (aeo_status s = dalloc(&b, n)) return s;
        if (aeo_status s = dalloc(&x, n)) return s;
        if (aeo_status s = dalloc(&r, n)) return s;
        if (aeo_status s = dalloc(&p, n)) return s;
        if (aeo_status s = dalloc(&Ap, n)) return s;
        if (cfg.precond == AEO_PC_JACOBI) {
            if (aeo_status s = dalloc(&invd, n)) return s;
            if (aeo_status s = dalloc(&zj, n)) return s;
            CK(cudaMemcpy(invd, h_invd.data(), sizeof(double) * n, cudaMemcpyHostToDevice));
        }
        part_cap = (size_t)RED_BLOCKS * 8;
        for (int l = 0; l + 1 < nl; ++l) {
            dim3 g = restrict_grid(L[l + 1]);
            size_t nb = (size_t)g.x * g.y * g.z;
            if (nb > part_cap) part_cap = nb;
        }
        if (aeo_status s = dalloc(&part, part_cap)) return s;
        if (aeo_status s = dalloc(&S, 1)) return s;
        if (aeo_status s = dalloc(&dzero, 1)) return s;
        CK(cudaMemset(dzero, 0, sizeof(int)));
        CK(cudaMallocHost(&hS, sizeof(PcgState)));
        PcgState h0{};
        h0.tol = cfg.tol;
        h0.n = double(n);
        h0.maxit = cfg.maxit;
        h0.project = 1;            // periodic / Neumann on every axis: always singular
        h0.flexible = cfg.flexible;
        CK(cudaMemcpy(S, &h0, sizeof(PcgState), cudaMemcpyHostToDevice));
        CK(cudaMemset(part, 0, sizeof(double) * part_cap));
        return AEO_OK;
    }

    aeo_status launch_apply(cudaStream_t s, const double* in, double* out, int standalone) {
        const double ix2 = 1.0 / (cfg.dx * cfg.dx), iy2 = 1.0 / (cfg.dy * cfg.dy), iz2 = 1.0 / (cfg.dz * cfg.dz);
        const dim3 blk(RB_X, RB_Y);
        const int nb = row_blocks(cfg.ny * cfg.nz);
        if (op_f32)
            AEO_PDL_LAUNCH((pcg_apply_kernel<float, CF_VALUES>), nb, blk, 0, s, in, out, opf, cfg.nx, cfg.ny, cfg.nz, bc, ix2, iy2,
                                                                  iz2, S, part, standalone);
        else if (opd.kx)
            AEO_PDL_LAUNCH((pcg_apply_kernel<double, CF_CODES>), nb, blk, 0, s, in, out, opd, cfg.nx, cfg.ny, cfg.nz, bc, ix2, iy2,
                                                                  iz2, S, part, standalone);
        else if (opd.cx)
            AEO_PDL_LAUNCH((pcg_apply_kernel<double, CF_VALUES>), nb, blk, 0, s, in, out, opd, cfg.nx, cfg.ny, cfg.nz, bc, ix2, iy2,
                                                                   iz2, S, part, standalone);
        else
            AEO_PDL_LAUNCH((pcg_apply_kernel<double, CF_CONST>), nb, blk, 0, s, in, out, opd, cfg.nx, cfg.ny, cfg.nz, bc, ix2, iy2,
                                                                  iz2, S, part, standalone);
        CKL();
        return AEO_OK;
    }

    int vcycle_launches() const {
        int c = 1;   // coarsest
        for (int l = 0; l < nl - 1; ++l) c += 2 * cfg.nu1 + 2 * cfg.nu2 + 3;
        return c;
    }

    aeo_status launch_coarsest(cudaStream_t s, Level<R>& C, const double* r0, const int* done) {
        if (coarse_mat) {
            AEO_PDL_LAUNCH((mg_coarse_matvec_kernel<R>), (C.n + 7) / 8, 256, 0, s, C, coarse_mat, r0, &S->mr, done);
            CKL();
            return AEO_OK;
        }
        if (coarse_col) {
            if (coarse_col_threads <= 256)
                AEO_PDL_LAUNCH((mg_coarsest_col_kernel<R, 256>), 1, coarse_col_threads, coarse_col_smem, s, C, bc, cfg.coarse_sweeps,
                                                                                             r0, &S->mr, done);
            else
                AEO_PDL_LAUNCH((mg_coarsest_col_kernel<R, COARSE_THREADS>), 1, coarse_col_threads, coarse_col_smem, s, 
                    C, bc, cfg.coarse_sweeps, r0, &S->mr, done);
            CKL();
            return AEO_OK;
        }
        mg_coarsest_kernel<R><<<1, COARSE_THREADS, coarse_smem, s>>>(C, coarse_spare, bc, cfg.coarse_sweeps,
                                                                     coarse_staged, coarse_inplace, r0, &S->mr, done,
                                                                     nullptr);
        CKL();
        return AEO_OK;
    }

    // One V-cycle from phi = 0 with level-0 right-hand side r0 - mean
    // (mg_vcycle!, src/Multigrid.jl:706-739); from_zero = false: level 0
    // keeps its phi and b (the standalone cycles).
    aeo_status launch_vcycle(cudaStream_t s, const double* r0, bool from_zero, const int* done) {
        const double* mr = &S->mr;
        const dim3 blk(RB_X, RB_Y);
        if (nl == 1) {
            if (!from_zero) {
                fail("standalone multigrid cycles need at least two levels");
                return AEO_ERR_ARGUMENT;
            }
            return launch_coarsest(s, L[0], r0, done);
        }
        for (int l = 0; l < nl - 1; ++l) {
            Level<R>& F = L[l];
            const dim3 hg = half_grid(F);
            int sw0 = 0;
            if (l > 0 || from_zero) {
                AEO_PDL_LAUNCH((mg_first_kernel<R>), hg, blk, 0, s, F, bc, l == 0 ? r0 : nullptr, mr, done);
                CKL();
                if (aeo_status q = launch_rbgs(s, F, 1, done)) return q;
                sw0 = 1;
            }
            for (int sw = sw0; sw < cfg.nu1; ++sw)
                for (int c = 0; c < 2; ++c)
                    if (aeo_status q = launch_rbgs(s, F, c, done)) return q;
            Level<R>& Cl = L[l + 1];
            if (aeo_status q = launch_residual(s, F, done)) return q;
            AEO_PDL_LAUNCH((mg_restrict_kernel<R>), restrict_grid(Cl), blk, 0, s, F, Cl, part, &S->counter, done);
            CKL();
        }
        if (aeo_status q = launch_coarsest(s, L[nl - 1], nullptr, done)) return q;
        for (int l = nl - 2; l >= 0; --l) {
            Level<R>& F = L[l];
            AEO_PDL_LAUNCH((mg_prolong_kernel<R>), cell_grid(F), blk, 0, s, F, L[l + 1], bc, done);
            CKL();
            for (int sw = 0; sw < cfg.nu2; ++sw)
                for (int c = 0; c < 2; ++c)
                    if (aeo_status q = launch_rbgs(s, F, c, done)) return q;
        }
        return AEO_OK;
    }

    // one colour pass / the residual of level F in its coefficient form
    // columns of 8 levels a thread where that still leaves 8 blocks an SM
    aeo_status launch_rbgs(cudaStream_t s, const Level<R>& F, int colour, const int* done) {
        const unsigned bx = (unsigned)((F.nx / 2 + RB_X - 1) / RB_X), by = (unsigned)((F.ny + RB_Y - 1) / RB_Y);
        const bool col = (size_t)bx * by * ((F.nz + 7) / 8) >= 8 * 148;
        const dim3 hg(bx, by, (unsigned)(col ? (F.nz + 7) / 8 : F.nz)), blk(RB_X, RB_Y);
        if (col) {
            if (F.c.kx) AEO_PDL_LAUNCH((mg_rbgs_kernel<R, CF_CODES, 8>), hg, blk, 0, s, F, bc, colour, done);
            else if (F.c.cx) AEO_PDL_LAUNCH((mg_rbgs_kernel<R, CF_VALUES, 8>), hg, blk, 0, s, F, bc, colour, done);
            else AEO_PDL_LAUNCH((mg_rbgs_kernel<R, CF_CONST, 8>), hg, blk, 0, s, F, bc, colour, done);
        } else {
            if (F.c.kx) AEO_PDL_LAUNCH((mg_rbgs_kernel<R, CF_CODES, 1>), hg, blk, 0, s, F, bc, colour, done);
            else if (F.c.cx) AEO_PDL_LAUNCH((mg_rbgs_kernel<R, CF_VALUES, 1>), hg, blk, 0, s, F, bc, colour, done);
            else AEO_PDL_LAUNCH((mg_rbgs_kernel<R, CF_CONST, 1>), hg, blk, 0, s, F, bc, colour, done);
        }
        CKL();
        return AEO_OK;
    }
    aeo_status launch_residual(cudaStream_t s, const Level<R>& F, const int* done) {
        const dim3 g = cell_grid(F), blk(RB_X, RB_Y);
        if (F.c.kx) AEO_PDL_LAUNCH((mg_residual_kernel<R, CF_CODES>), g, blk, 0, s, F, bc, done);
        else if (F.c.cx) AEO_PDL_LAUNCH((mg_residual_kernel<R, CF_VALUES>), g, blk, 0, s, F, bc, done);
        else AEO_PDL_LAUNCH((mg_residual_kernel<R, CF_CONST>), g, blk, 0, s, F, bc, done);
        CKL();
        return AEO_OK;
    }

    // z: level-0 phi after the cycle, the network's output, or r itself for plain CG
    aeo_status launch_rz_dir(cudaStream_t s, int first, int pc = -1) {
        if (pc < 0) pc = cfg.precond;
        if (pc == AEO_PC_LEARNED) {
            const float* zf = aeo_unet_output(net);
            AEO_PDL_LAUNCH((pcg_rz_kernel<float>), RED_BLOCKS, TPB, 0, s, r, zf, Ap, n, S, part, first);
            CKL();
            AEO_PDL_LAUNCH((pcg_dir_kernel<float>), RED_BLOCKS, TPB, 0, s, p, zf, n, S, first);
        } else if (pc == AEO_PC_VCYCLE) {
            AEO_PDL_LAUNCH((pcg_rz_kernel<R>), RED_BLOCKS, TPB, 0, s, r, L[0].phi, Ap, n, S, part, first);
            CKL();
            AEO_PDL_LAUNCH((pcg_dir_kernel<R>), RED_BLOCKS, TPB, 0, s, p, L[0].phi, n, S, first);
        } else if (pc == AEO_PC_JACOBI) {
            AEO_PDL_LAUNCH((pcg_jacobi_kernel), RED_BLOCKS, TPB, 0, s, zj, r, invd, n, S);
            CKL();
            AEO_PDL_LAUNCH((pcg_rz_kernel<double>), RED_BLOCKS, TPB, 0, s, r, zj, Ap, n, S, part, first);
            CKL();
            AEO_PDL_LAUNCH((pcg_dir_kernel<double>), RED_BLOCKS, TPB, 0, s, p, zj, n, S, first);
        } else {
            AEO_PDL_LAUNCH((pcg_rz_kernel<double>), RED_BLOCKS, TPB, 0, s, r, r, Ap, n, S, part, first);
            CKL();
            AEO_PDL_LAUNCH((pcg_dir_kernel<double>), RED_BLOCKS, TPB, 0, s, p, r, n, S, first);
        }
        CKL();
        return AEO_OK;
    }

    // The conditional handle of the graph being captured on `st` (value 0 at
    // every launch until a kernel sets it).
    aeo_status make_handle(cudaGraphConditionalHandle* hdl) {
        cudaStreamCaptureStatus cs;
        cudaGraph_t g = nullptr;
        CK(cudaStreamGetCaptureInfo(st, &cs, nullptr, &g, nullptr, nullptr));
        if (cs != cudaStreamCaptureStatusActive) {
            fail("internal: stream is not capturing");
            return AEO_ERR_STATE;
        }
        CK(cudaGraphConditionalHandleCreate(hdl, g, 0, cudaGraphCondAssignDefault));
        return AEO_OK;
    }

    // A conditional handle on the graph being captured on `s`, value `dflt`
    // at every launch until a kernel sets it.
    aeo_status make_handle_on(cudaStream_t s, cudaGraphConditionalHandle* hdl, unsigned dflt) {
        cudaStreamCaptureStatus cs;
        cudaGraph_t g = nullptr;
        CK(cudaStreamGetCaptureInfo(s, &cs, nullptr, &g, nullptr, nullptr));
        if (cs != cudaStreamCaptureStatusActive) {
            fail("internal: stream is not capturing");
            return AEO_ERR_STATE;
        }
        CK(cudaGraphConditionalHandleCreate(hdl, g, dflt, cudaGraphCondAssignDefault));
        return AEO_OK;
    }

    // Adds a conditional node (WHILE with one body, or IF with one or two) on
    // `hdl` to the graph being captured on `s`, captures body i on stream
    // bs[i], and continues the capture on `s` after the node.
    template <typename F0, typename F1>
    aeo_status capture_cond(cudaStream_t s, cudaGraphConditionalHandle hdl, cudaGraphConditionalNodeType type,
                            int nbodies, const cudaStream_t* bs, F0 body0, F1 body1) {
        cudaStreamCaptureStatus cs;
        cudaGraph_t g = nullptr;
        const cudaGraphNode_t* deps = nullptr;
        size_t ndeps = 0;
        CK(cudaStreamGetCaptureInfo(s, &cs, nullptr, &g, &deps, &ndeps));
        if (cs != cudaStreamCaptureStatusActive) {
            fail("internal: stream is not capturing");
            return AEO_ERR_STATE;
        }
        cudaGraphNodeParams cp = {};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = hdl;
        cp.conditional.type = type;
        cp.conditional.size = (unsigned)nbodies;
        cudaGraphNode_t node;
        std::vector<cudaGraphNode_t> dv(deps, deps + ndeps);
        CK(cudaGraphAddNode(&node, g, dv.data(), dv.size(), &cp));
        for (int i = 0; i < nbodies; ++i) {
            cudaGraph_t bodyg = cp.conditional.phGraph_out[i];
            CK(cudaStreamBeginCaptureToGraph(bs[i], bodyg, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
            aeo_status q = i == 0 ? body0(bs[i]) : body1(bs[i]);
            cudaGraph_t out = nullptr;
            cudaError_t e = cudaStreamEndCapture(bs[i], &out);
            if (q) return q;
            if (e != cudaSuccess) {
                fail(std::string("cudaStreamEndCapture(body): ") + cudaGetErrorString(e));
                return AEO_ERR_CUDA;
            }
        }
        CK(cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies));
        return AEO_OK;
    }

    template <typename F>
    aeo_status capture_while(cudaGraphConditionalHandle hdl, F body) {
        return capture_cond(st, hdl, cudaGraphCondTypeWhile, 1, &st_body, body,
                            [](cudaStream_t) -> aeo_status { return AEO_OK; });
    }

    // the preconditioner application of the body: the network or, after a
    // stagnation, the multigrid cycle, chosen on the device by an IF node
    aeo_status launch_learned_pc(cudaStream_t sb, int* count) {
        cudaGraphConditionalHandle h2;
        if (aeo_status q = make_handle_on(sb, &h2, 1)) return q;
        pcg_select_kernel<<<1, 1, 0, sb>>>(S, h2);
        CKL();
        *count += 1;
        return capture_cond(
            sb, h2, cudaGraphCondTypeIf, 2, st_br,
            [&](cudaStream_t s0) -> aeo_status {
                if (aeo_status q = aeo_unet_forward_on(net, r, s0)) {
                    fail("learned preconditioner: forward pass could not be captured");
                    return q;
                }
                return launch_rz_dir(s0, 0, AEO_PC_LEARNED);
            },
            [&](cudaStream_t s1) -> aeo_status {
                if (aeo_status q = launch_vcycle(s1, r, true, &S->done)) return q;
                return launch_rz_dir(s1, 0, AEO_PC_VCYCLE);
            });
    }

    aeo_status end_capture(cudaGraphExec_t* ex, aeo_status s) {
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(st, &g);
        if (s) {
            if (g) cudaGraphDestroy(g);
            return s;
        }
        if (e != cudaSuccess) {
            fail(std::string("cudaStreamEndCapture: ") + cudaGetErrorString(e));
            return AEO_ERR_CUDA;
        }
        cudaError_t e2 = cudaGraphInstantiate(ex, g, 0);
        cudaGraphDestroy(g);
        if (e2 != cudaSuccess) {
            fail(std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e2));
            return AEO_ERR_CUDA;
        }
        return AEO_OK;
    }

    // The solve graph: prologue, WHILE(one CG iteration), the mean shift.
    // The loop condition is set by pcg_cond_kernel before the loop and at
    // the end of every iteration.
    aeo_status build_solve(bool harvest = false) {
        CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed));
        aeo_status s = capture_solve(st, harvest);
        return end_capture(harvest ? &g_harvest : &g_solve, s);
    }

    // The solve's nodes captured on `s` (a stream capturing into this
    // handle's graph or into the caller's: the conditional nodes go into
    // whichever graph `s` is capturing).
    aeo_status capture_solve(cudaStream_t s0, bool harvest) {
        cudaGraphConditionalHandle hdl;
        if (aeo_status q = make_handle_on(s0, &hdl, 0)) return q;
        pcg_mean_kernel<<<RED_BLOCKS, TPB, 0, s0>>>(b, n, S, part, 0);
        CKL();
        pcg_init_kernel<<<RED_BLOCKS, TPB, 0, s0>>>(b, r, x, n, S, part);
        CKL();
        if (harvest) {
            pcg_harvest_kernel<<<RED_BLOCKS, TPB, 0, s0>>>(x, r, hist_x, hist_r, n, hist_cap, S);
            CKL();
        }
        if (cfg.precond == AEO_PC_VCYCLE)
            if (aeo_status q = launch_vcycle(s0, r, true, &S->done)) return q;
        if (cfg.precond == AEO_PC_LEARNED)
            if (aeo_status q = aeo_unet_forward_on(net, r, s0)) return q;
        if (aeo_status q = launch_rz_dir(s0, 1)) return q;
        pcg_cond_kernel<<<1, 1, 0, s0>>>(S, hdl, 0);
        CKL();
        if (!harvest)
            prologue_launches = 5 + (cfg.precond == AEO_PC_VCYCLE ? vcycle_launches() : 0) +
                                (cfg.precond == AEO_PC_JACOBI ? 1 : 0);
        if (aeo_status q = capture_cond(s0, hdl, cudaGraphCondTypeWhile, 1, &st_body,
                [&](cudaStream_t sb) -> aeo_status {
                    int c0 = 0;
                    if (aeo_status q2 = launch_apply(sb, p, Ap, 0)) return q2;
                    AEO_PDL_LAUNCH((pcg_update_kernel), RED_BLOCKS, TPB, 0, sb, x, r, p, Ap, n, S, part);
                    CKL();
                    c0 += 2;
                    if (harvest) {
                        pcg_harvest_kernel<<<RED_BLOCKS, TPB, 0, sb>>>(x, r, hist_x, hist_r, n, hist_cap, S);
                        CKL();
                        c0 += 1;
                    }
                    if (cfg.precond == AEO_PC_LEARNED) {
                        if (aeo_status q2 = launch_learned_pc(sb, &c0)) return q2;
                        c0 += 2;
                    } else {
                        if (cfg.precond == AEO_PC_VCYCLE) {
                            if (aeo_status q2 = launch_vcycle(sb, r, true, &S->done)) return q2;
                            c0 += vcycle_launches();
                        }
                        if (aeo_status q2 = launch_rz_dir(sb, 0)) return q2;
                        c0 += cfg.precond == AEO_PC_JACOBI ? 3 : 2;
                    }
                    pcg_cond_kernel<<<1, 1, 0, sb>>>(S, hdl, 0);
                    CKL();
                    body_launches = c0 + 1;
                    return AEO_OK;
                },
                [](cudaStream_t) -> aeo_status { return AEO_OK; }))
            return q;
        pcg_mean_kernel<<<RED_BLOCKS, TPB, 0, s0>>>(x, n, S, part, 1);
        CKL();
        shift_kernel<<<RED_BLOCKS, TPB, 0, s0>>>(x, n, S);
        CKL();
        return AEO_OK;
    }

    aeo_status stats_out(aeo_mg_stats* o, bool relative) {
        CK(cudaMemcpyAsync(hS, S, sizeof(PcgState), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        if (o) {
            o->iterations = hS->iters;
            o->status = hS->status;
            o->residual = relative ? hS->rel : hS->rnorm;
            o->bnorm = hS->bnorm;
            o->curvature = hS->curvature;
            o->fallback_at = hS->fallback_at;
            if (hS->status == AEO_MG_ZERO_RHS) o->residual = 0.0;
        }
        return AEO_OK;
    }

    void buffers(double** bo, double** xo) override {
        *bo = b;
        *xo = x;
    }
    // x = A^-1 b from the rhs buffer into the solution buffer, ordered on s
    // (the graph is captured once on this handle's stream; a graph launch
    // runs on any stream)
    aeo_status launch_on(cudaStream_t s) override {
        if (!g_solve)
            if (aeo_status q = build_solve()) return q;
        if (s != st) {
            // everything this handle queued on its own stream (set-up, the
            // coarsest map, weight changes) precedes the solve on s
            if (!ev_own) CK(cudaEventCreateWithFlags(&ev_own, cudaEventDisableTiming));
            CK(cudaEventRecord(ev_own, st));
            CK(cudaStreamWaitEvent(s, ev_own, 0));
        }
        CK(cudaGraphLaunch(g_solve, s));
        return AEO_OK;
    }
    // x = A^-1 b on s: captured inline when s is capturing (the caller's
    // graph then holds the loop), else the handle's own solve graph
    aeo_status enqueue_on(cudaStream_t s) override {
        cudaStreamCaptureStatus cs;
        CK(cudaStreamIsCapturing(s, &cs));
        if (cs == cudaStreamCaptureStatusActive) return capture_solve(s, false);
        return launch_on(s);
    }
    // everything this handle queued on its own stream precedes what s runs next
    aeo_status order_before(cudaStream_t s) override {
        if (s == st) return AEO_OK;
        if (!ev_own) CK(cudaEventCreateWithFlags(&ev_own, cudaEventDisableTiming));
        CK(cudaEventRecord(ev_own, st));
        CK(cudaStreamWaitEvent(s, ev_own, 0));
        return AEO_OK;
    }
    aeo_status last_stats(aeo_mg_stats* o) override {
        CK(cudaDeviceSynchronize());
        return stats_out(o, false);
    }

    aeo_status solve(const double* bin, double* xout, bool device, aeo_mg_stats* o) override {
        if (!g_solve)
            if (aeo_status s = build_solve()) return s;
        CK(cudaMemcpyAsync(b, bin, sizeof(double) * n, device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st));
        CK(cudaGraphLaunch(g_solve, st));
        CK(cudaMemcpyAsync(xout, x, sizeof(double) * n, device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, st));
        return stats_out(o, false);
    }

    aeo_status build_cycles() {
        if (nl == 1) {
            fail("standalone multigrid cycles need at least two levels");
            return AEO_ERR_ARGUMENT;
        }
        CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed));
        aeo_status s = [&]() -> aeo_status {
            cudaGraphConditionalHandle hdl;
            if (aeo_status q = make_handle(&hdl)) return q;
            pcg_mean_kernel<<<RED_BLOCKS, TPB, 0, st>>>(b, n, S, part, 0);
            CKL();
            // b0 = b - mean(b) (_load_rhs!), phi0 = 0
            mg_load_kernel<R><<<RED_BLOCKS, TPB, 0, st>>>(L[0], b, &S->mb);
            CKL();
            mg_bnorm_kernel<R><<<RED_BLOCKS, TPB, 0, st>>>(L[0], S, part);
            CKL();
            pcg_cond_kernel<<<1, 1, 0, st>>>(S, hdl, 1);
            CKL();
            if (aeo_status q = capture_while(hdl, [&](cudaStream_t sb) -> aeo_status {
                    if (aeo_status q2 = launch_vcycle(sb, nullptr, false, &S->done)) return q2;
                    mg_resnorm_kernel<R><<<row_blocks(cfg.ny * cfg.nz), dim3(RB_X, RB_Y), 0, sb>>>(L[0], bc, S, part);
                    CKL();
                    pcg_cond_kernel<<<1, 1, 0, sb>>>(S, hdl, 1);
                    CKL();
                    return AEO_OK;
                }))
                return q;
            mg_store_kernel<R><<<RED_BLOCKS, TPB, 0, st>>>(L[0], x);
            CKL();
            pcg_mean_kernel<<<RED_BLOCKS, TPB, 0, st>>>(x, n, S, part, 1);
            CKL();
            shift_kernel<<<RED_BLOCKS, TPB, 0, st>>>(x, n, S);
            CKL();
            return AEO_OK;
        }();
        return end_capture(&g_cycles, s);
    }

    aeo_status cycles(const double* bin, double* xout, aeo_mg_stats* o) override {
        if (!g_cycles)
            if (aeo_status s = build_cycles()) return s;
        CK(cudaMemcpyAsync(b, bin, sizeof(double) * n, cudaMemcpyHostToDevice, st));
        CK(cudaGraphLaunch(g_cycles, st));
        CK(cudaMemcpyAsync(xout, x, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
        return stats_out(o, true);
    }

    aeo_status apply(const double* xin, double* out) override {
        CK(cudaMemcpyAsync(p, xin, sizeof(double) * n, cudaMemcpyHostToDevice, st));
        if (aeo_status s = launch_apply(st, p, Ap, 1)) return s;
        CK(cudaMemcpyAsync(out, Ap, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        return AEO_OK;
    }

    // z = M r: r loaded with its mean removed (as in the solve), one cycle,
    // then z - mean(z) (the deflated preconditioner of the reference)
    aeo_status precondition(const double* rin, double* zout) override {
        if (cfg.precond == AEO_PC_LEARNED) {
            CK(cudaMemcpyAsync(r, rin, sizeof(double) * n, cudaMemcpyHostToDevice, st));
            if (aeo_status s = aeo_unet_forward_on(net, r, st)) return s;
            std::vector<float> hz((size_t)n);
            CK(cudaMemcpyAsync(hz.data(), aeo_unet_output(net), sizeof(float) * n, cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            for (int q = 0; q < n; ++q) zout[q] = double(hz[q]);
        } else if (cfg.precond == AEO_PC_JACOBI) {
            for (int q = 0; q < n; ++q) zout[q] = rin[q] * h_invd[q];
        } else if (cfg.precond != AEO_PC_VCYCLE) {
            std::memcpy(zout, rin, sizeof(double) * n);
        } else {
            CK(cudaMemcpyAsync(b, rin, sizeof(double) * n, cudaMemcpyHostToDevice, st));
            pcg_mean_kernel<<<RED_BLOCKS, TPB, 0, st>>>(b, n, S, part, 0);
            CKL();
            pcg_init_kernel<<<RED_BLOCKS, TPB, 0, st>>>(b, r, x, n, S, part);
            CKL();
            if (aeo_status s = launch_vcycle(st, r, true, dzero)) return s;
            std::vector<R> hz((size_t)n);
            CK(cudaMemcpyAsync(hz.data(), L[0].phi, sizeof(R) * n, cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            for (int q = 0; q < n; ++q) zout[q] = double(hz[q]);
        }
        double s = 0;
        for (int q = 0; q < n; ++q) s += zout[q];
        s /= double(n);
        for (int q = 0; q < n; ++q) zout[q] -= s;
        return AEO_OK;
    }

    void drop_graphs() {
        if (g_solve) cudaGraphExecDestroy(g_solve);
        if (g_harvest) cudaGraphExecDestroy(g_harvest);
        g_solve = g_harvest = nullptr;
    }

    aeo_status set_learned(aeo_unet* nn, double stag) override {
        if (nn && aeo_unet_cells(nn) != (long long)n) {
            fail("set_learned: the network's grid differs from the solver's");
            return AEO_ERR_ARGUMENT;
        }
        CK(cudaStreamSynchronize(st));
        drop_graphs();
        net = nn;
        cfg.precond = nn ? AEO_PC_LEARNED : AEO_PC_VCYCLE;
        PcgState h0{};
        CK(cudaMemcpy(&h0, S, sizeof(PcgState), cudaMemcpyDeviceToHost));
        h0.learned_init = nn ? 1 : 0;
        h0.stag = stag;
        h0.flexible = nn ? 1 : cfg.flexible;
        CK(cudaMemcpy(S, &h0, sizeof(PcgState), cudaMemcpyHostToDevice));
        return AEO_OK;
    }

    aeo_status harvest(const double* bin, double* xout, aeo_mg_stats* o, double* rh, double* xh, int cap,
                       int* count) override {
        if (cap != hist_cap) {
            CK(cudaStreamSynchronize(st));
            if (hist_x) cudaFree(hist_x);
            if (hist_r) cudaFree(hist_r);
            hist_x = hist_r = nullptr;
            hist_cap = 0;
            if (g_harvest) cudaGraphExecDestroy(g_harvest);
            g_harvest = nullptr;
            CK(cudaMalloc(&hist_x, sizeof(double) * (size_t)cap * n));
            CK(cudaMalloc(&hist_r, sizeof(double) * (size_t)cap * n));
            hist_cap = cap;
        }
        if (!g_harvest)
            if (aeo_status s = build_solve(true)) return s;
        CK(cudaMemcpyAsync(b, bin, sizeof(double) * n, cudaMemcpyHostToDevice, st));
        CK(cudaGraphLaunch(g_harvest, st));
        CK(cudaMemcpyAsync(xout, x, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
        if (aeo_status s = stats_out(o, false)) return s;
        const int c = hS->iters + 1 < cap ? hS->iters + 1 : cap;
        CK(cudaMemcpyAsync(rh, hist_r, sizeof(double) * (size_t)c * n, cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(xh, hist_x, sizeof(double) * (size_t)c * n, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        *count = c;
        return AEO_OK;
    }

    aeo_status profile(int what, int reps, double* ms) override {
        if (what == 0 && !g_solve) {
            fail("profile: no solve has run yet");
            return AEO_ERR_STATE;
        }
        cudaEvent_t e0, e1;
        CK(cudaEventCreate(&e0));
        CK(cudaEventCreate(&e1));
        auto run = [&]() -> aeo_status {
            switch (what) {
            case 0: CK(cudaGraphLaunch(g_solve, st)); return AEO_OK;
            case 1: {
                Level<R>& F = L[0];
                if (F.nx % 2) { fail("profile: odd finest nx"); return AEO_ERR_ARGUMENT; }
                return launch_rbgs(st, F, 0, dzero);
            }
            case 2: return launch_apply(st, p, Ap, 1);
            case 3: return launch_vcycle(st, r, true, dzero);
            case 4: return launch_coarsest(st, L[nl - 1], nl == 1 ? r : nullptr, dzero);
            case 5: {
                if (nl < 2) { fail("profile: one level, no restriction"); return AEO_ERR_ARGUMENT; }
                if (aeo_status q = launch_residual(st, L[0], dzero)) return q;
                AEO_PDL_LAUNCH((mg_restrict_kernel<R>), restrict_grid(L[1]), dim3(RB_X, RB_Y), 0, st, L[0], L[1], part, &S->counter,
                                                                                      dzero);
                CKL();
                return AEO_OK;
            }
            case 6: {
                if (nl < 2) { fail("profile: one level, no smoothing sweep"); return AEO_ERR_ARGUMENT; }
                if (aeo_status q = launch_rbgs(st, L[0], 0, dzero)) return q;
                return launch_rbgs(st, L[0], 1, dzero);
            }
            default: fail("profile: unknown part"); return AEO_ERR_ARGUMENT;
            }
        };
        for (int w = 0; w < 3; ++w)
            if (aeo_status s = run()) return s;
        CK(cudaEventRecord(e0, st));
        for (int i = 0; i < reps; ++i)
            if (aeo_status s = run()) return s;
        CK(cudaEventRecord(e1, st));
        CK(cudaEventSynchronize(e1));
        float t = 0;
        CK(cudaEventElapsedTime(&t, e0, e1));
        *ms = double(t) / reps;
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        return AEO_OK;
    }
};

std::string g_mg_error;

}  // namespace

struct aeo_mg {
    MgBase* core;
};

extern "C" {

aeo_status aeo_mg_create(const aeo_mg_config* c, const double* cx, const double* cy, const double* cz, aeo_mg** out) {
    if (!out) { g_mg_error = "out is NULL"; return AEO_ERR_ARGUMENT; }
    *out = nullptr;
    if (!c) { g_mg_error = "config is NULL"; return AEO_ERR_ARGUMENT; }
    if (c->nx < 1 || c->ny < 1 || c->nz < 1) { g_mg_error = "grid dimensions must be positive"; return AEO_ERR_ARGUMENT; }
    if (!(c->dx > 0) || !(c->dy > 0) || !(c->dz > 0)) { g_mg_error = "spacings must be positive"; return AEO_ERR_ARGUMENT; }
    for (int b : {c->bc_x, c->bc_y, c->bc_z})
        if (b != AEO_MG_PERIODIC && b != AEO_MG_NEUMANN) {
            g_mg_error = "unsupported BC (use periodic or Neumann, src/Multigrid.jl:62-66)";
            return AEO_ERR_ARGUMENT;
        }
    if ((cx == nullptr) != (cy == nullptr) || (cx == nullptr) != (cz == nullptr)) {
        g_mg_error = "give all three face coefficient arrays or none";
        return AEO_ERR_ARGUMENT;
    }
    if (c->precision != AEO_PREC_FP64 && c->precision != AEO_PREC_FP32_MIXED) { g_mg_error = "unknown precision"; return AEO_ERR_ARGUMENT; }
    if (c->precond != AEO_PC_IDENTITY && c->precond != AEO_PC_VCYCLE && c->precond != AEO_PC_JACOBI) {
        g_mg_error = "unknown preconditioner";
        return AEO_ERR_ARGUMENT;
    }
    if (!(c->tol >= 0) || c->maxit < 0 || c->nu1 < 1 || c->nu2 < 0 || c->coarse_sweeps < 0 || c->min_size < 1) {
        g_mg_error = "invalid tol / maxit / sweep counts (nu1 >= 1)";
        return AEO_ERR_ARGUMENT;
    }
    long long ncell = (long long)(c->nx + 1) * (c->ny + 1) * (c->nz + 1);
    if (ncell >= (1LL << 30)) { g_mg_error = "grid at or above 2^30 cells"; return AEO_ERR_ARGUMENT; }
    if (cudaSetDevice(c->device) != cudaSuccess) { g_mg_error = "cudaSetDevice failed"; return AEO_ERR_CUDA; }
    MgBase* m = nullptr;
    if (c->precision == AEO_PREC_FP64) m = new (std::nothrow) Mg<double>();
    else m = new (std::nothrow) Mg<float>();
    if (!m) { g_mg_error = "out of host memory"; return AEO_ERR_CUDA; }
    m->cfg = *c;
    if (aeo_status s = m->init(cx, cy, cz)) {
        g_mg_error = m->err;
        delete m;
        return s;
    }
    aeo_mg* h = new (std::nothrow) aeo_mg;
    if (!h) { delete m; g_mg_error = "out of host memory"; return AEO_ERR_CUDA; }
    h->core = m;
    *out = h;
    return AEO_OK;
}

aeo_status aeo_mg_destroy(aeo_mg* h) {
    if (!h) return AEO_OK;
    cudaSetDevice(h->core->cfg.device);
    delete h->core;
    delete h;
    return AEO_OK;
}

#define MG_ENTER(h)                                                    \
    if (!h) return AEO_ERR_ARGUMENT;                                   \
    if (cudaSetDevice(h->core->cfg.device) != cudaSuccess) {           \
        h->core->fail("cudaSetDevice failed");                         \
        return AEO_ERR_CUDA;                                           \
    }

aeo_status aeo_mg_levels(aeo_mg* h, int32_t* nlevels, int32_t* dims) {
    MG_ENTER(h);
    if (nlevels) *nlevels = h->core->nlevels();
    if (dims)
        for (int l = 0; l < h->core->nlevels(); ++l) h->core->level_dims(l, dims + 3 * l);
    return AEO_OK;
}

aeo_status aeo_mg_solve(aeo_mg* h, const double* b, double* x, aeo_mg_stats* st) {
    MG_ENTER(h);
    if (!b || !x) { h->core->fail("b and x must not be NULL"); return AEO_ERR_ARGUMENT; }
    return h->core->solve(b, x, false, st);
}

aeo_status aeo_mg_solve_device(aeo_mg* h, const double* b, double* x, aeo_mg_stats* st) {
    MG_ENTER(h);
    if (!b || !x) { h->core->fail("b and x must not be NULL"); return AEO_ERR_ARGUMENT; }
    return h->core->solve(b, x, true, st);
}

aeo_status aeo_mg_vcycle_solve(aeo_mg* h, const double* b, double* x, aeo_mg_stats* st) {
    MG_ENTER(h);
    if (!b || !x) { h->core->fail("b and x must not be NULL"); return AEO_ERR_ARGUMENT; }
    return h->core->cycles(b, x, st);
}

aeo_status aeo_mg_apply(aeo_mg* h, const double* x, double* out) {
    MG_ENTER(h);
    if (!x || !out) { h->core->fail("x and out must not be NULL"); return AEO_ERR_ARGUMENT; }
    return h->core->apply(x, out);
}

aeo_status aeo_mg_precondition(aeo_mg* h, const double* r, double* z) {
    MG_ENTER(h);
    if (!r || !z) { h->core->fail("r and z must not be NULL"); return AEO_ERR_ARGUMENT; }
    return h->core->precondition(r, z);
}

aeo_status aeo_mg_profile(aeo_mg* h, int32_t what, int32_t reps, double* ms) {
    MG_ENTER(h);
    if (!ms || reps < 1) { h->core->fail("profile: ms NULL or reps < 1"); return AEO_ERR_ARGUMENT; }
    return h->core->profile(what, reps, ms);
}

int32_t aeo_mg_launches_per_iteration(const aeo_mg* h) { return h ? h->core->launches_per_iteration() : 0; }

aeo_status aeo_mg_set_learned(aeo_mg* h, aeo_unet* net, double stagnation) {
    MG_ENTER(h);
    if (net && !(stagnation > 0 && stagnation <= 1)) {
        h->core->fail("set_learned: the stagnation ratio lies in (0, 1]");
        return AEO_ERR_ARGUMENT;
    }
    return h->core->set_learned(net, stagnation);
}

aeo_status aeo_mg_solve_harvest(aeo_mg* h, const double* b, double* x, aeo_mg_stats* st, double* r_hist,
                                double* x_hist, int32_t cap, int32_t* count) {
    MG_ENTER(h);
    if (!b || !x || !r_hist || !x_hist || !count || cap < 1) {
        h->core->fail("solve_harvest: NULL array or cap < 1");
        return AEO_ERR_ARGUMENT;
    }
    return h->core->harvest(b, x, st, r_hist, x_hist, cap, count);
}

const char* aeo_mg_last_error(const aeo_mg* h) { return h ? h->core->err.c_str() : g_mg_error.c_str(); }

}  // extern "C"

// ---- internal (C++ linkage) entry points of the stepping engine (aeolus_b200.cu)
aeo_status aeo_mg_buffers(aeo_mg* h, double** b, double** x) {
    if (!h || !b || !x) return AEO_ERR_ARGUMENT;
    h->core->buffers(b, x);
    return AEO_OK;
}
aeo_status aeo_mg_launch(aeo_mg* h, cudaStream_t s) {
    if (!h) return AEO_ERR_ARGUMENT;
    return h->core->launch_on(s);
}
aeo_status aeo_mg_read_stats(aeo_mg* h, aeo_mg_stats* o) {
    if (!h || !o) return AEO_ERR_ARGUMENT;
    return h->core->last_stats(o);
}
aeo_status aeo_mg_enqueue(aeo_mg* h, cudaStream_t s) {
    if (!h) return AEO_ERR_ARGUMENT;
    return h->core->enqueue_on(s);
}
aeo_status aeo_mg_order_before(aeo_mg* h, cudaStream_t s) {
    if (!h) return AEO_ERR_ARGUMENT;
    return h->core->order_before(s);
}
int aeo_mg_launches_per_solve(const aeo_mg* h, int iterations) {
    return h ? h->core->launches_per_solve(iterations) : 0;
}
