// aeo_noalloc.cu -- a column pressure solve that allocates no device memory.
//
// aeo_pressure_solve_column_noalloc runs the same kernels as the column
// pressure solve of a domain handle (r2c along x, DFT along y, FP64 Thomas
// per horizontal wavenumber with the mean mode integrated, inverse
// transforms) but takes every input and output as a caller-owned device
// pointer and keeps all of its scratch -- twiddles, eigenvalues, the column
// coefficients and the spectrum -- in one file-scope static device array
// of AEO_NOALLOC_SCRATCH_BYTES.  It is for callers that cannot call
// cudaMalloc: a host runtime whose device memory belongs to its own pool or
// budget (a Julia or Python array allocator that must own every byte), an
// embedding application that pre-reserves all device memory at start-up, or
// a time-stepping loop that must not pay cudaMalloc's implicit device
// synchronisation.  Each device that loads the library holds the static
// array until the process exits.
#include <cuda_runtime.h>

#include <string>

#include "../../include/aeolus_b200.h"
#include "aeo_common.cuh"
#include "aeo_fft.cuh"

#define AEO_NOALLOC_SCRATCH_BYTES (32u << 20)   // 32 MiB per device
static __device__ __align__(256) unsigned char aeo_noalloc_scratch[AEO_NOALLOC_SCRATCH_BYTES];

// defined in aeolus_b200.cu: the message aeo_last_error(NULL) returns
void aeo_set_global_error(const std::string& m);

namespace {

// The device address of the static scratch on the current device.  In host
// code the symbol is only a host-side stand-in, never a device address:
// kernels get this pointer instead.  It is looked up on every call (the
// lookup allocates nothing), so a pointer never outlives the context it
// belongs to: after a cudaDeviceReset the next call finds the array of the
// new context.
aeo_status scratch_address(unsigned char** out) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, aeo_noalloc_scratch);
    if (e != cudaSuccess || !p) {
        aeo_set_global_error(std::string("cudaGetSymbolAddress(aeo_noalloc_scratch): ") + cudaGetErrorString(e));
        return AEO_ERR_CUDA;
    }
    *out = reinterpret_cast<unsigned char*>(p);
    return AEO_OK;
}

size_t up256(size_t b) { return (b + 255) & ~(size_t)255; }
bool pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

__global__ void noalloc_tables_kernel(cplx<double>* tw, int NT, double* kx2, int nx, double* ky2, int ny,
                                      double dx, double dy) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < NT) {
        double s, c;
        sincospi(-2.0 * (double)t / (double)NT, &s, &c);
        tw[t] = cmk<double>(c, s);
    }
    if (t <= nx / 2) {
        int m = t < nx - t ? t : nx - t;
        double s = sinpi((double)m / nx);
        kx2[t] = 4 / (dx * dx) * (s * s);
    }
    if (t < ny) {
        int m = t < ny - t ? t : ny - t;
        double s = sinpi((double)m / ny);
        ky2[t] = 4 / (dy * dy) * (s * s);
    }
}

}  // namespace

extern "C" aeo_status aeo_pressure_solve_column_noalloc(int32_t nx, int32_t ny, int32_t nz, double lx, double ly,
                                                        const double* lower, const double* upper,
                                                        const double* hweight, const double* measure,
                                                        const double* inv_coupling, const double* gauge,
                                                        const double* src, double* phi, void* stream) {
    if (!lower || !upper || !hweight || !measure || !inv_coupling || !gauge || !src || !phi) {
        aeo_set_global_error("pressure_solve_column_noalloc: NULL argument");
        return AEO_ERR_ARGUMENT;
    }
    if (!pow2(nx) || !pow2(ny) || nx < 4 || ny < 4 || nx / 2 > 2048 || ny > 2048 || nz < 1 || nz > AEO_COLUMN_NZ_MAX) {
        aeo_set_global_error("pressure_solve_column_noalloc: nx, ny must be powers of two (4 <= nx <= 4096, "
                             "4 <= ny <= 2048) and 1 <= nz <= " + std::to_string(AEO_COLUMN_NZ_MAX));
        return AEO_ERR_ARGUMENT;
    }
    if (lower[0] != 0.0 || upper[nz - 1] != 0.0 || !(lx > 0) || !(ly > 0)) {
        aeo_set_global_error("pressure_solve_column_noalloc: the bottom and top faces carry no flux "
                             "(lower[0] = upper[nz-1] = 0) and lx, ly must be positive");
        return AEO_ERR_ARGUMENT;
    }
    const int Mh = nx / 2 + 1;
    int NT = 1;
    while (NT < (nx > ny ? nx : ny)) NT <<= 1;
    const size_t b_tw = up256(sizeof(cplx<double>) * (size_t)NT);
    const size_t b_kx = up256(sizeof(double) * (size_t)Mh);
    const size_t b_ky = up256(sizeof(double) * (size_t)ny);
    const size_t b_cf = up256(sizeof(double) * 6 * (size_t)(nz + 1));
    const size_t b_sp = up256(sizeof(cplx<double>) * (size_t)Mh * ny * nz);
    const size_t need = b_tw + b_kx + b_ky + b_cf + b_sp;
    if (need > AEO_NOALLOC_SCRATCH_BYTES) {
        aeo_set_global_error("pressure_solve_column_noalloc: the grid needs " + std::to_string(need) +
                             " bytes of scratch, more than the fixed " +
                             std::to_string((size_t)AEO_NOALLOC_SCRATCH_BYTES) +
                             " (32 MiB: (nx/2+1)*ny*nz*16 bytes plus tables must fit)");
        return AEO_ERR_ARGUMENT;
    }
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    // the call copies pageable host arrays and synchronises the stream, which
    // would invalidate a capture in progress: refuse a capturing stream
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    cudaError_t e = cudaStreamIsCapturing(st, &cap);
    if (e != cudaSuccess) {
        aeo_set_global_error(std::string("pressure_solve_column_noalloc: cudaStreamIsCapturing: ") + cudaGetErrorString(e));
        return AEO_ERR_CUDA;
    }
    if (cap != cudaStreamCaptureStatusNone) {
        aeo_set_global_error("pressure_solve_column_noalloc: the stream is capturing a graph; call it outside a capture");
        return AEO_ERR_ARGUMENT;
    }
    double ms = 0, gs = 0;
    for (int k = 0; k < nz; ++k) { ms += measure[k]; gs += gauge[k]; }
    if (!(ms != 0.0) || !(gs != 0.0)) {
        aeo_set_global_error("pressure_solve_column_noalloc: the sums of measure and of gauge must be nonzero "
                             "(the mean mode divides by them)");
        return AEO_ERR_ARGUMENT;
    }
    unsigned char* base = nullptr;
    if (aeo_status sa = scratch_address(&base)) return sa;

    cplx<double>* tw = reinterpret_cast<cplx<double>*>(base);
    double* kx2 = reinterpret_cast<double*>(base + b_tw);
    double* ky2 = reinterpret_cast<double*>(base + b_tw + b_kx);
    double* cf = reinterpret_cast<double*>(base + b_tw + b_kx + b_ky);
    cplx<double>* S = reinterpret_cast<cplx<double>*>(base + b_tw + b_kx + b_ky + b_cf);

    // every scratch region below is fully written before it is read, so the
    // previous call's contents never leak into this one
    const int L = nz + 1;
    const double* host[6] = {lower, upper, hweight, measure, inv_coupling, gauge};
    for (int a = 0; a < 6; ++a) {
        size_t n = (a == 4) ? (size_t)(nz + 1) : (size_t)nz;
        e = cudaMemcpyAsync(cf + (size_t)a * L, host[a], n * sizeof(double), cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) {
            aeo_set_global_error(std::string("pressure_solve_column_noalloc: cudaMemcpyAsync: ") + cudaGetErrorString(e));
            return AEO_ERR_CUDA;
        }
    }
    Geo g{};
    g.nx = nx; g.ny = ny; g.nz = nz;
    g.nin = (long long)nx * ny * nz;
    const double dx = lx / nx, dy = ly / ny;
    int tmax = NT > Mh ? NT : Mh;
    if (ny > tmax) tmax = ny;
    noalloc_tables_kernel<<<(tmax + 255) / 256, 256, 0, st>>>(tw, NT, kx2, nx, ky2, ny, dx, dy);

    ColumnCoef cc{};
    cc.lower = cf; cc.upper = cf + L; cc.hw = cf + 2 * L; cc.meas = cf + 3 * L; cc.iota = cf + 4 * L;
    cc.gauge = cf + 5 * L; cc.meas_sum = ms; cc.gauge_sum = gs; cc.kx2 = kx2; cc.ky2 = ky2;

    const int M = nx / 2;
    const int rows = 2048 / M > 1 ? 2048 / M : 1;
    const int tpx = 2048 / ny > 16 ? 16 : (2048 / ny > 1 ? 2048 / ny : 1);
    unsigned gx = (unsigned)(((long long)ny * nz + rows - 1) / rows);
    size_t smx = (size_t)rows * xrow(M) * sizeof(cplx<double>);
    dim3 gy((Mh + tpx - 1) / tpx, nz);
    size_t smy = (size_t)tpx * ny * sizeof(cplx<double>);
    size_t smt = thomas_smem(g, false);
    if (smt > 48 * 1024) {
        e = cudaFuncSetAttribute(thomas_kernel<double, false, double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smt);
        if (e != cudaSuccess) {
            aeo_set_global_error(std::string("pressure_solve_column_noalloc: ") + cudaGetErrorString(e));
            return AEO_ERR_CUDA;
        }
    }
    src_fftx_kernel<double><<<gx, FFT_THREADS(double), smx, st>>>(g, src, S, tw, NT, rows);
    ffty_kernel<double, 0><<<gy, FFT_THREADS(double), smy, st>>>(g, S, tw, NT, tpx);
    thomas_kernel<double, false, double><<<thomas_blocks(g), 32, smt, st>>>(g, S, S, nullptr, cc);
    ffty_kernel<double, 1><<<gy, FFT_THREADS(double), smy, st>>>(g, S, tw, NT, tpx);
    ifftx_kernel<double><<<gx, FFT_THREADS(double), smx, st>>>(g, S, phi, tw, NT, rows, 1.0 / ((double)nx * ny));
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        aeo_set_global_error(std::string("pressure_solve_column_noalloc: ") + cudaGetErrorString(e));
        return AEO_ERR_CUDA;
    }
    return AEO_OK;
}
