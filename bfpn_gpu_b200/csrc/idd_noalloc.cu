// Integrated depth dose of caller-owned device state with no device
// allocation (bfpn_idd_noalloc in include/bfpn_capi.h).
//
// Who needs it: a caller that owns every byte of device memory itself and may
// not have a library allocate behind its back -- a serving process that
// reserves the GPU up front for its own pool, or a framework whose caching
// allocator holds the state tensors and must stay the only allocator on the
// device -- and a caller that cannot afford cudaMalloc/cudaFree in the middle
// of its pipeline, since both synchronise the device.  Such a caller cannot
// create a solver context (bfpn_create allocates all of its buffers), so this
// entry point takes the four state arrays, the dose weights and the output as
// device pointers and keeps its only working memory, the per-block partial
// sums, in a fixed file-scope device array.
//
// The work is the same reduction bfpn_idd does (computeIntegratedDepthDose +
// computeScalarDoseProxy, bfpm_solver.cu:3473-3502, 3418-3444 of the
// reference), done in one launch: every block reduces its lanes to a
// (dose, psi^2) pair in the scratch, and the last block to finish -- found
// with a ticket counter -- adds the pairs in block order, so the result does
// not depend on which block finishes last.

#include "../../include/bfpn_capi.h"
#include "common.cuh"
#include "tables.hpp"

#include <string>

using namespace bfpn;

namespace {

constexpr int kThreads = 256;
constexpr int kLanesPerThread = 4;
constexpr int kLanesPerBlock = kThreads * kLanesPerThread;  // 1024
// Largest grid the scratch holds partials for, and so the largest
// transverse-angular plane (nyz * NA) one call accepts: 4096 * 1024 lanes.
constexpr int kMaxBlocks = 4096;
constexpr long long kMaxLanes = static_cast<long long>(kMaxBlocks) * kLanesPerBlock;
// Scratch layout: bytes [0, 256) hold the ticket counter (an unsigned int
// that must be zero when a launch starts; every call clears it on its stream
// first), bytes [256, 256 + 16 * kMaxBlocks) the (dose, psi^2) double pair of
// each block.  65,792 bytes in all.
constexpr size_t kHeaderBytes = 256;
constexpr size_t kScratchBytes = kHeaderBytes + 2 * sizeof(double) * kMaxBlocks;

}  // namespace

static __device__ __align__(256) unsigned char g_idd_scratch[kScratchBytes];

namespace {

template <typename T>
__global__ void __launch_bounds__(kThreads) idd_noalloc_kernel(const T* __restrict__ F0, const T* __restrict__ f0,
                                                               const T* __restrict__ F1, const T* __restrict__ f1,
                                                               const double* __restrict__ dc, int Ng, long long lanes,
                                                               int NA, int Ny, int Nz, int trap, double idd_scale,
                                                               double proxy_scale, unsigned char* scratch,
                                                               double* out) {
    unsigned int* ticket = reinterpret_cast<unsigned int*>(scratch);
    double* part = reinterpret_cast<double*>(scratch + kHeaderBytes);
    double acc = 0.0, accp = 0.0;
    for (int k = 0; k < kLanesPerThread; ++k) {
        const long long lane = static_cast<long long>(blockIdx.x) * kLanesPerBlock + k * kThreads + threadIdx.x;
        if (lane >= lanes) break;
        double w = 1.0;
        if (trap) {
            const int pos = static_cast<int>(lane / NA), iy = pos % (Ny + 1), iz = pos / (Ny + 1);
            if (iy == 0 || iy == Ny) w *= 0.5;
            if (iz == 0 || iz == Nz) w *= 0.5;
        }
        double d = 0.0;
        for (int ek = 0; ek < Ng; ++ek) {
            const long long i = ek * lanes + lane;
            const double x = static_cast<double>(F0[i]), y = static_cast<double>(f0[i]);
            d += dc[2 * ek] * x + dc[2 * ek + 1] * y;
            accp += y;
            if (F1) d += dc[2 * ek] * static_cast<double>(F1[i]) + dc[2 * ek + 1] * static_cast<double>(f1[i]);
        }
        acc += w * d;
    }
    __shared__ double red[2][kThreads / 32];
    __shared__ bool last;
    for (int o = 16; o > 0; o >>= 1) {
        acc += __shfl_down_sync(0xffffffffu, acc, o);
        accp += __shfl_down_sync(0xffffffffu, accp, o);
    }
    const int wi = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) { red[0][wi] = acc; red[1][wi] = accp; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0;
        for (int i = 0; i < kThreads / 32; ++i) { a += red[0][i]; b += red[1][i]; }
        part[2 * blockIdx.x] = a;
        part[2 * blockIdx.x + 1] = b;
        __threadfence();  // the pair is visible device-wide before the ticket is taken
        last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    const volatile double* vp = part;
    double a = 0.0, b = 0.0;
    for (int i = threadIdx.x; i < static_cast<int>(gridDim.x); i += kThreads) { a += vp[2 * i]; b += vp[2 * i + 1]; }
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_down_sync(0xffffffffu, a, o);
        b += __shfl_down_sync(0xffffffffu, b, o);
    }
    __syncthreads();
    if (l == 0) { red[0][wi] = a; red[1][wi] = b; }
    __syncthreads();
    if (threadIdx.x == 0) {
        a = 0.0;
        b = 0.0;
        for (int i = 0; i < kThreads / 32; ++i) { a += red[0][i]; b += red[1][i]; }
        out[0] = a * idd_scale;
        out[1] = b * proxy_scale;
    }
}

bfpn_status noalloc_fail(bfpn_status s, const std::string& msg) {
    set_context_free_error(msg);
    return s;
}

// Restores the caller's current device when the call returns.
struct DeviceGuard {
    int prev = -1;
    ~DeviceGuard() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

}  // namespace

extern "C" bfpn_status bfpn_idd_noalloc(const bfpn_grid* grid, int32_t precision, int32_t trapezoidal_yz,
                                        const void* F0, const void* f0, const void* F1, const void* f1,
                                        const double* dose_coef, double* out, int32_t device, void* stream) {
    if (!grid || !F0 || !f0 || !dose_coef || !out)
        return noalloc_fail(BFPN_INVALID_ARG, "bfpn_idd_noalloc: null grid, state, dose_coef or out pointer");
    if ((F1 == nullptr) != (f1 == nullptr))
        return noalloc_fail(BFPN_INVALID_ARG, "bfpn_idd_noalloc: give both secondary arrays or neither");
    if (precision != BFPN_PREC_FP64 && precision != BFPN_PREC_MIXED)
        return noalloc_fail(BFPN_INVALID_ARG, "bfpn_idd_noalloc: unknown precision");
    const bfpn_grid& g = *grid;
    if (g.Ny <= 0 || g.Nz <= 0 || g.Ng <= 0 || g.Nmu <= 0 || g.Nom <= 0 || !(g.Ly > 0) || !(g.Lz > 0) ||
        !(g.Lu > 0) || !(g.Lv > 0) || !(g.Lg > 0))
        return noalloc_fail(BFPN_INVALID_ARG, "bfpn_idd_noalloc: grid sizes and lengths must be positive");
    const long long nyz = static_cast<long long>(g.Ny + 1) * (g.Nz + 1);
    const long long NA = static_cast<long long>(g.Nmu) * g.Nom;
    const long long lanes = nyz * NA;
    if (lanes > kMaxLanes)
        return noalloc_fail(BFPN_INVALID_ARG, "bfpn_idd_noalloc: (Ny+1)(Nz+1) Nmu Nom = " + std::to_string(lanes) +
                                                  " exceeds the " + std::to_string(kMaxLanes) +
                                                  " lanes its fixed scratch holds (use bfpn_idd)");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) {
        cudaGetLastError();
        return noalloc_fail(BFPN_NO_DEVICE, "bfpn_idd_noalloc: no CUDA device available");
    }
    if (device < 0 || device >= ndev)
        return noalloc_fail(BFPN_INVALID_ARG, "bfpn_idd_noalloc: device ordinal out of range");

    DeviceGuard guard;
    cudaError_t e = cudaGetDevice(&guard.prev);
    if (e != cudaSuccess) return noalloc_fail(BFPN_CUDA_ERROR, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    e = cudaSetDevice(device);
    if (e != cudaSuccess) return noalloc_fail(BFPN_CUDA_ERROR, std::string("cudaSetDevice: ") + cudaGetErrorString(e));

    // The device address of the scratch (the host-side symbol is not one),
    // with the device current.  It is looked up on every call rather than
    // cached: after a cudaDeviceReset (or any other teardown of the primary
    // context) the module is loaded again and the array may move.  The first
    // call on a device also loads the module there.
    unsigned char* scratch = nullptr;
    {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_idd_scratch);
        if (e != cudaSuccess || !p)
            return noalloc_fail(BFPN_CUDA_ERROR,
                                std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
        scratch = static_cast<unsigned char*>(p);
    }

    const Deltas d = compute_deltas(g);
    const double idd_scale = d.du * d.dv * d.dy * d.dz;
    const int blocks = static_cast<int>((lanes + kLanesPerBlock - 1) / kLanesPerBlock);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    e = cudaMemsetAsync(scratch, 0, sizeof(unsigned int), s);  // the ticket counter starts at zero
    if (e != cudaSuccess) return noalloc_fail(BFPN_CUDA_ERROR, std::string("cudaMemsetAsync: ") + cudaGetErrorString(e));
    const int trap = trapezoidal_yz ? 1 : 0;
    if (precision == BFPN_PREC_FP64)
        idd_noalloc_kernel<double><<<blocks, kThreads, 0, s>>>(
            static_cast<const double*>(F0), static_cast<const double*>(f0), static_cast<const double*>(F1),
            static_cast<const double*>(f1), dose_coef, g.Ng, lanes, static_cast<int>(NA), g.Ny, g.Nz, trap, idd_scale,
            d.dg, scratch, out);
    else
        idd_noalloc_kernel<float><<<blocks, kThreads, 0, s>>>(
            static_cast<const float*>(F0), static_cast<const float*>(f0), static_cast<const float*>(F1),
            static_cast<const float*>(f1), dose_coef, g.Ng, lanes, static_cast<int>(NA), g.Ny, g.Nz, trap, idd_scale,
            d.dg, scratch, out);
    e = cudaGetLastError();
    if (e != cudaSuccess) return noalloc_fail(BFPN_CUDA_ERROR, std::string("idd_noalloc_kernel: ") + cudaGetErrorString(e));
    return BFPN_OK;
}
