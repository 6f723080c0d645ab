// lbf_flux_sums_noalloc: the pore-measure reduction of lbf_flux_sums over
// arrays the caller already holds on the device, without allocating device
// memory.
//
// Who needs it: callers that must not call cudaMalloc -- code running while a
// memory pool is frozen or near exhaustion, allocators that forbid foreign
// allocations on their device, or embedded hosts that own every device byte.
// They pass device pointers for the inputs and for the 9-double output; the
// per-tile partial sums go to a fixed scratch array compiled into this
// library (g_flux_scratch, kMaxTiles * 9 doubles = 1,179,648 bytes).  The
// array comes into device memory with this library's module: under CUDA's
// default lazy module loading that happens at the first call on a device
// (eager loading: when the library's context is set up), and the device
// then holds it until the process exits.
//
// Limits and rules:
//  - at most kMaxNodes = kTile * kMaxTiles = 16,777,216 nodes per call;
//    larger n is rejected with LBF_EINVAL before any GPU work;
//  - the first call on a device looks up the scratch array's device address
//    (cudaGetSymbolAddress) with that device current, which also loads the
//    module and so needs the 1.2 MB once; make that first call (n = 0 is
//    enough) while device memory is still free and before any stream
//    capture;
//  - all calls share the one scratch array, so calls whose GPU work overlaps
//    (different streams or threads at the same time) race; serialise them.
//    Every tile's partial is rewritten by each call before it is read, so
//    nothing has to start at zero.
#include "../../include/lbflow.h"
#include "internal.h"
#include "reduce.cuh"

#include <mutex>
#include <string>

namespace {

constexpr uint32_t kTile = 1024;           // nodes reduced by one pass-1 block
constexpr uint32_t kMaxTiles = 16384;
constexpr uint64_t kMaxNodes = (uint64_t)kTile * kMaxTiles;
constexpr int kThreads = 256;
constexpr int K = lbf::FluxFn::K;

static __device__ __align__(256) double g_flux_scratch[kMaxTiles * K];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
double* g_scratch_ptr[kMaxDevices] = {};

// Block-wide sum of K values; thread 0 receives the totals.
__device__ void block_sum(double (&acc)[K], double (&sm)[K][kThreads / 32])
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        double v = acc[k];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
        if (lane == 0) sm[k][warp] = v;
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) {
            double v = lane < kThreads / 32 ? sm[k][lane] : 0.0;
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
            acc[k] = v;
        }
    }
}

// Pass 1: one block per tile of kTile nodes writes its K partial sums.
__global__ void __launch_bounds__(kThreads) flux_tiles(const lbf::FluxFn fn, uint32_t n, double* __restrict__ scratch)
{
    __shared__ double sm[K][kThreads / 32];
    double acc[K];
#pragma unroll
    for (int k = 0; k < K; ++k) acc[k] = 0.0;
    const uint32_t base = blockIdx.x * kTile;
    for (uint32_t j = threadIdx.x; j < kTile; j += kThreads) {
        const uint32_t i = base + j;
        if (i < n) fn(i, acc);
    }
    block_sum(acc, sm);
    if (threadIdx.x == 0)
#pragma unroll
        for (int k = 0; k < K; ++k) scratch[(size_t)blockIdx.x * K + k] = acc[k];
}

// Pass 2: one block sums the tile partials into the caller's output.
__global__ void __launch_bounds__(kThreads) flux_final(const double* __restrict__ scratch, uint32_t tiles,
                                                       double* __restrict__ out)
{
    __shared__ double sm[K][kThreads / 32];
    double acc[K];
#pragma unroll
    for (int k = 0; k < K; ++k) acc[k] = 0.0;
    for (uint32_t t = threadIdx.x; t < tiles; t += kThreads)
#pragma unroll
        for (int k = 0; k < K; ++k) acc[k] += scratch[(size_t)t * K + k];
    block_sum(acc, sm);
    if (threadIdx.x == 0)
#pragma unroll
        for (int k = 0; k < K; ++k) out[k] = acc[k];
}

int scratch_for_current_device(double** ptr)
{
    int dev = 0;
    cudaError_t r = cudaGetDevice(&dev);
    if (r != cudaSuccess) {
        lbf::set_global_error(std::string("cudaGetDevice: ") + cudaGetErrorString(r));
        return LBF_ECUDA;
    }
    if (dev < 0 || dev >= kMaxDevices) {
        lbf::set_global_error("lbf_flux_sums_noalloc: device ordinal out of range");
        return LBF_EINVAL;
    }
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratch_ptr[dev]) {
        void* p = nullptr;
        r = cudaGetSymbolAddress(&p, g_flux_scratch);
        if (r != cudaSuccess) {
            lbf::set_global_error(std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(r));
            return LBF_ECUDA;
        }
        g_scratch_ptr[dev] = static_cast<double*>(p);
    }
    *ptr = g_scratch_ptr[dev];
    return LBF_OK;
}

}  // namespace

extern "C" int lbf_flux_sums_noalloc(const double* u, const double* rho0, const double* rho1,
                                     uint32_t n, uint32_t stride, double* out, void* stream)
{
    if (!u || !rho0 || !out) {
        lbf::set_global_error("lbf_flux_sums_noalloc: u, rho0 and out must be device pointers");
        return LBF_EINVAL;
    }
    if ((uint64_t)n > kMaxNodes) {
        lbf::set_global_error("lbf_flux_sums_noalloc: n = " + std::to_string(n) +
                              " exceeds the fixed scratch capacity of " + std::to_string(kMaxNodes) + " nodes");
        return LBF_EINVAL;
    }
    if (stride < n) {
        lbf::set_global_error("lbf_flux_sums_noalloc: stride must be >= n");
        return LBF_EINVAL;
    }
    double* scratch = nullptr;
    const int rc = scratch_for_current_device(&scratch);
    if (rc != LBF_OK) return rc;
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    const uint32_t tiles = n ? (n + kTile - 1) / kTile : 1;
    lbf::FluxFn fn{u, rho0, rho1, stride};
    flux_tiles<<<tiles, kThreads, 0, s>>>(fn, n, scratch);
    flux_final<<<1, kThreads, 0, s>>>(scratch, tiles, out);
    const cudaError_t r = cudaGetLastError();
    if (r != cudaSuccess) {
        lbf::set_global_error(std::string("lbf_flux_sums_noalloc: ") + cudaGetErrorString(r));
        return LBF_ECUDA;
    }
    return LBF_OK;
}
