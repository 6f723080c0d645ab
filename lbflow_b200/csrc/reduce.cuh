// Deterministic FP64 reductions over the fluid nodes.
//
// These replace the MPI AllReduce call sites of the reference's reports and
// convergence test (simulator.cpp:284, 310; scsp.cpp:331-341;
// colorfluid.cpp:852-866).  Pass 1 runs a fixed grid of blocks, each thread
// accumulating a grid-strided subset of nodes, then reduces the block with
// warp shuffles; pass 2 reduces the per-block partials in one block.  Grid and
// block sizes are fixed, so the summation order -- and the result -- is the
// same on every call.
#pragma once
#include "kernels.cuh"

namespace lbf {

constexpr int kReduceThreads = 256;
constexpr int kReduceBlocks = 148 * 4;
constexpr int kReduceMaxK = 16;

template <class Fn>
__global__ void __launch_bounds__(kReduceThreads)
reduce_pass1(const Fn fn, uint32_t n, double* __restrict__ partial)
{
    constexpr int K = Fn::K;
    double acc[K];
#pragma unroll
    for (int k = 0; k < K; ++k) acc[k] = 0.0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        fn(i, acc);
    __shared__ double sm[K][kReduceThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        double v = acc[k];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            const double o = __shfl_down_sync(0xffffffffu, v, off);
            v = Fn::is_max(k) ? fmax(v, o) : v + o;
        }
        if (lane == 0) sm[k][warp] = v;
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) {
            double v = lane < kReduceThreads / 32 ? sm[k][lane] : 0.0;
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) {
                const double o = __shfl_down_sync(0xffffffffu, v, off);
                v = Fn::is_max(k) ? fmax(v, o) : v + o;
            }
            if (lane == 0) partial[(size_t)blockIdx.x * K + k] = v;
        }
    }
}

template <class Fn>
__global__ void __launch_bounds__(kReduceThreads)
reduce_pass2(const double* __restrict__ partial, int nblocks, double* __restrict__ out)
{
    constexpr int K = Fn::K;
    double acc[K];
#pragma unroll
    for (int k = 0; k < K; ++k) acc[k] = 0.0;
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x)
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const double v = partial[(size_t)b * K + k];
            acc[k] = Fn::is_max(k) ? fmax(acc[k], v) : acc[k] + v;
        }
    __shared__ double sm[K][kReduceThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        double v = acc[k];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            const double o = __shfl_down_sync(0xffffffffu, v, off);
            v = Fn::is_max(k) ? fmax(v, o) : v + o;
        }
        if (lane == 0) sm[k][warp] = v;
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) {
            double v = lane < kReduceThreads / 32 ? sm[k][lane] : 0.0;
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) {
                const double o = __shfl_down_sync(0xffffffffu, v, off);
                v = Fn::is_max(k) ? fmax(v, o) : v + o;
            }
            if (lane == 0) out[k] = v;
        }
    }
}

// Simulator::updateConvergence sums (simulator.cpp:263-310).
struct ConvergenceFn {
    static constexpr int K = 5;
    const double *u, *uprev, *uadj, *ind, *indprev, *indadj;
    uint32_t nfp;
    int color;
    __host__ __device__ static constexpr bool is_max(int k) { return k >= 3; }
    __device__ void operator()(uint32_t i, double (&a)[K]) const
    {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const size_t j = (size_t)c * nfp + i;
            const double v = u[j], d = v - uprev[j], da = v - uadj[j];
            a[0] += d * d;
            a[1] += v * v;
            a[2] += da * da;
        }
        if (color) {
            a[3] = fmax(a[3], fabs(ind[i] - indprev[i]));
            a[4] = fmax(a[4], fabs(ind[i] - indadj[i]));
        }
    }
};

// Slice sums of SCSP::report / ColorFluid::report.
struct ReportFn {
    static constexpr int K = 10;
    const uint32_t* coord;
    const double *u, *rho0, *rho1;
    uint32_t nfp;
    int axis;
    int lo, hi;
    __host__ __device__ static constexpr bool is_max(int) { return false; }
    __device__ void operator()(uint32_t i, double (&a)[K]) const
    {
        int x, y, z;
        unpack(coord[i], x, y, z);
        const int c = axis == 0 ? x : (axis == 1 ? y : z);
        if (c < lo || c > hi) return;
        const double r0 = rho0[i], r1 = rho1 ? rho1[i] : 0.0;
        a[0] += u[(size_t)axis * nfp + i];
        a[1] += r0;
        a[2] += r1;
        a[9] += 1.0;
        if (c == lo) { a[3] += r0; a[4] += r1; a[7] += 1.0; }
        if (c == hi) { a[5] += r0; a[6] += r1; a[8] += 1.0; }
    }
};

// Pore measures of scripts/porous_media.py:20-44 (sums over fluid voxels).
struct FluxFn {
    static constexpr int K = 9;
    const double *u, *rho0, *rho1;
    uint32_t nfp;
    __host__ __device__ static constexpr bool is_max(int) { return false; }
    __device__ void operator()(uint32_t i, double (&a)[K]) const
    {
        const double r0 = rho0[i], r1 = rho1 ? rho1[i] : 0.0;
        const double phi0 = rho1 ? r0 / (r0 + r1) : 1.0;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const double v = u[(size_t)c * nfp + i];
            a[c] += v;
            a[3 + c] += phi0 * v;
        }
        a[6] += r0;
        a[7] += r1;
        a[8] += phi0;
    }
};

}  // namespace lbf
