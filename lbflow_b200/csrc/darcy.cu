// Block-scale Darcy pressure solve of the convergence accelerator.
//
// Given a mobility M per block of a periodic block grid (nz x ny x nx
// blocks of edge h voxels) and a body force g along +x, find the zero-mean
// pressure phi (over rho0) with a conserved block flux
//     F_f = M_f (g [f is an x face] - (phi_nb - phi) / h)
// across every block face, M_f the geometric mean of the two blocks'
// mobilities:   sum_f M_f (phi_nb - phi) / h^2 = g (Mx_{i+1/2} - Mx_{i-1/2}) / h.
//
// Conjugate gradients in FP64 preconditioned by one symmetric multigrid
// V-cycle in FP32: damped Jacobi (2 + 2 sweeps), trilinear prolongation,
// its adjoint / 8 as restriction, coarse face mobilities = mean of the four
// fine faces of each coarse interface, and a single-CTA Jacobi solve on the
// coarsest grid.  One kernel per smoothing sweep, transfer and vector
// update; dot products are two-pass (deterministic) and the only host
// synchronisation per iteration is the residual norm.
#include "../../include/lbflow.h"
#include "internal.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <utility>
#include <vector>

namespace {

constexpr int kT = 256;
constexpr int kCoarseSweeps = 120;   // Jacobi sweeps on the coarsest (<= 1024-cell) grid

struct Dims {
    int nz, ny, nx;
    __host__ __device__ size_t n() const { return (size_t)nz * ny * nx; }
};

__device__ __forceinline__ int wrapi(int v, int n) { return v < 0 ? v + n : (v >= n ? v - n : v); }

__device__ __forceinline__ void coords(const Dims& d, size_t i, int& z, int& y, int& x)
{
    x = (int)(i % d.nx);
    const size_t t = i / d.nx;
    y = (int)(t % d.ny);
    z = (int)(t / d.ny);
}

__device__ __forceinline__ size_t idx(const Dims& d, int z, int y, int x)
{
    return ((size_t)z * d.ny + y) * d.nx + x;
}

// Face mobilities on the + faces (geometric mean) and the right-hand side.
__global__ void setup_fine(Dims d, const double* __restrict__ mob, double g, double h, float* __restrict__ mx,
                           float* __restrict__ my, float* __restrict__ mz, double* __restrict__ rhs)
{
    const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i >= d.n()) return;
    int z, y, x;
    coords(d, i, z, y, x);
    const double m = fmax(mob[i], 1e-300);
    const double fx = sqrt(m * fmax(mob[idx(d, z, y, wrapi(x + 1, d.nx))], 1e-300));
    const double fxm = sqrt(fmax(mob[idx(d, z, y, wrapi(x - 1, d.nx))], 1e-300) * m);
    mx[i] = (float)fx;
    my[i] = (float)sqrt(m * fmax(mob[idx(d, z, wrapi(y + 1, d.ny), x)], 1e-300));
    mz[i] = (float)sqrt(m * fmax(mob[idx(d, wrapi(z + 1, d.nz), y, x)], 1e-300));
    rhs[i] = g * (fx - fxm) / h;
}

// sum_faces M_f (x_nb - x_i), and the diagonal -sum_faces M_f.
template <class T>
__device__ __forceinline__ T stencil(const Dims& d, const T* x, const float* __restrict__ mx,
                                     const float* __restrict__ my, const float* __restrict__ mz, size_t i, int z,
                                     int y, int xx, T& diag)
{
    const size_t xm = idx(d, z, y, wrapi(xx - 1, d.nx)), xp = idx(d, z, y, wrapi(xx + 1, d.nx));
    const size_t ym = idx(d, z, wrapi(y - 1, d.ny), xx), yp = idx(d, z, wrapi(y + 1, d.ny), xx);
    const size_t zm = idx(d, wrapi(z - 1, d.nz), y, xx), zp = idx(d, wrapi(z + 1, d.nz), y, xx);
    const T c = x[i];
    const T a = (T)mx[i], b = (T)mx[xm], e = (T)my[i], f = (T)my[ym], gg = (T)mz[i], k = (T)mz[zm];
    diag = -(a + b + e + f + gg + k);
    return a * (x[xp] - c) - b * (c - x[xm]) + e * (x[yp] - c) - f * (c - x[ym]) + gg * (x[zp] - c) -
           k * (c - x[zm]);
}

// out = A x  (FP64, the CG operator)
__global__ void apply64(Dims d, double h2inv, const double* __restrict__ x, const float* __restrict__ mx,
                        const float* __restrict__ my, const float* __restrict__ mz, double* __restrict__ out)
{
    const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i >= d.n()) return;
    int z, y, xx;
    coords(d, i, z, y, xx);
    double dg;
    out[i] = stencil<double>(d, x, mx, my, mz, i, z, y, xx, dg) * h2inv;
}

// One damped Jacobi sweep: xo = xi + omega (r - A xi) / diag   (FP32)
__global__ void jacobi(Dims d, float h2inv, float omega, const float* __restrict__ xi, const float* __restrict__ r,
                       const float* __restrict__ mx, const float* __restrict__ my, const float* __restrict__ mz,
                       float* __restrict__ xo)
{
    const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i >= d.n()) return;
    int z, y, xx;
    coords(d, i, z, y, xx);
    float dg;
    const float ax = stencil<float>(d, xi, mx, my, mz, i, z, y, xx, dg) * h2inv;
    xo[i] = dg != 0.f ? xi[i] + omega * (r[i] - ax) / (dg * h2inv) : xi[i];
}

// res = r - A x  (FP32)
__global__ void residual(Dims d, float h2inv, const float* __restrict__ x, const float* __restrict__ r,
                         const float* __restrict__ mx, const float* __restrict__ my, const float* __restrict__ mz,
                         float* __restrict__ res)
{
    const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i >= d.n()) return;
    int z, y, xx;
    coords(d, i, z, y, xx);
    float dg;
    res[i] = r[i] - stencil<float>(d, x, mx, my, mz, i, z, y, xx, dg) * h2inv;
}

// Coarse face mobilities: mean of the four fine faces on each coarse interface.
__global__ void coarsen_faces(Dims c, Dims f, const float* __restrict__ fmx, const float* __restrict__ fmy,
                              const float* __restrict__ fmz, float* __restrict__ cmx, float* __restrict__ cmy,
                              float* __restrict__ cmz)
{
    const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i >= c.n()) return;
    int z, y, x;
    coords(c, i, z, y, x);
    const int Z = 2 * z, Y = 2 * y, X = 2 * x;
    float sx = 0.f, sy = 0.f, sz = 0.f;
    for (int a = 0; a < 2; ++a)
        for (int b = 0; b < 2; ++b) {
            sx += fmx[idx(f, Z + a, Y + b, X + 1)];
            sy += fmy[idx(f, Z + a, Y + 1, X + b)];
            sz += fmz[idx(f, Z + 1, Y + a, X + b)];
        }
    cmx[i] = 0.25f * sx;
    cmy[i] = 0.25f * sy;
    cmz[i] = 0.25f * sz;
}

// Restriction: adjoint of the trilinear prolongation / 8; weights
// 1/8, 3/8, 3/8, 1/8 over fine cells 2i-1 .. 2i+2 on each axis.
__global__ void restrict3(Dims c, Dims f, const float* __restrict__ rf, float* __restrict__ rc)
{
    const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i >= c.n()) return;
    int z, y, x;
    coords(c, i, z, y, x);
    const float w[4] = {0.125f, 0.375f, 0.375f, 0.125f};
    float s = 0.f;
    for (int a = 0; a < 4; ++a) {
        const int Z = wrapi(2 * z - 1 + a, f.nz);
        for (int b = 0; b < 4; ++b) {
            const int Y = wrapi(2 * y - 1 + b, f.ny);
            for (int e = 0; e < 4; ++e) {
                const int X = wrapi(2 * x - 1 + e, f.nx);
                s += w[a] * w[b] * w[e] * rf[idx(f, Z, Y, X)];
            }
        }
    }
    rc[i] = s;
}

// xf += trilinear prolongation of ec.
__global__ void prolong_add(Dims f, Dims c, const float* __restrict__ ec, float* __restrict__ xf)
{
    const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i >= f.n()) return;
    int z, y, x;
    coords(f, i, z, y, x);
    const int cz0 = z >> 1, cy0 = y >> 1, cx0 = x >> 1;
    const int cz1 = wrapi(cz0 + ((z & 1) ? 1 : -1), c.nz);
    const int cy1 = wrapi(cy0 + ((y & 1) ? 1 : -1), c.ny);
    const int cx1 = wrapi(cx0 + ((x & 1) ? 1 : -1), c.nx);
    const int cz[2] = {cz0, cz1}, cy[2] = {cy0, cy1}, cx[2] = {cx0, cx1};
    const float w[2] = {0.75f, 0.25f};
    float s = 0.f;
    for (int a = 0; a < 2; ++a)
        for (int b = 0; b < 2; ++b)
            for (int e = 0; e < 2; ++e) s += w[a] * w[b] * w[e] * ec[idx(c, cz[a], cy[b], cx[e])];
    xf[i] += s;
}

// Coarsest grid (n <= 1024 cells): zero-mean damped Jacobi sweeps inside one CTA.
__global__ void __launch_bounds__(1024) coarse_solve(Dims d, float h2inv, int sweeps, const float* __restrict__ r,
                                                     const float* __restrict__ mx, const float* __restrict__ my,
                                                     const float* __restrict__ mz, float* __restrict__ x)
{
    __shared__ float xs[1024], rs[1024], red[32];
    const int n = (int)d.n();
    const int t = threadIdx.x;
    const int nwarps = (int)(blockDim.x + 31) / 32;
    // Block mean of a per-thread value, into red[0].
    auto block_mean = [&](float v) {
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        __syncthreads();
        if ((t & 31) == 0) red[t >> 5] = v;
        __syncthreads();
        if (t == 0) {
            float s = 0.f;
            for (int w = 0; w < nwarps; ++w) s += red[w];
            red[0] = s / (float)n;
        }
        __syncthreads();
        return red[0];
    };
    const float rmean = block_mean(t < n ? r[t] : 0.f);
    if (t < n) { xs[t] = 0.f; rs[t] = r[t] - rmean; }
    __syncthreads();
    int z = 0, y = 0, xx = 0;
    if (t < n) coords(d, (size_t)t, z, y, xx);
    for (int k = 0; k < sweeps; ++k) {
        float nv = 0.f;
        if (t < n) {
            float dg;
            const float ax = stencil<float>(d, xs, mx, my, mz, (size_t)t, z, y, xx, dg) * h2inv;
            nv = dg != 0.f ? xs[t] + 0.8f * (rs[t] - ax) / (dg * h2inv) : xs[t];
        }
        __syncthreads();
        if (t < n) xs[t] = nv;
        __syncthreads();
    }
    const float xmean = block_mean(t < n ? xs[t] : 0.f);
    if (t < n) x[t] = xs[t] - xmean;
}

__global__ void to_f32(size_t n, const double* __restrict__ a, float* __restrict__ b)
{
    const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i < n) b[i] = (float)a[i];
}
__global__ void to_f64(size_t n, const float* __restrict__ a, double* __restrict__ b)
{
    const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i < n) b[i] = (double)a[i];
}
__global__ void fill0(size_t n, float* __restrict__ a)
{
    const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i < n) a[i] = 0.f;
}
// y += sign * (num / den) * x, the ratio read on the device.
__global__ void axpy_ratio(size_t n, const double* __restrict__ num, const double* __restrict__ den, double sign,
                           const double* __restrict__ x, double* __restrict__ y)
{
    const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i < n) y[i] += sign * (num[0] / den[0]) * x[i];
}
// p = z + (num / den) p
__global__ void xpby_ratio(size_t n, const double* __restrict__ z, const double* __restrict__ num,
                           const double* __restrict__ den, double* __restrict__ p)
{
    const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i < n) p[i] = z[i] + (num[0] / den[0]) * p[i];
}
// Two-pass deterministic reductions: per-block partials, then one thread in order.
// b == nullptr sums a alone.
__global__ void dot_partial(size_t n, const double* __restrict__ a, const double* __restrict__ b,
                            double* __restrict__ part)
{
    __shared__ double s[kT];
    double v = 0.0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        v += b ? a[i] * b[i] : a[i];
    s[threadIdx.x] = v;
    __syncthreads();
    for (int o = kT / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) s[threadIdx.x] += s[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = s[0];
}
// Second pass: one block sums the partials in a fixed tree order.
__global__ void dot_final(int nb, const double* __restrict__ part, double* __restrict__ out)
{
    __shared__ double s[kT];
    double v = 0.0;
    for (int i = threadIdx.x; i < nb; i += kT) v += part[i];
    s[threadIdx.x] = v;
    __syncthreads();
    for (int o = kT / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) s[threadIdx.x] += s[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[0] = s[0];
}
__global__ void copy_scalar(const double* __restrict__ a, double* __restrict__ b) { b[0] = a[0]; }
__global__ void sub_mean(size_t n, const double* __restrict__ sum, double* __restrict__ a)
{
    const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i < n) a[i] -= sum[0] / (double)n;
}

unsigned nblk(size_t n) { return (unsigned)((n + kT - 1) / kT); }

struct Level {
    Dims d;
    float h2inv;
    float *mx, *my, *mz, *x, *r, *t;
};

struct Solver {
    cudaStream_t s = nullptr;
    std::vector<Level> L;
    double* part = nullptr;
    int nb_dot = 0;
    cudaError_t err = cudaSuccess;
    // One device allocation carved into 256-byte-aligned arrays: a first
    // pass (base == nullptr) only adds up the size.
    char* base = nullptr;
    size_t used = 0;

    template <class T> T* alloc(size_t n)
    {
        T* p = base ? reinterpret_cast<T*>(base + used) : nullptr;
        used += (n * sizeof(T) + 255) / 256 * 256;
        return p;
    }
    ~Solver() { if (base) cudaFreeAsync(base, s); }

    void smooth(int l, int sweeps)
    {
        Level& v = L[l];
        for (int k = 0; k < sweeps; ++k) {
            jacobi<<<nblk(v.d.n()), kT, 0, s>>>(v.d, v.h2inv, 0.7f, v.x, v.r, v.mx, v.my, v.mz, v.t);
            std::swap(v.x, v.t);
        }
    }

    // L[l].x = V-cycle applied to L[l].r.
    void vcycle(int l)
    {
        Level& v = L[l];
        if (l + 1 == (int)L.size()) {
            coarse_solve<<<1, 1024, 0, s>>>(v.d, v.h2inv, kCoarseSweeps, v.r, v.mx, v.my, v.mz, v.x);
            return;
        }
        fill0<<<nblk(v.d.n()), kT, 0, s>>>(v.d.n(), v.x);
        smooth(l, 2);
        residual<<<nblk(v.d.n()), kT, 0, s>>>(v.d, v.h2inv, v.x, v.r, v.mx, v.my, v.mz, v.t);
        Level& c = L[l + 1];
        restrict3<<<nblk(c.d.n()), kT, 0, s>>>(c.d, v.d, v.t, c.r);
        vcycle(l + 1);
        prolong_add<<<nblk(v.d.n()), kT, 0, s>>>(v.d, c.d, c.x, v.x);
        smooth(l, 2);
    }

    void dot(size_t n, const double* a, const double* b, double* out)
    {
        dot_partial<<<nb_dot, kT, 0, s>>>(n, a, b, part);
        dot_final<<<1, kT, 0, s>>>(nb_dot, part, out);
    }
};

int fail(const std::string& m, int code = LBF_EINVAL)
{
    lbf::set_global_error(m);
    return code;
}

}  // namespace

extern "C" int lbf_darcy_pressure(const double* mob, uint32_t nz, uint32_t ny, uint32_t nx, double h, double g,
                                  double rtol, uint32_t max_iter, double* phi, uint32_t* iterations, void* stream)
{
    if (!mob || !phi || !nz || !ny || !nx || !(h > 0)) return fail("lbf_darcy_pressure: bad arguments");
    const Dims d0{(int)nz, (int)ny, (int)nx};
    const size_t n = d0.n();
    if (n > ((size_t)1 << 30)) return fail("lbf_darcy_pressure: grid too large");
    // Level hierarchy: halve while every extent is even and the grid has > 512 cells.
    std::vector<Dims> dims{d0};
    while (dims.back().n() > 512 && !((dims.back().nz | dims.back().ny | dims.back().nx) & 1))
        dims.push_back(Dims{dims.back().nz / 2, dims.back().ny / 2, dims.back().nx / 2});
    if (dims.back().n() > 1024)
        return fail("lbf_darcy_pressure: grid extents must halve down to at most 1024 cells");
    cudaPointerAttributes pa{};
    if (cudaPointerGetAttributes(&pa, mob) != cudaSuccess || pa.type != cudaMemoryTypeDevice ||
        cudaPointerGetAttributes(&pa, phi) != cudaSuccess || pa.type != cudaMemoryTypeDevice) {
        cudaGetLastError();
        return fail("lbf_darcy_pressure: mob and phi must be device memory");
    }
    Solver S;
    S.s = static_cast<cudaStream_t>(stream);
    S.nb_dot = (int)std::min<size_t>(nblk(n), 1184);
    double *rhs = nullptr, *r = nullptr, *z = nullptr, *p = nullptr, *Ap = nullptr, *sc = nullptr;
    for (int pass = 0; pass < 2; ++pass) {
        if (pass == 1) {
            // The workspace comes from the library's device pool on the
            // solve's stream: a correction inside a timed run reuses memory
            // reserved by earlier solves instead of calling the driver.
            void* mem = nullptr;
            int dev = 0;
            cudaMemPool_t pool = nullptr;
            S.err = cudaGetDevice(&dev);
            if (S.err == cudaSuccess) S.err = lbf::device_pool(dev, &pool);
            if (S.err == cudaSuccess) S.err = cudaMallocFromPoolAsync(&mem, S.used, pool, S.s);
            if (S.err != cudaSuccess)
                return fail(std::string("lbf_darcy_pressure: ") + cudaGetErrorString(S.err), LBF_ENOMEM);
            S.base = static_cast<char*>(mem);
            S.used = 0;
            S.L.clear();
        }
        float hh = (float)h;
        for (const Dims& d : dims) {
            Level v{};
            v.d = d;
            v.h2inv = 1.0f / (hh * hh);
            const size_t m = d.n();
            v.mx = S.alloc<float>(m); v.my = S.alloc<float>(m); v.mz = S.alloc<float>(m);
            v.x = S.alloc<float>(m); v.r = S.alloc<float>(m); v.t = S.alloc<float>(m);
            S.L.push_back(v);
            hh *= 2.f;
        }
        rhs = S.alloc<double>(n);
        r = S.alloc<double>(n);
        z = S.alloc<double>(n);
        p = S.alloc<double>(n);
        Ap = S.alloc<double>(n);
        sc = S.alloc<double>(8);          // scalars: rz, pAp, rz_new, rr, sum
        S.part = S.alloc<double>(S.nb_dot);
    }
    cudaStream_t s = S.s;
    const double h2inv = 1.0 / (h * h);
    setup_fine<<<nblk(n), kT, 0, s>>>(d0, mob, g, h, S.L[0].mx, S.L[0].my, S.L[0].mz, rhs);
    for (size_t l = 1; l < S.L.size(); ++l)
        coarsen_faces<<<nblk(S.L[l].d.n()), kT, 0, s>>>(S.L[l].d, S.L[l - 1].d, S.L[l - 1].mx, S.L[l - 1].my,
                                                          S.L[l - 1].mz, S.L[l].mx, S.L[l].my, S.L[l].mz);
    // Zero-mean right-hand side; phi = 0; r = rhs.
    S.dot(n, rhs, nullptr, sc + 4);
    sub_mean<<<nblk(n), kT, 0, s>>>(n, sc + 4, rhs);
    cudaMemsetAsync(phi, 0, n * sizeof(double), s);
    cudaMemcpyAsync(r, rhs, n * sizeof(double), cudaMemcpyDeviceToDevice, s);
    double hr = 0.0;
    S.dot(n, r, r, sc + 3);
    cudaMemcpyAsync(&hr, sc + 3, sizeof(double), cudaMemcpyDeviceToHost, s);
    cudaError_t e = cudaStreamSynchronize(s);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) return fail(std::string("lbf_darcy_pressure: ") + cudaGetErrorString(e), LBF_ECUDA);
    const double nrm0 = std::sqrt(hr);
    uint32_t it = 0;
    if (nrm0 > 0) {
        auto precondition = [&](const double* rin, double* zout) {
            to_f32<<<nblk(n), kT, 0, s>>>(n, rin, S.L[0].r);
            S.vcycle(0);
            to_f64<<<nblk(n), kT, 0, s>>>(n, S.L[0].x, zout);
        };
        precondition(r, z);
        cudaMemcpyAsync(p, z, n * sizeof(double), cudaMemcpyDeviceToDevice, s);
        S.dot(n, r, z, sc + 0);
        while (it < max_iter) {
            apply64<<<nblk(n), kT, 0, s>>>(d0, h2inv, p, S.L[0].mx, S.L[0].my, S.L[0].mz, Ap);
            S.dot(n, p, Ap, sc + 1);
            axpy_ratio<<<nblk(n), kT, 0, s>>>(n, sc + 0, sc + 1, 1.0, p, phi);
            axpy_ratio<<<nblk(n), kT, 0, s>>>(n, sc + 0, sc + 1, -1.0, Ap, r);
            ++it;
            S.dot(n, r, r, sc + 3);
            cudaMemcpyAsync(&hr, sc + 3, sizeof(double), cudaMemcpyDeviceToHost, s);
            e = cudaStreamSynchronize(s);
            if (e != cudaSuccess) return fail(std::string("lbf_darcy_pressure: ") + cudaGetErrorString(e), LBF_ECUDA);
            if (!(std::sqrt(hr) > rtol * nrm0)) break;
            precondition(r, z);
            S.dot(n, r, z, sc + 2);
            xpby_ratio<<<nblk(n), kT, 0, s>>>(n, z, sc + 2, sc + 0, p);
            copy_scalar<<<1, 1, 0, s>>>(sc + 2, sc + 0);
        }
    }
    // Zero mean.
    S.dot(n, phi, nullptr, sc + 4);
    sub_mean<<<nblk(n), kT, 0, s>>>(n, sc + 4, phi);
    e = cudaStreamSynchronize(s);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) return fail(std::string("lbf_darcy_pressure: ") + cudaGetErrorString(e), LBF_ECUDA);
    if (iterations) *iterations = it;
    return LBF_OK;
}
