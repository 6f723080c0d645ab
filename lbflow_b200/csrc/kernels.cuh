// Device kernels of the lattice Boltzmann engine (sm_100a).
//
// Data layout in HBM (one geometry per engine):
//   occ[w]   uint2 per 32 voxels of an x-row: .x = fluid bits, .y = number of
//            fluid voxels in all earlier words (row-major z, y, x-word order).
//            The compact index of fluid voxel (x,y,z) is
//            occ[w].y + popc(occ[w].x & ((1 << (x & 31)) - 1)).
//   coord[i] packed (x | y << 11 | z << 22) of fluid node i; nodes are in
//            voxel (z, y, x) order, so threads of a warp touch neighbouring x.
//   f[p][q][i] populations of phase p, direction q, fluid node i (stride nfp).
// Only fluid voxels are stored; a pull from a solid neighbour becomes the
// halfway bounce-back f_q(x) = f*_{op q}(x) of the reference
// (solver/src/lbm/simulator.cpp:103-111 with the link lists of :386-436).
#pragma once
#include <cuda_fp16.h>
#include <cuda_bf16.h>
#include <cstdint>
#include "lattice.cuh"
#include "moments_gen.cuh"

namespace lbf {

// Device error word bits (the reference's throw sites).
enum : uint32_t {
    kErrDensity   = 1u << 0,  // non-finite or non-positive density (scsp.cpp:144-145; colorfluid.cpp:255-257)
    kErrComponent = 1u << 1,  // negative component density (colorfluid.cpp:258-259)
    kErrTau       = 1u << 2,  // local relaxation time <= 0.5 (colorfluid.cpp:269-270)
    kErrVelocity  = 1u << 3,  // non-finite velocity (colorfluid.cpp:282-283)
};

// Output requests for a step kernel.
enum : int { kOutMacros = 1, kOutAdjacent = 2 };

struct Grid {
    int nx, ny, nz, W;          // W: 32-bit occupancy words per x-row
    uint32_t nf;                // fluid nodes
    uint32_t nfp;               // padded stride between direction blocks
    const uint2* __restrict__ occ;
    const uint32_t* __restrict__ coord;
};

struct Force {
    // uniform != 0: every fluid node feels (fx, fy, fz); otherwise the force
    // is label_force[label[i]] (x, y, z per label, zero for non-GV labels).
    int uniform;
    double fx, fy, fz;
    const uint8_t* __restrict__ label;
    const double* __restrict__ label_force;   // [256][3]
};

struct Macros {                 // compact per-node outputs, stride nfp
    double* rho0;               // density (single phase) / rho_0 (color)
    double* rho1;               // color: rho_1
    double* u;                  // [3][nfp] x, y, z (includes the half force)
    double* uadj;               // [3][nfp] velocity of the step before a report
    double* ind;                // color: phase indicator (rho0-rho1)/rho
    double* indadj;             // color: indicator of the step before a report
};

__device__ __forceinline__ int wrap(int v, int n) { return v < 0 ? v + n : (v >= n ? v - n : v); }

__device__ __forceinline__ void unpack(uint32_t c, int& x, int& y, int& z)
{ x = c & 2047; y = (c >> 11) & 2047; z = c >> 22; }

// Compact index of voxel (x, y, z); fluid = whether it holds a fluid node.
__device__ __forceinline__ uint32_t lookup(const Grid& g, int x, int y, int z, bool& fluid)
{
    const uint2 e = __ldg(&g.occ[((size_t)z * g.ny + y) * g.W + (x >> 5)]);
    const uint32_t bit = x & 31;
    fluid = (e.x >> bit) & 1u;
    return e.y + __popc(e.x & ((1u << bit) - 1u));
}

// ---- storage policies -------------------------------------------------------
// Full FP64 populations (the plain path; arithmetic close to the reference).
struct StoreF64 {
    using T = double;
    using R = double;
    static constexpr bool shifted = false;
    __device__ static R load(const T* p, int, R) { return __ldg(p); }
    __device__ static void store(T* p, R v, int, R) { *p = v; }
};
// Shifted deviations g_q = f_q - w_q rho0, stored as h_q = g_q * (4096 / w_q)
// in a 16-bit float; arithmetic in FP32 on the deviations.
template <class L> struct ShiftScale {
    __device__ static float scale(int q) { return 4096.0f * 36.0f / (float)L::w36f(q); }
    __device__ static float inv(int q) { return (float)L::w36f(q) / (36.0f * 4096.0f); }
};
template <class L> struct StoreF16 {
    using T = __half;
    using R = float;
    static constexpr bool shifted = true;
    __device__ static R load(const T* p, int q, R) { return __half2float(__ldg(p)) * ShiftScale<L>::inv(q); }
    __device__ static void store(T* p, R v, int q, R) { *p = __float2half_rn(v * ShiftScale<L>::scale(q)); }
};
template <class L> struct StoreBF16 {
    using T = __nv_bfloat16;
    using R = float;
    static constexpr bool shifted = true;
    __device__ static R load(const T* p, int q, R) { return __bfloat162float(__ldg(p)) * ShiftScale<L>::inv(q); }
    __device__ static void store(T* p, R v, int q, R) { *p = __float2bfloat16_rn(v * ShiftScale<L>::scale(q)); }
};
template <class L> struct StoreF32 {
    using T = float;
    using R = float;
    static constexpr bool shifted = true;
    __device__ static R load(const T* p, int, R) { return __ldg(p); }
    __device__ static void store(T* p, R v, int, R) { *p = v; }
};

// Full (unshifted) populations in FP32 with FP32 arithmetic.
struct StoreF32Full {
    using T = float;
    using R = float;
    static constexpr bool shifted = false;
    __device__ static R load(const T* p, int, R) { return __ldg(p); }
    __device__ static void store(T* p, R v, int, R) { *p = v; }
};

// ---- gather: pull-stream with halfway bounce-back ----------------------------
// src[q] receives f_q(x - e_q) after streaming, or f*_{op q}(x) when the
// upstream voxel is solid.  nbr[q] (q >= 1) records the compact index of the
// voxel x + e_q (the pull source of op q) or UINT32_MAX when it is solid.
template <class L, class S, bool PULL>
__device__ __forceinline__ void gather(const Grid& g, const typename S::T* __restrict__ fin,
                                       uint32_t i, int x, int y, int z,
                                       typename S::R (&f)[L::Q], uint32_t (&nbr)[L::Q],
                                       typename S::R rho0)
{
    f[0] = S::load(fin + i, 0, rho0);
    nbr[0] = i;
#pragma unroll
    for (int q = 1; q < L::Q; ++q) {
        if (!PULL) { f[q] = S::load(fin + (size_t)q * g.nfp + i, q, rho0); nbr[q] = 0; continue; }
        const int sx = wrap(x - L::ex(q), g.nx);
        const int sy = wrap(y - L::ey(q), g.ny);
        const int sz = L::D == 3 ? wrap(z - L::ez(q), g.nz) : 0;
        bool fluid;
        const uint32_t j = lookup(g, sx, sy, sz, fluid);
        nbr[L::op(q)] = fluid ? j : 0xffffffffu;
        const typename S::T* p = fluid ? fin + (size_t)q * g.nfp + j
                                       : fin + (size_t)L::op(q) * g.nfp + i;
        f[q] = S::load(p, q, rho0);
    }
}

// ---- moments (straight-line code generated by gen_moments.py) ---------------
template <class R> __device__ __forceinline__ void mforward(const R (&f)[9], R (&m)[9]) { forward_d2q9(f, m); }
template <class R> __device__ __forceinline__ void mforward(const R (&f)[19], R (&m)[19]) { forward_d3q19(f, m); }
template <class R> __device__ __forceinline__ void minverse_add(const R (&c)[9], R (&f)[9]) { inverse_add_d2q9(c, f); }
template <class R> __device__ __forceinline__ void minverse_add(const R (&c)[19], R (&f)[19]) { inverse_add_d3q19(c, f); }
template <class L, class R>
__device__ __forceinline__ R mequil(int k, R rho, R rho0, const R (&u)[3], const R (&uu)[6])
{
    if constexpr (L::Q == 9) return meq_d2q9<R>(k, rho, rho0, u, uu);
    else return meq_d3q19<R>(k, rho, rho0, u, uu);
}
template <class L, class R>
__device__ __forceinline__ R msource(int k, const R (&F)[3], const R (&uF)[3][3], R uf)
{
    if constexpr (L::Q == 9) return msrc_d2q9<R>(k, F, uF, uf);
    else return msrc_d3q19<R>(k, F, uF, uf);
}

// Per-row MRT coefficients: cr[k] = s_k / |M_k|^2, cs[k] = (1 - s_k/2) / |M_k|^2,
// inv_n[k] = 1 / |M_k|^2.
struct MrtCoef { double cr[19], cs[19], inv_n[19]; };

// ---- single-phase step (SCSP) ----------------------------------------------------
// One launch = Simulator::streaming + bounceBack (simulator.cpp:73-111),
// SCSP::calcMacroVar + bodyForce (scsp.cpp:136-175) and SCSP::equilSRT /
// equilMRT (scsp.cpp:374-464) for every fluid node.  PULL = false is the t = 0
// collision of SCSP::Run (scsp.cpp:60-71), which reads the node's own values.
struct ScspParams {
    double rho0;       // reference density (incompressible form, lbcfg.h:13)
    double inv_rho0;
    double omega;      // SRT relaxation frequency 1/tau
    MrtCoef mrt;
};

template <class L, bool MRT, class S, bool PULL>
__global__ void __launch_bounds__(128)
scsp_step(const Grid g, const Force F, const ScspParams P,
          const typename S::T* __restrict__ fin, typename S::T* __restrict__ fout,
          Macros mo, const int out, uint32_t* __restrict__ err)
{
    using R = typename S::R;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.nf) return;
    int x, y, z;
    unpack(__ldg(&g.coord[i]), x, y, z);
    const R rho0 = R(P.rho0);
    R f[L::Q];
    uint32_t nbr[L::Q];
    gather<L, S, PULL>(g, fin, i, x, y, z, f, nbr, rho0);

    R Fv[3];
    if (F.uniform) { Fv[0] = R(F.fx); Fv[1] = R(F.fy); Fv[2] = R(F.fz); }
    else {
        const double* lf = F.label_force + 3 * __ldg(&F.label[i]);
        Fv[0] = R(lf[0]); Fv[1] = R(lf[1]); Fv[2] = R(lf[2]);
    }

    R m[L::Q];
    R rho, j[3];
    if (MRT) {
        mforward<R>(f, m);
        rho = m[0];
        j[0] = m[L::jrow(0)]; j[1] = m[L::jrow(1)]; j[2] = L::D == 3 ? m[L::jrow(2)] : R(0);
    } else {
        rho = f[0];
#pragma unroll
        for (int q = 1; q < L::Q; ++q) rho += f[q];
        j[0] = j[1] = j[2] = R(0);
#pragma unroll
        for (int p = 0; p < L::NPAIR; ++p) {
            const int q = L::pair(p);
            const R b = f[q] - f[L::op(q)];
            if (L::ex(q)) j[0] += R(L::ex(q)) * b;
            if (L::ey(q)) j[1] += R(L::ey(q)) * b;
            if (L::ez(q)) j[2] += R(L::ez(q)) * b;
        }
    }
    const R rho_full = S::shifted ? rho0 + rho : rho;
    if (!(rho_full > R(0)) || !isfinite(rho_full)) atomicOr(err, kErrDensity);

    const R irho0 = R(P.inv_rho0);
    R u[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) u[a] = j[a] * irho0 + Fv[a] * R(0.5) * irho0;
    const R usq = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
    const R uf = u[0] * Fv[0] + u[1] * Fv[1] + u[2] * Fv[2];

    if (out & kOutMacros) {
        mo.rho0[i] = (double)rho0 * (S::shifted ? 1.0 : 0.0) + (double)rho;
#pragma unroll
        for (int a = 0; a < 3; ++a) mo.u[(size_t)a * g.nfp + i] = (double)u[a];
    }
    if (out & kOutAdjacent) {
#pragma unroll
        for (int a = 0; a < 3; ++a) mo.uadj[(size_t)a * g.nfp + i] = (double)u[a];
    }

    if (MRT) {
        const R uu[6] = {u[0] * u[0], u[1] * u[1], u[2] * u[2], u[0] * u[1], u[0] * u[2], u[1] * u[2]};
        R uF[3][3];
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int b = 0; b < 3; ++b) uF[a][b] = u[a] * Fv[b];
        R c[L::Q];
#pragma unroll
        for (int k = 0; k < L::Q; ++k) {
            if (L::rowclass(k) == kConserved) {
                // s = 0: only the force moment survives (0 for mass, F for momentum).
                R v = R(0);
                if (k == L::jrow(0)) v = Fv[0];
                else if (k == L::jrow(1)) v = Fv[1];
                else if (L::D == 3 && k == L::jrow(2)) v = Fv[2];
                c[k] = v * R(P.mrt.inv_n[k]);
            } else {
                c[k] = R(P.mrt.cr[k]) * (mequil<L, R>(k, rho, rho0, u, uu) - m[k])
                     + R(P.mrt.cs[k]) * msource<L, R>(k, Fv, uF, uf);
            }
        }
        minverse_add<R>(c, f);
    } else {
        const R om = R(P.omega);
        const R fo = R(1) - R(0.5) * om;
#pragma unroll
        for (int q = 0; q < L::Q; ++q) {
            const R eu = R(L::ex(q)) * u[0] + R(L::ey(q)) * u[1] + R(L::ez(q)) * u[2];
            const R ef = R(L::ex(q)) * Fv[0] + R(L::ey(q)) * Fv[1] + R(L::ez(q)) * Fv[2];
            const R wq = R(w<L>(q));
            const R feq = wq * (rho + rho0 * (R(3) * eu + R(4.5) * eu * eu - R(1.5) * usq));
            const R src = wq * (R(3) * (ef - uf) + R(9) * eu * ef);
            f[q] += (feq - f[q]) * om + fo * src;
        }
    }
#pragma unroll
    for (int q = 0; q < L::Q; ++q) S::store(fout + (size_t)q * g.nfp + i, f[q], q, rho0);
}

// t = 0 populations of SCSP::initialize (scsp.cpp:116-134):
// f_q = w_q rho0 - 1.5 w_q (e_q . F).
template <class L, class S>
__global__ void scsp_init(const Grid g, const Force F, double rho0, typename S::T* __restrict__ f)
{
    using R = typename S::R;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.nf) return;
    double Fv[3];
    if (F.uniform) { Fv[0] = F.fx; Fv[1] = F.fy; Fv[2] = F.fz; }
    else { const double* lf = F.label_force + 3 * F.label[i]; Fv[0] = lf[0]; Fv[1] = lf[1]; Fv[2] = lf[2]; }
#pragma unroll
    for (int q = 0; q < L::Q; ++q) {
        const double wq = L::w36f(q) / 36.0;
        // Same operand order as the reference: w*rho, then -= 1.5*w*ef.
        double ef = 0.0;
        if (L::D == 3) ef = L::ez(q) * Fv[2];
        ef += L::ey(q) * Fv[1];
        ef += L::ex(q) * Fv[0];
        double v = wq * rho0;
        v -= 1.5 * wq * ef;
        S::store(f + (size_t)q * g.nfp + i, S::shifted ? R(v - wq * rho0) : R(v), q, R(rho0));
    }
}

}  // namespace lbf
