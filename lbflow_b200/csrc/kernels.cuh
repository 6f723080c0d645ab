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

namespace lbf {

// Device error word bits (the reference's throw sites).
enum : uint32_t {
    kErrDensity   = 1u << 0,  // non-finite or non-positive density (scsp.cpp:144-145; colorfluid.cpp:255-257)
    kErrComponent = 1u << 1,  // negative component density (colorfluid.cpp:258-259)
    kErrTau       = 1u << 2,  // local relaxation time <= 0.5 (colorfluid.cpp:269-270)
    kErrVelocity  = 1u << 3,  // non-finite velocity (colorfluid.cpp:282-283)
    kErrOutput    = 1u << 4,  // non-finite population in a dense checkpoint copy (simulator.cpp:327-333)
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
    static constexpr bool blocked = false;
    static constexpr bool dither = false;
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
// Stochastic rounding of a float to a narrower float format that keeps the
// float's exponent field layout: `drop` low mantissa bits are discarded;
// adding `drop` random bits before truncating rounds up with probability
// equal to the discarded fraction, so the stored value is unbiased.  This
// keeps slow modes whose per-step change is below half a unit in the last
// place evolving, where round-to-nearest would freeze them.
__device__ __forceinline__ float dither_bits(float x, uint32_t r, int drop)
{
    return __uint_as_float(__float_as_uint(x) + (r >> (32 - drop)));
}

// Stochastic rounding of two floats to a 16-bit pair in one instruction
// (cvt.rs, sm_100a): the low half (lo) takes the random bits 0..12 of rbits
// for IEEE half, 0..15 for bfloat16; the high half (hi) bits 16..28 / 16..31.
// A value rounds away from zero with probability equal to the discarded
// fraction (subnormals included); satfinite saturates at the largest finite
// value, as truncation does.
__device__ __forceinline__ uint32_t pack_sr(__half, float hi, float lo, uint32_t rbits)
{
    uint32_t d;
    asm("cvt.rs.satfinite.f16x2.f32 %0, %1, %2, %3;" : "=r"(d) : "f"(hi), "f"(lo), "r"(rbits));
    return d;
}
__device__ __forceinline__ uint32_t pack_sr(__nv_bfloat16, float hi, float lo, uint32_t rbits)
{
    uint32_t d;
    asm("cvt.rs.satfinite.bf16x2.f32 %0, %1, %2, %3;" : "=r"(d) : "f"(hi), "f"(lo), "r"(rbits));
    return d;
}

// Shifted 16-bit float storage (H: __half or __nv_bfloat16).
template <class L, class H> struct StoreShifted16 {
    static constexpr bool blocked = false;
    static constexpr bool dither = true;
    using T = H;
    using R = float;
    static constexpr bool shifted = true;
    // The scaling product is rounded on its own (never fused into the sums
    // that consume it), so every kernel inlining this load -- the single
    // and the batched step -- computes bitwise the same fields.
    __device__ static R load(const T* p, int q, R)
    {
        return __fmul_rn(float(__ldg(p)), ShiftScale<L>::inv(q));
    }
    __device__ static void store(T* p, R v, int q, R) { *p = T(v * ShiftScale<L>::scale(q)); }
    // Directions qa (low half) and qb (high half) rounded together; rbits
    // carries 16 random bits for each.
    __device__ static void store_sr2(T* pa, T* pb, R va, R vb, int qa, int qb, uint32_t rbits)
    {
        const uint32_t d = pack_sr(H(0.0f), vb * ShiftScale<L>::scale(qb), va * ShiftScale<L>::scale(qa), rbits);
        *reinterpret_cast<uint16_t*>(pa) = (uint16_t)d;
        *reinterpret_cast<uint16_t*>(pb) = (uint16_t)(d >> 16);
    }
    __device__ static void store_sr1(T* p, R v, int q, uint32_t rbits)
    {
        *reinterpret_cast<uint16_t*>(p) = (uint16_t)pack_sr(H(0.0f), 0.0f, v * ShiftScale<L>::scale(q), rbits);
    }
};
template <class L> using StoreF16 = StoreShifted16<L, __half>;
template <class L> using StoreBF16 = StoreShifted16<L, __nv_bfloat16>;
template <class L> struct StoreF32 {
    static constexpr bool blocked = false;
    static constexpr bool dither = false;
    using T = float;
    using R = float;
    static constexpr bool shifted = true;
    __device__ static R load(const T* p, int, R) { return __ldg(p); }
    __device__ static void store(T* p, R v, int, R) { *p = v; }
};

// Full (unshifted) populations in FP32 with FP32 arithmetic.
struct StoreF32Full {
    static constexpr bool blocked = false;
    static constexpr bool dither = false;
    using T = float;
    using R = float;
    static constexpr bool shifted = false;
    __device__ static R load(const T* p, int, R) { return __ldg(p); }
    __device__ static void store(T* p, R v, int, R) { *p = v; }
};

// Block-scaled 16-bit deviations: per node, x_q = (f_q - w_q rho0) / w_q is
// stored as the int16 mantissa s_q = round(x_q * 2^(15 - E)), with one
// exponent E per node chosen so that max_q |x_q| < 2^E.  The values that
// carry a node's velocity keep 15 bits relative to the node's largest
// deviation (IEEE FP16 keeps 11 relative to each value), for one extra byte
// per node.  Arithmetic in FP32.
__device__ __forceinline__ float pow2f(int e) { return __int_as_float((e + 127) << 23); }
template <class L> struct StoreBFP16 {
    using T = int16_t;
    using R = float;
    static constexpr bool shifted = true;
    static constexpr bool blocked = true;
    static constexpr bool dither = false;
    static constexpr int kEmin = -100, kEmax = 100;
    __device__ static R load(const T*, int, R) { return R(0); }
    __device__ static void store(T*, R, int, R) {}
    __device__ static R load_blk(const T* p, int q, int e)
    { return (float)__ldg(p) * (pow2f(e - 15) * ((float)L::w36f(q) / 36.0f)); }
    // Exponent of a node whose largest |x_q| is m.
    __device__ static int exponent(float m)
    {
        if (!(m > 0.0f)) return kEmin;
        int e = ((__float_as_int(m) >> 23) & 0xff) - 126;
        return e < kEmin ? kEmin : (e > kEmax ? kEmax : e);
    }
    template <int Q>
    __device__ static void store_blk(T* base, size_t nfp, uint32_t i, const R (&g)[Q], int8_t* eout)
    {
        float x[Q];
        float m = 0.0f;
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            x[q] = g[q] * (36.0f / (float)L::w36f(q));
            m = fmaxf(m, fabsf(x[q]));
        }
        const int e = exponent(m);
        const float sc = pow2f(15 - e);
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            int v = __float2int_rn(x[q] * sc);
            v = v > 32767 ? 32767 : (v < -32767 ? -32767 : v);
            base[(uint32_t)q * (uint32_t)nfp + i] = (T)v;
        }
        eout[i] = (int8_t)e;
    }
};

// ---- gather: pull-stream with halfway bounce-back ----------------------------
// src[q] receives f_q(x - e_q) after streaming, or f*_{op q}(x) when the
// upstream voxel is solid.  nbr[q] (q >= 1) records the compact index of the
// voxel x + e_q (the pull source of op q) or UINT32_MAX when it is solid.
template <class S>
__device__ __forceinline__ typename S::R load_pop(const typename S::T* p, int q, typename S::R rho0,
                                                  const int8_t* __restrict__ ein, uint32_t src)
{
    if constexpr (S::blocked) return S::load_blk(p, q, (int)__ldg(&ein[src]));
    else return S::load(p, q, rho0);
}

// Pull sources of every direction: src[q] = compact index of voxel x - e_q
// and bit q of the returned mask set when that voxel is fluid.  The sources
// lie in (at most) nine x-rows (y - ey, z - ez); each row's occupancy word
// at x is loaded once for the sources at x.  The sources at x - 1 and x + 1
// (periodic in x) come in two forms:
//   UNIFORM = true:  looked up in the word that holds them (the same word
//                    except at a word boundary or the wrap) by one
//                    branch-free formula, so a warp's lanes never split;
//   UNIFORM = false: read from the row word at x, with a separate lookup only
//                    at a word boundary or the wrap (fewer loads and
//                    registers, but most warps take both sides of the split).
// The indices are the same either way.  Which is faster depends on the
// kernel: the FP64 single-geometry step (latency-bound at 72 registers) runs
// 9 % slower uniform; the FP32-arithmetic steps (issue-bound) run 4-12 %
// faster uniform (FP16 storage 28,230 -> 31,230 fluid MLUPS on the 256^3
// cube) and the batched FP64 step 5 % faster.
template <class L, bool UNIFORM>
__device__ __forceinline__ uint32_t pull_sources(const Grid& g, int x, int y, int z, uint32_t (&src)[L::Q])
{
    const int b = x & 31;
    const int wx = x >> 5;
    const uint32_t below = (1u << b) - 1u;
    const int xl = x == 0 ? g.nx - 1 : x - 1;
    const int xr = x + 1 == g.nx ? 0 : x + 1;
    const int wl = xl >> 5, wr = xr >> 5;
    const uint32_t bl = xl & 31, br = xr & 31;
    const uint32_t belowl = (1u << bl) - 1u, belowr = (1u << br) - 1u;
    uint32_t mask = 0;
    uint32_t rbase[9], ridx[9], rbits[9];
    bool rload[9] = {false, false, false, false, false, false, false, false, false};
#pragma unroll
    for (int q = 1; q < L::Q; ++q) rload[(1 - L::ey(q)) * 3 + (1 - L::ez(q))] = true;
#pragma unroll
    for (int r = 0; r < 9; ++r) {
        if (!rload[r]) continue;
        const int dy = r / 3 - 1, dz = r % 3 - 1;
        const int yy = dy == 0 ? y : wrap(y + dy, g.ny);
        const int zz = (L::D == 2 || dz == 0) ? z : wrap(z + dz, g.nz);
        rbase[r] = ((uint32_t)zz * (uint32_t)g.ny + (uint32_t)yy) * (uint32_t)g.W;
        const uint2 e = __ldg(&g.occ[rbase[r] + wx]);
        rbits[r] = e.x;
        ridx[r] = e.y + __popc(e.x & below);
    }
#pragma unroll
    for (int q = 1; q < L::Q; ++q) {
        const int r = (1 - L::ey(q)) * 3 + (1 - L::ez(q));
        const int dx = -L::ex(q);
        const uint32_t bits = rbits[r];
        uint32_t idx, fl;
        if (dx == 0) {
            fl = (bits >> b) & 1u;
            idx = ridx[r];
        } else if (UNIFORM) {
            const uint2 e = __ldg(&g.occ[rbase[r] + (dx < 0 ? wl : wr)]);
            fl = (e.x >> (dx < 0 ? bl : br)) & 1u;
            idx = e.y + __popc(e.x & (dx < 0 ? belowl : belowr));
        } else if (dx < 0 && b > 0) {
            fl = (bits >> (b - 1)) & 1u;
            idx = ridx[r] - fl;
        } else if (dx > 0 && b < 31 && x + 1 < g.nx) {
            fl = (bits >> (b + 1)) & 1u;
            idx = ridx[r] + ((bits >> b) & 1u);
        } else {
            const uint2 e = __ldg(&g.occ[rbase[r] + (dx < 0 ? wl : wr)]);
            const uint32_t sb = dx < 0 ? bl : br;
            fl = (e.x >> sb) & 1u;
            idx = e.y + __popc(e.x & ((1u << sb) - 1u));
        }
        src[q] = idx;
        mask |= fl << q;
    }
    return mask;
}

template <class L, class S, bool PULL, bool UNIFORM = (sizeof(typename S::R) == 4)>
__device__ __forceinline__ void gather(const Grid& g, const typename S::T* __restrict__ fin,
                                       uint32_t i, int x, int y, int z,
                                       typename S::R (&f)[L::Q], uint32_t (&nbr)[L::Q],
                                       typename S::R rho0, const int8_t* __restrict__ ein = nullptr)
{
    // Element offsets stay 32-bit (phases * Q * nfp < 2^32 is checked at
    // creation); only the final address is 64-bit.
    const uint32_t nfp = g.nfp;
    f[0] = load_pop<S>(fin + i, 0, rho0, ein, i);
    nbr[0] = i;
    if (!PULL) {
#pragma unroll
        for (int q = 1; q < L::Q; ++q) { f[q] = load_pop<S>(fin + (q * nfp + i), q, rho0, ein, i); nbr[q] = 0; }
        return;
    }
    uint32_t src[L::Q];
    const uint32_t mask = pull_sources<L, UNIFORM>(g, x, y, z, src);
#pragma unroll
    for (int q = 1; q < L::Q; ++q) {
        const bool fluid = (mask >> q) & 1u;
        const uint32_t node = fluid ? src[q] : i;
        nbr[L::op(q)] = fluid ? src[q] : 0xffffffffu;
        const uint32_t off = (fluid ? (uint32_t)q : (uint32_t)L::op(q)) * nfp + node;
        f[q] = load_pop<S>(fin + off, q, rho0, ein, node);
    }
}

// ---- collision: the reference's MRT as a two-relaxation-time update ---------
// In the legacy D2Q9/D3Q19 spectrum (simulator.cpp:209-214) every
// non-conserved even moment relaxes at s+ = 1/tau and every non-conserved odd
// moment at s- = 8(2 - s+)/(8 - s+).  Because (f - feq) has zero mass moment
// and momentum moment -F/2 (the half-force velocity shift), and the Guo term
// is scaled by (1 - s/2), the conserved rows come out the same as with s = 0.
// So M^-1 S M (feq - f) + M^-1 (I - S/2) M S_guo equals, per opposite pair,
//   f_q  += -s+ (f+ - feq+) + (1 - s+/2) src+  -  s- (f- - feq-) + (1 - s-/2) src-
//   f_q' +=   ... same even part ...           +  s- (f- - feq-) - (1 - s-/2) src-
// with f+- = (f_q +- f_q')/2 (verified against the reference's matrices to
// round-off in tests/test_moments.py).  SRT is the case s+ = s-.
struct Trt { double sp, sm; };

// One fused pass over the opposite pairs.  The equilibrium is written as
//   feq_q = A_q + w_q (B + C (e.u)^2) + w_q K (e.u)
// (single phase: A = 0, B = rho - 1.5 rho0 u^2, C = 4.5 rho0, K = 3 rho0;
//  color: A = feq_u0, B = -1.5 rho u^2, C = 4.5 rho, K = 3 rho) and the Guo
// source as w_q (3 (e.F - u.F) + 9 (e.u)(e.F)).
template <class L, bool HAS_A>
__device__ __forceinline__ void collide_trt_x2(float (&f)[L::Q], const float* A, float B, float C, float K,
                                               const float (&u)[3], const float (&F)[3], float uf, float sp,
                                               float sm);

template <class L, class R, bool HAS_A>
__device__ __forceinline__ void collide_trt(R (&f)[L::Q], const R* A, R B, R C, R K,
                                            const R (&u)[3], const R (&F)[3], R uf, R sp, R sm)
{
    if constexpr (sizeof(R) == 4) {
        collide_trt_x2<L, HAS_A>(f, A, B, C, K, u, F, uf, sp, sm);
        return;
    }
    const R hp = R(1) - R(0.5) * sp, hm = R(1) - R(0.5) * sm;
    {
        const R w0 = R(w<L>(0));
        const R feq0 = (HAS_A ? A[0] : R(0)) + w0 * B;
        f[0] += -sp * (f[0] - feq0) + hp * (w0 * (R(-3) * uf));
    }
#pragma unroll
    for (int p = 0; p < L::NPAIR; ++p) {
        const int q = L::pair(p), o = L::op(q);
        const R eu = R(L::ex(q)) * u[0] + R(L::ey(q)) * u[1] + R(L::ez(q)) * u[2];
        const R ef = R(L::ex(q)) * F[0] + R(L::ey(q)) * F[1] + R(L::ez(q)) * F[2];
        const R wq = R(w<L>(q));
        const R feqp = (HAS_A ? A[q] : R(0)) + wq * (B + C * eu * eu);
        const R feqm = wq * K * eu;
        const R fp = R(0.5) * (f[q] + f[o]);
        const R fm = R(0.5) * (f[q] - f[o]);
        const R ev = -sp * (fp - feqp) + hp * (wq * (R(9) * eu * ef - R(3) * uf));
        const R od = -sm * (fm - feqm) + hm * (wq * R(3) * ef);
        f[q] += ev + od;
        f[o] += ev - od;
    }
}

// e_q . v with the direction's components known at compile time.
template <class L> __device__ __forceinline__ float dot_e(int q, const float (&v)[3])
{
    float s = 0.0f;
    if (L::ex(q)) s = L::ex(q) > 0 ? v[0] : -v[0];
    if (L::ey(q)) s = L::ey(q) > 0 ? s + v[1] : s - v[1];
    if (L::ez(q)) s = L::ez(q) > 0 ? s + v[2] : s - v[2];
    return s;
}
__device__ __forceinline__ float2 neg2(float2 a) { return make_float2(-a.x, -a.y); }
__device__ __forceinline__ float2 dup2(float a) { return make_float2(a, a); }

// The two-rate update in FP32 arithmetic, two opposite pairs per instruction
// with the packed FP32 operations of sm_100 (__ffma2_rn, __fadd2_rn,
// __fmul2_rn: each lane rounds as the scalar operation does).  The FP32
// storages are issue-bound, and this halves the collision's share of the
// issued instructions.
template <class L, bool HAS_A>
__device__ __forceinline__ void collide_trt_x2(float (&f)[L::Q], const float* A, float B, float C, float K,
                                               const float (&u)[3], const float (&F)[3], float uf, float sp,
                                               float sm)
{
    const float hp = 1.0f - 0.5f * sp, hm = 1.0f - 0.5f * sm;
    {
        const float w0 = float(w<L>(0));
        const float feq0 = (HAS_A ? A[0] : 0.0f) + w0 * B;
        f[0] += -sp * (f[0] - feq0) + hp * (w0 * (-3.0f * uf));
    }
    const float2 B2 = dup2(B), C2 = dup2(C), K2 = dup2(K), nsp = dup2(-sp), nsm = dup2(-sm);
    const float2 hp2 = dup2(hp), hm2 = dup2(hm), m3uf = dup2(-3.0f * uf), half = dup2(0.5f), nine = dup2(9.0f);
#pragma unroll
    for (int p = 0; p < L::NPAIR; p += 2) {
        if (p + 1 < L::NPAIR) {
            const int qa = L::pair(p), oa = L::op(qa), qb = L::pair(p + 1), ob = L::op(qb);
            const float2 eu = make_float2(dot_e<L>(qa, u), dot_e<L>(qb, u));
            const float2 ef = make_float2(dot_e<L>(qa, F), dot_e<L>(qb, F));
            const float2 wq = make_float2(float(w<L>(qa)), float(w<L>(qb)));
            const float2 w3 = make_float2(float(3.0 * w<L>(qa)), float(3.0 * w<L>(qb)));
            float2 feqp = __fmul2_rn(wq, __ffma2_rn(C2, __fmul2_rn(eu, eu), B2));
            if (HAS_A) feqp = __fadd2_rn(make_float2(A[qa], A[qb]), feqp);
            const float2 feqm = __fmul2_rn(__fmul2_rn(wq, K2), eu);
            const float2 fq = make_float2(f[qa], f[qb]), fo = make_float2(f[oa], f[ob]);
            const float2 fp = __fmul2_rn(half, __fadd2_rn(fq, fo));
            const float2 fm = __fmul2_rn(half, __fadd2_rn(fq, neg2(fo)));
            const float2 srcp = __fmul2_rn(__fmul2_rn(hp2, wq), __ffma2_rn(nine, __fmul2_rn(eu, ef), m3uf));
            const float2 srcm = __fmul2_rn(__fmul2_rn(hm2, w3), ef);
            const float2 ev = __ffma2_rn(nsp, __fadd2_rn(fp, neg2(feqp)), srcp);
            const float2 od = __ffma2_rn(nsm, __fadd2_rn(fm, neg2(feqm)), srcm);
            const float2 nq = __fadd2_rn(fq, __fadd2_rn(ev, od));
            const float2 no = __fadd2_rn(fo, __fadd2_rn(ev, neg2(od)));
            f[qa] = nq.x; f[qb] = nq.y;
            f[oa] = no.x; f[ob] = no.y;
        } else {
            const int q = L::pair(p), o = L::op(q);
            const float eu = dot_e<L>(q, u), ef = dot_e<L>(q, F), wq = float(w<L>(q));
            const float feqp = (HAS_A ? A[q] : 0.0f) + wq * (B + C * eu * eu);
            const float feqm = wq * K * eu;
            const float fp = 0.5f * (f[q] + f[o]);
            const float fm = 0.5f * (f[q] - f[o]);
            const float ev = -sp * (fp - feqp) + hp * (wq * (9.0f * eu * ef - 3.0f * uf));
            const float od = -sm * (fm - feqm) + hm * (wq * 3.0f * ef);
            f[q] += ev + od;
            f[o] += ev - od;
        }
    }
}

// ---- single-phase step (SCSP) ----------------------------------------------------
// One launch = Simulator::streaming + bounceBack (simulator.cpp:73-111),
// SCSP::calcMacroVar + bodyForce (scsp.cpp:136-175) and SCSP::equilSRT /
// equilMRT (scsp.cpp:374-464) for every fluid node.  PULL = false is the t = 0
// collision of SCSP::Run (scsp.cpp:60-71), which reads the node's own values.
struct ScspParams {
    double rho0;       // reference density (incompressible form, lbcfg.h:13)
    double inv_rho0;
    Trt rate;          // SRT: s+ = s- = 1/tau; MRT: legacy spectrum
    int mrt = 0;       // MRT: mass and momentum rows are not relaxed (rate 0)
    uint32_t seed = 0; // non-zero: stochastic rounding of 16-bit float storage (per-step seed)
    uint32_t node0 = 0; // first node of the geometry: rounding streams follow the geometry's own node order
    int reverse = 0;    // blocks in descending node order (alternated every step; see scsp_step)
};

// Integer hash (lowbias32 of C. Wellons) seeding the per-node rounding stream.
__device__ __forceinline__ uint32_t hash32(uint32_t x)
{
    x ^= x >> 16; x *= 0x7feb352du;
    x ^= x >> 15; x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}

// Update of one fluid node i (the body of scsp_step, shared with the batched
// kernel).
template <class L, class S, bool PULL, bool UNIFORM = (sizeof(typename S::R) == 4)>
__device__ __forceinline__ void scsp_update(const Grid& g, const Force& F, const ScspParams& P,
                                            const typename S::T* __restrict__ fin,
                                            typename S::T* __restrict__ fout, const uint32_t i,
                                            const Macros& mo, const int out, uint32_t* __restrict__ err,
                                            const int8_t* __restrict__ ein, int8_t* __restrict__ eout)
{
    using R = typename S::R;
    int x, y, z;
    unpack(__ldg(&g.coord[i]), x, y, z);
    const R rho0 = R(P.rho0);
    R f[L::Q];
    uint32_t nbr[L::Q];
    gather<L, S, PULL, UNIFORM>(g, fin, i, x, y, z, f, nbr, rho0, ein);

    R Fv[3];
    if (F.uniform) { Fv[0] = R(F.fx); Fv[1] = R(F.fy); Fv[2] = R(F.fz); }
    else {
        const double* lf = F.label_force + 3 * __ldg(&F.label[i]);
        Fv[0] = R(lf[0]); Fv[1] = R(lf[1]); Fv[2] = R(lf[2]);
    }

    // SCSP::calcMacroVar + bodyForce: rho = sum f, u = sum e f / rho0 + F/(2 rho0).
    R rho = f[0];
#pragma unroll
    for (int q = 1; q < L::Q; ++q) rho += f[q];
    R j[3] = {R(0), R(0), R(0)};
#pragma unroll
    for (int p = 0; p < L::NPAIR; ++p) {
        const int q = L::pair(p);
        const R b = f[q] - f[L::op(q)];
        if (L::ex(q)) j[0] += R(L::ex(q)) * b;
        if (L::ey(q)) j[1] += R(L::ey(q)) * b;
        if (L::ez(q)) j[2] += R(L::ez(q)) * b;
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

    // Equilibrium w (rho + rho0 (3 e.u + 4.5 (e.u)^2 - 1.5 u^2)) (scsp.cpp:398-402)
    // and Guo source (simulator.cpp:230-246), relaxed in the two-rate form.
    collide_trt<L, R, false>(f, nullptr, rho - rho0 * R(1.5) * usq, rho0 * R(4.5), rho0 * R(3),
                             u, Fv, uf, R(P.rate.sp), R(P.rate.sm));

    if constexpr (S::blocked) {
        S::store_blk(fout, g.nfp, i, f, eout);
    } else if constexpr (S::dither) {
        if (P.seed) {
            // One linear congruential stream per node and step, one draw per
            // direction; the high 16 bits of each draw are its rounding
            // offsets (a pair of directions takes the high halves of two
            // draws, the first in bits 0..15).
            uint32_t r = hash32((i - P.node0) * 0x9e3779b9u + P.seed);
#pragma unroll
            for (int q = 0; q < L::Q; q += 2) {
                r = r * 1664525u + 1013904223u;
                const uint32_t ra = r;
                if (q + 1 < L::Q) {
                    r = r * 1664525u + 1013904223u;
                    S::store_sr2(fout + (q * g.nfp + i), fout + ((q + 1) * g.nfp + i), f[q], f[q + 1], q, q + 1,
                                 __byte_perm(ra, r, 0x7632));
                } else {
                    S::store_sr1(fout + (q * g.nfp + i), f[q], q, ra >> 16);
                }
            }
        } else {
#pragma unroll
            for (int q = 0; q < L::Q; ++q) S::store(fout + (q * g.nfp + i), f[q], q, rho0);
        }
    } else {
#pragma unroll
        for (int q = 0; q < L::Q; ++q) S::store(fout + (q * g.nfp + i), f[q], q, rho0);
    }
}

// Resident 128-thread blocks per SM the step kernel is compiled for.  FP64:
// seven (at most 72 registers per thread); the step is latency-bound on the
// dependent occupancy -> population gather, and 28 warps per SM hide more of
// it than 16 at the 126 registers it takes unbounded (256^3 cube: 18,100 ->
// 19,270 fluid MLUPS with 32 bytes of spill; eight blocks spill 252 bytes and
// fall to 12,800).  FP32 arithmetic (the reduced-precision storages): nine
// (56 registers, no spill); capped at seven they take 72 registers and run
// slower (FP32 storage 28,650 -> 26,600, FP16 25,050 -> 24,700).
template <class S> struct StepBlocks { static constexpr int value = 9; };
template <> struct StepBlocks<StoreF64> { static constexpr int value = 7; };

template <class L, class S, bool PULL>
__global__ void __launch_bounds__(128, StepBlocks<S>::value)
scsp_step(const Grid g, const Force F, const ScspParams P,
          const typename S::T* __restrict__ fin, typename S::T* __restrict__ fout,
          Macros mo, const int out, uint32_t* __restrict__ err,
          const int8_t* __restrict__ ein, int8_t* __restrict__ eout)
{
    // The node order alternates between steps: a step that runs in the
    // opposite order to the previous one starts with the nodes whose
    // populations that step wrote last, which are still in L2.
    const uint32_t blk = P.reverse ? gridDim.x - 1 - blockIdx.x : blockIdx.x;
    const uint32_t i = blk * blockDim.x + threadIdx.x;
    if (i >= g.nf) return;
    scsp_update<L, S, PULL>(g, F, P, fin, fout, i, mo, out, err, ein, eout);
}

// ---- Zou-He pressure (PB) and velocity (VB) boundaries ---------------------------
// SCSP::zouHeBoundary (scsp.cpp:188-275) runs between streaming and the
// macroscopic update; PB/VB voxels then skip calcMacroVar (scsp.cpp:136-160)
// and collide with the density and velocity it set, under zero force
// (forceForIndex is zero for non-GV labels, simulator.cpp:218-228).  The main
// step kernel treats every fluid node alike; this pass, launched right after
// it on the same stream, recomputes the boundary nodes from the same input
// buffer and overwrites their populations and fields.
struct ZouHe {
    uint32_t n;                          // boundary nodes
    const uint32_t* __restrict__ node;   // compact node index
    const uint32_t* __restrict__ code;   // phase << 16 | kind << 8 | dir (dir 1..2D, the lattice direction)
    const double* __restrict__ value;    // PB density or VB speed
    double* num;                         // two-phase only: per-node adjacent-history numerator
};
enum : uint32_t { kZouHeVB = 1, kZouHePB = 2 };

// Axis (0 = x, 1 = y, 2 = z) and sign of the axial lattice direction DIR.
template <class L, int DIR> struct ZouHeDir {
    static constexpr int A = L::ex(DIR) != 0 ? 0 : (L::ey(DIR) != 0 ? 1 : 2);
    static constexpr int SG = comp<L>(DIR, A);
};

// Density and velocity of the boundary node from the known populations, then
// the unknown populations (those with the boundary direction's sign along its
// axis) rebuilt from their opposites:
//   VB: u_a = s v, rho = (2 sum f[opposite side] + sum f[normal plane]) / (1 - u_a)
//   PB: rho = p,   u_a = -s (that sum / p - 1)
//   f_q = f_op(q) + s 6 w_q rho u_a - 1/2 sum_{n in plane} (+-) f_n
// (6 w_q = wiT of simulator.cpp:28 at latticeSpeed 1)
// where the last sum runs over the normal-plane directions sharing a
// transverse component with q, + when the components agree.  With shifted
// storage (f - w rho0) the sums are rewritten so that only deviations are
// formed: the plane and opposite-side weights add up to 1 and the transverse
// sum is unchanged because mirrored directions have equal weights.
// Returns rho (a deviation when shifted) and the full density in dens.
template <class L, class S, int DIR>
__device__ __forceinline__ typename S::R zou_he_node(typename S::R (&f)[L::Q], uint32_t kind, double val,
                                                     double rho0, typename S::R (&u)[3], double& dens)
{
    using R = typename S::R;
    constexpr int A = ZouHeDir<L, DIR>::A, SG = ZouHeDir<L, DIR>::SG;
    R sum = R(0);
#pragma unroll
    for (int q = 1; q < L::Q; ++q)
        if (comp<L>(q, A) == -SG) sum += f[q] + f[q];
#pragma unroll
    for (int q = 0; q < L::Q; ++q)
        if (comp<L>(q, A) == 0) sum += f[q];
    R rho, ua;
    if (kind == kZouHeVB) {
        const double vel = SG > 0 ? val : -val;
        const R inv = R(1.0 / (1.0 - vel));
        ua = R(vel);
        if constexpr (S::shifted) { rho = (sum + R(rho0 * vel)) * inv; dens = rho0 + (double)rho; }
        else { rho = sum * inv; dens = (double)rho; }
    } else {
        R s;
        if constexpr (S::shifted) { rho = R(val - rho0); s = (sum - rho) / R(val); }
        else { rho = R(val); s = sum / R(val) - R(1); }
        ua = SG > 0 ? -s : s;
        dens = val;
    }
    const R rho_full = R(dens);
    R tr[L::Q];
#pragma unroll
    for (int q = 1; q < L::Q; ++q) {
        if (comp<L>(q, A) != SG) continue;
        R t = R(0);
#pragma unroll
        for (int n = 1; n < L::Q; ++n) {
            if (comp<L>(n, A) != 0) continue;
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                if (d == A || comp<L>(n, d) == 0 || comp<L>(q, d) == 0) continue;
                if (comp<L>(n, d) == comp<L>(q, d)) t += f[n];
                else t -= f[n];
            }
        }
        tr[q] = t;
    }
#pragma unroll
    for (int q = 1; q < L::Q; ++q) {
        if (comp<L>(q, A) != SG) continue;
        f[q] = f[L::op(q)] + R(SG) * R(6.0 * w<L>(q)) * rho_full * ua - tr[q] * R(0.5);
    }
    u[0] = u[1] = u[2] = R(0);
    u[A] = ua;
    return rho;
}

template <class L, class S>
__global__ void __launch_bounds__(128)
scsp_zou_he(const Grid g, const ScspParams P, const ZouHe z,
            const typename S::T* __restrict__ fin, typename S::T* __restrict__ fout,
            Macros mo, const int out, uint32_t* __restrict__ err,
            const int8_t* __restrict__ ein, int8_t* __restrict__ eout)
{
    using R = typename S::R;
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= z.n) return;
    const uint32_t i = __ldg(&z.node[k]);
    const uint32_t code = __ldg(&z.code[k]);
    const double val = __ldg(&z.value[k]);
    int x, y, zc;
    unpack(__ldg(&g.coord[i]), x, y, zc);
    const R rho0 = R(P.rho0);
    R f[L::Q];
    uint32_t nbr[L::Q];
    gather<L, S, true>(g, fin, i, x, y, zc, f, nbr, rho0, ein);

    const uint32_t kind = (code >> 8) & 0xffu;
    R u[3];
    R rho = R(0);
    double dens = 0.0;
    switch (code & 0xffu) {
    case 1: rho = zou_he_node<L, S, 1>(f, kind, val, P.rho0, u, dens); break;
    case 2: rho = zou_he_node<L, S, 2>(f, kind, val, P.rho0, u, dens); break;
    case 3: rho = zou_he_node<L, S, 3>(f, kind, val, P.rho0, u, dens); break;
    case 4: rho = zou_he_node<L, S, 4>(f, kind, val, P.rho0, u, dens); break;
    default:
        if constexpr (L::D == 3) {
            if ((code & 0xffu) == 5) rho = zou_he_node<L, S, 5>(f, kind, val, P.rho0, u, dens);
            else rho = zou_he_node<L, S, 6>(f, kind, val, P.rho0, u, dens);
        }
        break;
    }
    if (!isfinite(dens) || !isfinite((double)u[0] + (double)u[1] + (double)u[2])) atomicOr(err, kErrDensity);

    if (out & (kOutMacros | kOutAdjacent)) {
        // The reference takes the adjacent-step copy after zouHeBoundary of the
        // report step (scsp.cpp:80-81), so at these nodes it equals the reported
        // velocity.
#pragma unroll
        for (int a = 0; a < 3; ++a) mo.uadj[(size_t)a * g.nfp + i] = (double)u[a];
    }
    if (out & kOutMacros) {
        mo.rho0[i] = dens;
#pragma unroll
        for (int a = 0; a < 3; ++a) mo.u[(size_t)a * g.nfp + i] = (double)u[a];
    }

    // The two-rate update relaxes the mass row at s+ and the momentum rows at
    // s-, whereas the reference's MRT leaves them untouched (rate 0,
    // simulator.cpp:209-214).  In the bulk the difference vanishes (feq - f
    // carries no mass and only the momentum the Guo term restores), but here
    // the populations' mass and momentum differ from the prescribed rho and
    // rho0 u, so those two projections of feq - f are taken back out:
    // M^-1 diag(s) M d over the conserved rows is s (sum d) / Q on every
    // direction and s e_q . J / |e_a|^2 with J = sum e d.
    R dmass = R(0), dmom[3] = {R(0), R(0), R(0)};
    if (P.mrt) {
        R sf = f[0];
#pragma unroll
        for (int q = 1; q < L::Q; ++q) sf += f[q];
#pragma unroll
        for (int q = 1; q < L::Q; ++q) {
            if (L::ex(q)) dmom[0] -= R(L::ex(q)) * f[q];
            if (L::ey(q)) dmom[1] -= R(L::ey(q)) * f[q];
            if (L::ez(q)) dmom[2] -= R(L::ez(q)) * f[q];
        }
        dmass = rho - sf;               // sum of feq is rho (a deviation when shifted)
#pragma unroll
        for (int a = 0; a < 3; ++a) dmom[a] += rho0 * u[a];   // sum of e feq is rho0 u
    }
    const R usq = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
    const R F0[3] = {R(0), R(0), R(0)};
    collide_trt<L, R, false>(f, nullptr, rho - rho0 * R(1.5) * usq, rho0 * R(4.5), rho0 * R(3),
                             u, F0, R(0), R(P.rate.sp), R(P.rate.sm));
    if (P.mrt) {
        const R cm = R(P.rate.sp) * dmass / R(L::Q);
        const R cj = R(P.rate.sm) / R(L::D == 3 ? 10 : 6);   // |e_a|^2 over the velocity set
#pragma unroll
        for (int q = 0; q < L::Q; ++q)
            f[q] -= cm + cj * (R(L::ex(q)) * dmom[0] + R(L::ey(q)) * dmom[1] + R(L::ez(q)) * dmom[2]);
    }
    if constexpr (S::blocked) {
        S::store_blk(fout, g.nfp, i, f, eout);
    } else {
#pragma unroll
        for (int q = 0; q < L::Q; ++q) S::store(fout + (q * g.nfp + i), f[q], q, rho0);
    }
}

// t = 0 populations of SCSP::initialize (scsp.cpp:116-134):
// f_q = w_q rho0 - 1.5 w_q (e_q . F).
template <class L, class S>
__global__ void scsp_init(const Grid g, const Force F, double rho0, typename S::T* __restrict__ f,
                          int8_t* __restrict__ eout)
{
    using R = typename S::R;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.nf) return;
    double Fv[3];
    if (F.uniform) { Fv[0] = F.fx; Fv[1] = F.fy; Fv[2] = F.fz; }
    else { const double* lf = F.label_force + 3 * F.label[i]; Fv[0] = lf[0]; Fv[1] = lf[1]; Fv[2] = lf[2]; }
    R vals[L::Q];
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
        vals[q] = S::shifted ? R(v - wq * rho0) : R(v);
    }
    if constexpr (S::blocked) {
        S::store_blk(f, g.nfp, i, vals, eout);
    } else {
#pragma unroll
        for (int q = 0; q < L::Q; ++q) S::store(f + (size_t)q * g.nfp + i, vals[q], q, R(rho0));
    }
}

// Warm start: equilibrium populations of given per-voxel fields.  fields is
// a dense (z, y, x) array of records of `ld` floats: velocity x, y, z (the
// physical velocity, half force included) and density.  The raw momentum is
// rho0 * (u - F / (2 rho0)), as the macroscopic velocity of SCSP::calcMacroVar
// (solver/src/lbm/scsp.cpp:136-175) adds the half force back; the
// populations are the incompressible equilibrium of SCSP::equilSRT
// (scsp.cpp:374-409) at that momentum.
template <class L, class S>
__global__ void scsp_init_eq(const Grid g, const Force F, double rho0, const float* __restrict__ fields,
                             uint32_t ld, typename S::T* __restrict__ f, int8_t* __restrict__ eout)
{
    using R = typename S::R;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.nf) return;
    const uint32_t c = g.coord[i];
    const size_t vox = ((size_t)(c >> 22) * g.ny + ((c >> 11) & 0x7FFu)) * g.nx + (c & 0x7FFu);
    const float* r = fields + vox * ld;
    double Fv[3];
    if (F.uniform) { Fv[0] = F.fx; Fv[1] = F.fy; Fv[2] = F.fz; }
    else { const double* lf = F.label_force + 3 * F.label[i]; Fv[0] = lf[0]; Fv[1] = lf[1]; Fv[2] = lf[2]; }
    double v[3];
    for (int d = 0; d < 3; ++d) v[d] = (double)r[d] - Fv[d] / (2.0 * rho0);
    if (L::D == 2) v[2] = 0.0;
    const double rho = (double)r[3];
    const double vv = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
    R vals[L::Q];
#pragma unroll
    for (int q = 0; q < L::Q; ++q) {
        const double wq = L::w36f(q) / 36.0;
        double ev = L::ex(q) * v[0] + L::ey(q) * v[1];
        if (L::D == 3) ev += L::ez(q) * v[2];
        const double fq = wq * (rho + rho0 * (3.0 * ev + 4.5 * ev * ev - 1.5 * vv));
        vals[q] = S::shifted ? R(fq - wq * rho0) : R(fq);
    }
    if constexpr (S::blocked) {
        S::store_blk(f, g.nfp, i, vals, eout);
    } else {
#pragma unroll
        for (int q = 0; q < L::Q; ++q) S::store(f + (size_t)q * g.nfp + i, vals[q], q, R(rho0));
    }
}

// Density increment of a running state: f_q += w_q drho(voxel) at every fluid
// node, in place on the current populations (shifted storage holds f - w rho0,
// so the increment is the same).  Momentum is unchanged.
template <class L, class S>
__global__ void scsp_add_density(const Grid g, const float* __restrict__ drho, typename S::T* __restrict__ f,
                                 int8_t* __restrict__ ex, double rho0)
{
    using R = typename S::R;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.nf) return;
    const uint32_t c = g.coord[i];
    const size_t vox = ((size_t)(c >> 22) * g.ny + ((c >> 11) & 0x7FFu)) * g.nx + (c & 0x7FFu);
    const R d = R(drho[vox]);
    R vals[L::Q];
#pragma unroll
    for (int q = 0; q < L::Q; ++q) {
        const R wq = R(L::w36f(q)) / R(36);
        if constexpr (S::blocked) vals[q] = S::load_blk(f + (size_t)q * g.nfp + i, q, (int)ex[i]) + wq * d;
        else vals[q] = S::load(f + (size_t)q * g.nfp + i, q, R(rho0)) + wq * d;
    }
    if constexpr (S::blocked) {
        S::store_blk(f, g.nfp, i, vals, ex);
    } else {
#pragma unroll
        for (int q = 0; q < L::Q; ++q) S::store(f + (size_t)q * g.nfp + i, vals[q], q, R(rho0));
    }
}

}  // namespace lbf
