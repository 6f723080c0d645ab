// Two-phase color-gradient kernels (ColorFluid, solver/src/lbm/colorfluid.cpp).
//
// A step needs the phase field phi = (rho0 - rho1)/rho of every neighbour
// after streaming, so it runs as two launches over the fluid nodes:
//   pass 1  color_phase:   pull both components (with bounce-back), write the
//                          two component densities (compact) and phi (dense,
//                          per voxel);
//   pass 2  color_collide: color gradient from the dense phi (legacy interior
//           stencil or the geometric wall rotation), pull again into the
//           total distribution, macros, collision of the total,
//           perturbation and recoloring.
// Solid voxels read as phi = 86 (SOLID_DENS_N, colorfluid.cpp:49).
#pragma once
#include <type_traits>
#include "kernels.cuh"

namespace lbf {

struct ColorParams {
    double ai[2][19];      // phase weights (ColorFluid::initPhi, colorfluid.cpp:1131-1150)
    double rho_ref[2];     // reference densities
    double relax0, relax1; // tau_k / 2 (colorfluid.cpp:241-242)
    int uniform_tau;       // tau0 == tau1: fixed MRT rates (colorfluid.cpp:317-322)
    Trt rate;              // the uniform rates (used when uniform_tau)
    double ak;             // 2.25 sigma (colorfluid.cpp:305)
    double beta;           // recoloring parameter
    uint32_t seed;         // 16-bit storage: per-step seed of the stochastic rounding (0: round to nearest)
};

// ---- 16-bit storage of the two components ---------------------------------------
// The two components are kept as the total fT_q = f0_q + f1_q and the share
// r_q = f0_q / fT_q of component 0:
//   block 0: (fT_q - w_q rho0) * 4096 / w_q in IEEE half or bfloat16 -- the
//            single-phase shifted form, so the velocity-carrying deviations
//            keep their precision;
//   block 1: r_q as 16-bit fixed point over [-0.5, 1.5) (resolution 2^-15),
//            (recoloring keeps r_q within rho0/rho +- beta/4 of the node's
//            phase share).
// f0 = r fT, f1 = fT - f0, so the two components always add up to the stored
// total.  Both are rounded stochastically when a seed is given (unbiased
// stored values, as for single-phase 16-bit storage).  Arithmetic in FP32.
template <class L, class H> struct ColorPacked {
    static constexpr bool packed = true;
    static constexpr bool blocked = false;
    static constexpr bool dither = true;
    static constexpr bool shifted = false;
    using T = uint16_t;
    using R = float;
    static constexpr int kDrop = sizeof(H) == 2 && std::is_same<H, __half>::value ? 13 : 16;
    __device__ static float to_f(uint16_t h)
    {
        if constexpr (std::is_same<H, __half>::value) return __half2float(__ushort_as_half(h));
        else return __bfloat162float(__ushort_as_bfloat16(h));
    }
    __device__ static uint16_t from_f_rn(float x)
    {
        if constexpr (std::is_same<H, __half>::value) return __half_as_ushort(__float2half_rn(x));
        else return __bfloat16_as_ushort(__float2bfloat16_rn(x));
    }
    __device__ static uint16_t from_f_sr(float x, uint32_t r)
    {
        if constexpr (std::is_same<H, __half>::value)
            return __half_as_ushort(fabsf(x) >= 6.103515625e-05f ? __float2half_rz(dither_bits(x, r, 13))
                                                                 : __float2half_rn(x));
        else return __bfloat16_as_ushort(__float2bfloat16_rz(dither_bits(x, r, 16)));
    }
    __device__ static void load_pair(const uint16_t* __restrict__ fin, uint32_t off, uint32_t nblk, int q,
                                     float rho_bar, float& f0, float& f1)
    {
        const float g = to_f(__ldg(fin + off)) * ShiftScale<L>::inv(q);
        const float fT = (float)L::w36f(q) * (1.0f / 36.0f) * rho_bar + g;
        const float r = (float)__ldg(fin + nblk + off) * (1.0f / 32768.0f) - 0.5f;
        f0 = r * fT;
        f1 = fT - f0;
    }
    // a0 = component 0, fT = the total; r1, r2 random words (unused when !sr).
    __device__ static void store_pair(uint16_t* __restrict__ fout, uint32_t off, uint32_t nblk, int q,
                                      float rho_bar, float a0, float fT, bool sr, uint32_t r1, uint32_t r2)
    {
        const float g = (fT - (float)L::w36f(q) * (1.0f / 36.0f) * rho_bar) * ShiftScale<L>::scale(q);
        fout[off] = sr ? from_f_sr(g, r1) : from_f_rn(g);
        // The share only needs 2^-15: the fast approximate division is enough.
        const float share = fabsf(fT) > 1e-30f ? __fdividef(a0, fT) : 0.5f;
        float c = (share + 0.5f) * 32768.0f + (sr ? (float)(r2 >> 8) * (1.0f / 16777216.0f) : 0.5f);
        c = fminf(fmaxf(c, 0.0f), 65535.0f);
        fout[nblk + off] = (uint16_t)c;
    }
};

template <class S> struct IsPacked { static constexpr bool value = false; };
template <class L, class H> struct IsPacked<ColorPacked<L, H>> { static constexpr bool value = true; };

struct ColorWall {
    const uint16_t* __restrict__ angle_id;  // per fluid node; 0 = not next to a solid
    const double* __restrict__ angles;      // [id][2] = cos, sin of the mean contact angle
    const double* __restrict__ tib;         // per wall-normal code: TibNorm, row-major, reference {z,y,x} order
};

constexpr double kSolidPhi = 86.0;

// Half-permeable films (HF voxels): bits[k] marks the film voxels of phase k
// in the occupancy map's word layout (nullptr when the geometry has none).
struct Film {
    const uint32_t* __restrict__ bits[2];
};

// Bit q set when the pull source x - e_q is a film voxel of the bitmap.
template <class L>
__device__ __forceinline__ uint32_t film_sources(const Grid& g, const uint32_t* __restrict__ bits, int x, int y, int z)
{
    uint32_t m = 0;
#pragma unroll
    for (int q = 1; q < L::Q; ++q) {
        const int sx = wrap(x - L::ex(q), g.nx), sy = wrap(y - L::ey(q), g.ny);
        const int sz = L::D == 3 ? wrap(z - L::ez(q), g.nz) : 0;
        const uint32_t w = __ldg(&bits[((size_t)sz * g.ny + sy) * g.W + (sx >> 5)]);
        m |= ((w >> (sx & 31)) & 1u) << q;
    }
    return m;
}

// Both components' incoming populations of node i, handed to sink(q, f0_q,
// f1_q, source) with source the compact index of the pull source x - e_q, or
// UINT32_MAX when it is solid (bounce-back).  One neighbour lookup serves both
// components (the sources are the same).
template <class L, class S, bool PULL, class Sink>
__device__ __forceinline__ void color_pull(const Grid& g, const typename S::T* __restrict__ fin, uint32_t i,
                                           int x, int y, int z, typename S::R rho_bar, Sink&& sink)
{
    using R = typename S::R;
    const typename S::T* __restrict__ fin1 = fin + (size_t)L::Q * g.nfp;
    const uint32_t nfp = g.nfp;
    const uint32_t nblk = (uint32_t)L::Q * nfp;
    auto load2 = [&](uint32_t off, int q, R& a, R& b) {
        if constexpr (IsPacked<S>::value) S::load_pair(fin, off, nblk, q, rho_bar, a, b);
        else { a = S::load(fin + off, q, R(0)); b = S::load(fin1 + off, q, R(0)); }
    };
    {
        R a, b;
        load2(i, 0, a, b);
        sink(0, a, b, i);
    }
    if constexpr (!PULL) {
#pragma unroll
        for (int q = 1; q < L::Q; ++q) {
            R a, b;
            load2(q * nfp + i, q, a, b);
            sink(q, a, b, i);
        }
    } else {
        uint32_t src[L::Q];
        const uint32_t mask = pull_sources<L, (sizeof(R) == 4)>(g, x, y, z, src);
#pragma unroll
        for (int q = 1; q < L::Q; ++q) {
            const bool fluid = (mask >> q) & 1u;
            const uint32_t node = fluid ? src[q] : i;
            const uint32_t off = (fluid ? (uint32_t)q : (uint32_t)L::op(q)) * nfp + node;
            R a, b;
            load2(off, q, a, b);
            sink(q, a, b, fluid ? src[q] : 0xffffffffu);
        }
    }
}

// Both components' incoming populations of node i.  With films (FILM, pull
// steps only): phase 0 bounces back from films of phase 1 and phase 1 from
// films of phase 0 (ColorFluid::Run, colorfluid.cpp:155-158), then a film
// voxel keeps only its own phase (clearHalfFilm, colorfluid.cpp:752-765).
// nbr keeps the occupancy neighbours: a film voxel is fluid for the gradient.
template <class L, class S, bool PULL, bool FILM>
__device__ __forceinline__ void color_gather(const Grid& g, const Film& film, const typename S::T* __restrict__ fin,
                                             uint32_t i, int x, int y, int z, typename S::R (&f0)[L::Q],
                                             typename S::R (&f1)[L::Q], uint32_t (&nbr)[L::Q],
                                             typename S::R rho_bar = typename S::R(0))
{
    using R = typename S::R;
    color_pull<L, S, PULL>(g, fin, i, x, y, z, rho_bar, [&](int q, R a, R b, uint32_t src) {
        f0[q] = a;
        f1[q] = b;
        if (q == 0) nbr[0] = i;
        else if (PULL) nbr[L::op(q)] = src;
        else nbr[q] = 0;
    });
    if constexpr (FILM && PULL && !IsPacked<S>::value) {
        const uint32_t b1 = film_sources<L>(g, film.bits[1], x, y, z);   // blocks phase 0
        const uint32_t b0 = film_sources<L>(g, film.bits[0], x, y, z);   // blocks phase 1
        const typename S::T* in1 = fin + (size_t)L::Q * g.nfp;
#pragma unroll
        for (int q = 1; q < L::Q; ++q) {
            if ((b1 >> q) & 1u) f0[q] = S::load(fin + ((size_t)L::op(q) * g.nfp + i), L::op(q), R(0));
            if ((b0 >> q) & 1u) f1[q] = S::load(in1 + ((size_t)L::op(q) * g.nfp + i), L::op(q), R(0));
        }
        const size_t w = ((size_t)z * g.ny + y) * g.W + (x >> 5);
        const uint32_t own0 = (__ldg(&film.bits[0][w]) >> (x & 31)) & 1u;
        const uint32_t own1 = (__ldg(&film.bits[1][w]) >> (x & 31)) & 1u;
#pragma unroll
        for (int q = 0; q < L::Q; ++q) {
            if (own0) f1[q] = R(0);
            if (own1) f0[q] = R(0);
        }
    }
}

// Non-contracted IEEE arithmetic (never fused into FMA).
__device__ __forceinline__ double xmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double xadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double xsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float xmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float xadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float xsub(float a, float b) { return __fsub_rn(a, b); }

// Normal code of a wall node: n = -sum e_q over solid links, components in
// the reference order (n0, n1, n2) = {z,y,x} in 3D and (n0, n1) = {y,x} in 2D,
// each in [-5, 5] (3D) or [-3, 3] (2D).
template <class L> __host__ __device__ inline int normal_code(int n0, int n1, int n2)
{
    return L::D == 3 ? ((n0 + 5) * 11 + (n1 + 5)) * 11 + (n2 + 5) : (n0 + 3) * 7 + (n1 + 3);
}
template <class L> constexpr int normal_codes() { return L::D == 3 ? 11 * 11 * 11 : 7 * 7; }

// Pass 1: phase field.  PULL = false reads the node's own values (t = 0).
template <class L, class S, bool PULL, bool FILM>
__global__ void __launch_bounds__(128)
color_phase(const Grid g, const Film film, const typename S::T* __restrict__ fin, double2* __restrict__ dens,
            double* __restrict__ phid, uint32_t* __restrict__ err, const double rho_bar)
{
    using R = typename S::R;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.nf) return;
    int x, y, z;
    unpack(__ldg(&g.coord[i]), x, y, z);
    R f0[L::Q], f1[L::Q];
    uint32_t nbr[L::Q];
    color_gather<L, S, PULL, FILM>(g, film, fin, i, x, y, z, f0, f1, nbr, R(rho_bar));
    R d0 = f0[0], d1 = f1[0];
#pragma unroll
    for (int q = 1; q < L::Q; ++q) { d0 += f0[q]; d1 += f1[q]; }
    const R dt = d0 + d1;
    if (!isfinite(d0) || !isfinite(d1) || !isfinite(dt) || !(dt > R(0))) atomicOr(err, kErrDensity);
    // The reference's roundoff allowance, -1e-10 rho (colorfluid.cpp:258), is
    // about 450 FP64 ulps; at FP32 arithmetic the same 450 ulps is 2.7e-5 rho.
    // 16-bit storage quantises each component share to 2^-15 (a density
    // noise of about 1e-5 rho), so its allowance is 1e-3 rho.
    const R tol = sizeof(R) == 8 ? R(1e-10) : (IsPacked<S>::value ? R(1e-3) : R(2.7e-5));
    if (d0 < -tol * dt || d1 < -tol * dt) atomicOr(err, kErrComponent);
    // Pass 2 takes the densities from here (exactly the sums it would form
    // from the same populations) and gathers only the total.
    dens[i] = make_double2((double)d0, (double)d1);
    phid[((size_t)z * g.ny + y) * g.nx + x] = (double)((d0 - d1) / dt);
}

// ColorFluid::colorGradient of node i (colorfluid.cpp:435-570) from the
// phase field of its neighbours (phin[q]: phi at x + e_q, kSolidPhi for a
// solid voxel): gr in the reference component order {z,y,x} / {y,x}, after
// the geometric wall rotation at wall nodes, and the norm of the unrotated
// gradient.  Non-contracted IEEE operations in the reference's order: the
// rotation angle is undefined when the in-plane gradient vanishes, so exact
// cancellations must stay exact.
template <class L, class R>
__device__ __forceinline__ void color_gradient_node(const ColorWall& W, const uint32_t i, const R phi_i,
                                                    const R (&phin)[L::Q], R (&gr)[3], R& norm)
{
    // ColorFluid::colorGradient (colorfluid.cpp:435-570), gradient in the
    // reference component order gr[0..D-1] = {z,y,x} / {y,x}; it only needs
    // the neighbours' phase field, so it is done before the collision and
    // the neighbour data is dead by then.  The gradient and the wall rotation
    // use non-contracted IEEE operations in the reference's order: the
    // rotation angle is undefined when the in-plane gradient vanishes, so
    // exact cancellations must stay exact.
    gr[0] = gr[1] = gr[2] = R(0);
    const uint16_t wid = __ldg(&W.angle_id[i]);
#pragma unroll
    for (int d = 0; d < L::D; ++d) {
#pragma unroll
        for (int k = 0; k < L::NRELD; ++k) {
            const int q = L::reld(d, k);
            const int e = comp<L>(q, L::D - 1 - d);
            // Interior: the neighbour's phi; wall node: phi difference over
            // fluid neighbours only (a solid neighbour's term is skipped).
            // Selects instead of branches: the warp's lanes mix both kinds.
            const bool skip = wid && phin[q] == R(kSolidPhi);
            const R term = wid ? xsub(phin[q], phi_i) : phin[q];
            const R c = xmul(R(w<L>(q)), term);
            const R nv = e == 1 ? xadd(gr[d], c) : xsub(gr[d], c);
            gr[d] = skip ? gr[d] : nv;
        }
    }
    R n2 = R(0);
#pragma unroll
    for (int d = 0; d < L::D; ++d) gr[d] = xmul(gr[d], R(3));
#pragma unroll
    for (int d = 0; d < L::D; ++d) n2 = xadd(n2, xmul(gr[d], gr[d]));
    norm = sqrt(n2);
    if (wid) {
        const double* cs = W.angles + 2 * wid;
        const R cA = R(cs[0]), sA = R(cs[1]);
        int nn[3] = {0, 0, 0};   // normal in reference order
#pragma unroll
        for (int q = 1; q < L::Q; ++q)
            if (phin[q] == R(kSolidPhi)) {
#pragma unroll
                for (int d = 0; d < L::D; ++d) nn[d] -= comp<L>(q, L::D - 1 - d);
            }
        const int code = normal_code<L>(nn[0], nn[1], nn[2]);
        if (L::D == 3) {
            const double* T = W.tib + 9 * code;
            R gn[3];
#pragma unroll
            for (int r = 0; r < 3; ++r) {
                R s = R(0);
#pragma unroll
                for (int k = 0; k < 3; ++k) s = xadd(s, xmul(R(T[3 * r + k]), gr[k]));
                gn[r] = s;
            }
            // RotateTx3D(-gn0, gn1) (fn.cpp:129-139).
            R c = R(1), sn = R(0);
            const R o = -gn[0];
            const R h = sqrt(xadd(xmul(o, o), xmul(gn[1], gn[1])));
            if (h != R(0)) { c = gn[1] / h; sn = o / h; }
            const R tx[9] = {c, -sn, R(0), sn, c, R(0), R(0), R(0), R(1)};
            // tInv = TibNormInv * txInv with TibNormInv = TibNorm^T.
            R ti[9];
#pragma unroll
            for (int r = 0; r < 3; ++r)
#pragma unroll
                for (int col = 0; col < 3; ++col) {
                    R s = R(0);
#pragma unroll
                    for (int k = 0; k < 3; ++k) s = xadd(s, xmul(R(T[3 * k + r]), tx[3 * k + col]));
                    ti[3 * r + col] = s;
                }
            const R t[3] = {R(0), xmul(norm, sA), xmul(norm, cA)};
#pragma unroll
            for (int r = 0; r < 3; ++r) {
                R s = R(0);
#pragma unroll
                for (int k = 0; k < 3; ++k) s = xadd(s, xmul(ti[3 * r + k], t[k]));
                gr[r] = s;
            }
        } else {
            const double* T = W.tib + 4 * code;
            const R gn0 = xadd(xadd(R(0), xmul(R(T[0]), gr[0])), xmul(R(T[1]), gr[1]));
            R t[2];
            if (gn0 >= R(0)) { t[0] = xmul(norm, sA); t[1] = xmul(norm, cA); }
            else { t[0] = xmul(-norm, sA); t[1] = xmul(norm, cA); }
            // TibNormInv = TibNorm^T.
            const R g0 = xadd(xadd(R(0), xmul(R(T[0]), t[0])), xmul(R(T[2]), t[1]));
            const R g1 = xadd(xadd(R(0), xmul(R(T[1]), t[0])), xmul(R(T[3]), t[1]));
            gr[0] = g0; gr[1] = g1;
        }
    }

}

// Pass 2 for one node from the component densities d0, d1 (sums over
// q = 0..Q-1 in order) and the total distribution fT = f0 + f1: macros,
// collision, perturbation and recoloring.  COLL: 0 = SRT, 1 = MRT.
template <class L, class S, int COLL>
__device__ __forceinline__ void color_update_total(const Grid& g, const Force& F, const ColorParams& P,
                                                   typename S::T* __restrict__ fout,
                                                   const typename S::R (&gr)[3], const typename S::R norm,
                                                   const Macros& mo, const int out,
                                                   uint32_t* __restrict__ err, const uint32_t i,
                                                   const typename S::R d0, const typename S::R d1,
                                                   typename S::R (&fT)[L::Q])
{
    using R = typename S::R;
    // ColorFluid::calcMacroVar (colorfluid.cpp:238-290) and bodyForce (:736-750).
    const R dt = d0 + d1;
    const R phi_i = (d0 - d1) / dt;
    const R tau = (R(1) + phi_i) * R(P.relax0) + (R(1) - phi_i) * R(P.relax1);
    if (!isfinite(tau) || !(tau > R(0.5))) atomicOr(err, kErrTau);
    R Fv[3];
    if (F.uniform) { Fv[0] = R(F.fx); Fv[1] = R(F.fy); Fv[2] = R(F.fz); }
    else {
        const double* lf = F.label_force + 3 * __ldg(&F.label[i]);
        Fv[0] = R(lf[0]); Fv[1] = R(lf[1]); Fv[2] = R(lf[2]);
    }
    // Velocity components accumulated in the reference's component order.
    R u[3] = {R(0), R(0), R(0)};
#pragma unroll
    for (int a = 0; a < L::D; ++a) {
        R v = R(0);
#pragma unroll
        for (int q = 1; q < L::Q; ++q) {
            const int e = comp<L>(q, a);
            if (e == 1) v += fT[q];
            else if (e == -1) v -= fT[q];
        }
        u[a] = v / dt;
    }
    if (!isfinite(u[0]) || !isfinite(u[1]) || !isfinite(u[2])) atomicOr(err, kErrVelocity);
#pragma unroll
    for (int a = 0; a < L::D; ++a) u[a] += Fv[a] * R(0.5) / dt;

    if (out & kOutMacros) {
        mo.rho0[i] = (double)d0;
        mo.rho1[i] = (double)d1;
        mo.ind[i] = (double)phi_i;
#pragma unroll
        for (int a = 0; a < 3; ++a) mo.u[(size_t)a * g.nfp + i] = (double)u[a];
    }
    if (out & kOutAdjacent) {
        mo.indadj[i] = (double)phi_i;
#pragma unroll
        for (int a = 0; a < 3; ++a) mo.uadj[(size_t)a * g.nfp + i] = (double)u[a];
    }

    // ColorFluid::collision (colorfluid.cpp:334-387): collide the total
    // fT towards feq = feq_u0 + rho w (3 e.u + 4.5 (e.u)^2 - 1.5 u^2),
    // feq_u0 = rho0 ai0 + rho1 ai1, with the same two-rate form as the
    // single-phase step: SRT is s+ = s- = 1/tau_local; MRT uses the tau0 rates
    // when tau0 == tau1 and getMRTS(tau_local) otherwise (simulator.cpp:199-216).
    // ai_k,q takes one value per direction class (rest, axis, diagonal), so
    // feq_u0 is formed once per class.
    const R usq = u[2] * u[2] + u[1] * u[1] + u[0] * u[0];
    const R uf = u[2] * Fv[2] + u[1] * Fv[1] + u[0] * Fv[0];
    constexpr int kDiag = L::D == 3 ? 7 : 5;
    const R fuc[3] = {d0 * R(P.ai[0][0]) + d1 * R(P.ai[1][0]), d0 * R(P.ai[0][1]) + d1 * R(P.ai[1][1]),
                      d0 * R(P.ai[0][kDiag]) + d1 * R(P.ai[1][kDiag])};
    R fu0[L::Q];
#pragma unroll
    for (int q = 0; q < L::Q; ++q) fu0[q] = fuc[q == 0 ? 0 : (axis_dir<L>(q) ? 1 : 2)];
    R sp, sm;
    if (COLL == 0) {
        sp = sm = R(1) / tau;
    } else if (P.uniform_tau) {
        sp = R(P.rate.sp);
        sm = R(P.rate.sm);
    } else {
        sp = R(1) / tau;
        sm = R(8) * (R(2) - sp) / (R(8) - sp);
    }
    collide_trt<L, R, true>(fT, fu0, -dt * R(1.5) * usq, dt * R(4.5), dt * R(3), u, Fv, uf, sp, sm);

    // Perturbation and cosine recoloring (colorfluid.cpp:399-428).
    const R dens0T = d0 / dt;
    typename S::T* o0 = fout;
    typename S::T* o1 = fout + (size_t)L::Q * g.nfp;
    // 16-bit storage: one linear congruential stream per node and step.
    uint32_t rng = IsPacked<S>::value && P.seed ? hash32(i * 0x9e3779b9u + P.seed) : 0u;
    auto put = [&](int q, R a0, R tot) {
        if constexpr (IsPacked<S>::value) {
            uint32_t r1 = 0, r2 = 0;
            if (P.seed) {
                rng = rng * 1664525u + 1013904223u; r1 = rng;
                rng = rng * 1664525u + 1013904223u; r2 = rng;
            }
            S::store_pair(fout, (uint32_t)q * g.nfp + i, (uint32_t)L::Q * g.nfp, q, R(P.rho_ref[0]), a0, tot,
                          P.seed != 0, r1, r2);
        } else {
            S::store(o0 + (size_t)q * g.nfp + i, a0, q, R(0));
            S::store(o1 + (size_t)q * g.nfp + i, tot - a0, q, R(0));
        }
    };
    if (norm > R(1e-9)) {
        const R betaDens01TT = R(P.beta) * dens0T * d1 / dt;
        const R AkNorm = R(P.ak) * norm / tau;
        // cos(phi_q) = (e_q . gr) / norm, the reference summing the terms
        // +-gr[d] from 0 in component order and dividing per direction, then
        // once more by sqrt 2 for a diagonal (colorfluid.cpp:399-428).  IEEE
        // negation commutes with +, - and /, so a direction's value is the
        // signed value of one of D axis quotients gr[d]/norm or, for the
        // diagonal pair (d1 < d2), of (gr[d1] + gr[d2])/norm or
        // (gr[d1] - gr[d2])/norm: the same values (up to the sign of an exact
        // zero) from 15 divisions per node instead of 31 in 3D (6 instead of
        // 13 in 2D).
        R qa[3], qs[3], qd[3], qs2[3], qd2[3];
#pragma unroll
        for (int d = 0; d < L::D; ++d) qa[d] = gr[d] / norm;
#pragma unroll
        for (int d1 = 0; d1 < L::D; ++d1)
#pragma unroll
            for (int d2 = d1 + 1; d2 < L::D; ++d2) {
                const int pr = d1 + d2 - 1;
                qs[pr] = (gr[d1] + gr[d2]) / norm;
                qd[pr] = (gr[d1] - gr[d2]) / norm;
                qs2[pr] = qs[pr] / R(1.4142135623730951);
                qd2[pr] = qd[pr] / R(1.4142135623730951);
            }
#pragma unroll
        for (int q = 0; q < L::Q; ++q) {
            int d1 = -1, d2 = -1, s1 = 0, s2 = 0;
#pragma unroll
            for (int d = 0; d < L::D; ++d) {
                const int e = comp<L>(q, L::D - 1 - d);
                if (e != 0) {
                    if (d1 < 0) { d1 = d; s1 = e; }
                    else { d2 = d; s2 = e; }
                }
            }
            R angle = R(0), cosq = R(0);   // cos(phi_q), and over sqrt 2 for a diagonal
            if (d1 >= 0 && d2 < 0) {
                angle = s1 > 0 ? qa[d1] : -qa[d1];
                cosq = angle;
            } else if (d2 >= 0) {
                const int pr = d1 + d2 - 1;
                // s1 a + s2 b: a + b, a - b, -(a - b), -(a + b).
                angle = s1 > 0 ? (s2 > 0 ? qs[pr] : qd[pr]) : (s2 > 0 ? -qd[pr] : -qs[pr]);
                cosq = s1 > 0 ? (s2 > 0 ? qs2[pr] : qd2[pr]) : (s2 > 0 ? -qd2[pr] : -qs2[pr]);
            }
            fT[q] += AkNorm * (R(w<L>(q)) * angle * angle - R(L::B(q)));
            const R a0 = dens0T * fT[q] + betaDens01TT * cosq * fu0[q];
            put(q, a0, fT[q]);
        }
    } else {
#pragma unroll
        for (int q = 0; q < L::Q; ++q) put(q, dens0T * fT[q], fT[q]);
    }
}

// Pass 2 for one node from both components' gathered populations f0, f1
// (the film and Zou-He paths): macros, collision, perturbation and
// recoloring.  COLL: 0 = SRT, 1 = MRT.
template <class L, class S, int COLL>
__device__ __forceinline__ void color_update(const Grid& g, const Force& F, const ColorParams& P,
                                             typename S::T* __restrict__ fout,
                                             const typename S::R (&gr)[3], const typename S::R norm,
                                             const Macros& mo, const int out,
                                             uint32_t* __restrict__ err, const uint32_t i,
                                             typename S::R (&f0)[L::Q], typename S::R (&f1)[L::Q])
{
    using R = typename S::R;
    R d0 = f0[0], d1 = f1[0];
#pragma unroll
    for (int q = 1; q < L::Q; ++q) { d0 += f0[q]; d1 += f1[q]; }
    R fT[L::Q];
#pragma unroll
    for (int q = 0; q < L::Q; ++q) fT[q] = f0[q] + f1[q];
    color_update_total<L, S, COLL>(g, F, P, fout, gr, norm, mo, out, err, i, d0, d1, fT);
}

// Colour gradient of node i at (x, y, z) from the dense per-voxel phase
// field (solid voxels hold kSolidPhi, SOLID_DENS_N of colorfluid.cpp:49):
// each neighbour is one address computation, no occupancy lookup.
template <class L, class R>
__device__ __forceinline__ void color_gradient_dense(const Grid& g, const ColorWall& W,
                                                     const double* __restrict__ phid, const uint32_t i, int x, int y,
                                                     int z, R (&gr)[3], R& norm)
{
    const int xs[3] = {x == 0 ? g.nx - 1 : x - 1, x, x + 1 == g.nx ? 0 : x + 1};
    const int ys[3] = {y == 0 ? g.ny - 1 : y - 1, y, y + 1 == g.ny ? 0 : y + 1};
    const int zs[3] = {z == 0 ? g.nz - 1 : z - 1, z, z + 1 == g.nz ? 0 : z + 1};
    R phin[L::Q];
#pragma unroll
    for (int q = 0; q < L::Q; ++q) {
        const size_t v = ((size_t)zs[1 + L::ez(q)] * g.ny + ys[1 + L::ey(q)]) * g.nx + xs[1 + L::ex(q)];
        phin[q] = R(__ldg(&phid[v]));
    }
    color_gradient_node<L, R>(W, i, phin[0], phin, gr, norm);
}

// Pass 2: colour gradient, collision, perturbation and recoloring of every
// fluid node.  PULL = false is the t = 0 collision.  The gradient comes
// first, from the dense phase field (its loads hit L2), while the node's
// population loads are independent of it.  Without films the component
// densities come from pass 1 and each pulled pair is summed into the total
// as it arrives, so 19 populations stay live instead of 38.  The kernel is
// latency-bound; resident 128-thread blocks per SM (CollideBlocks): four for
// FP64 (128 registers; at five it spills 80 bytes and runs 3 % slower, at
// six 9 %), six for FP32 arithmetic (80 registers, no spill; 128x128x256
// medium, FP32 storage 6,880 -> 7,250 fluid MLUPS, 16-bit 5,215 -> 5,470).
template <class S> struct CollideBlocks { static constexpr int value = 6; };
template <> struct CollideBlocks<StoreF64> { static constexpr int value = 4; };

template <class L, class S, int COLL, bool PULL, bool FILM>
__global__ void __launch_bounds__(128, CollideBlocks<S>::value)
color_collide(const Grid g, const Film film, const Force F, const ColorParams P, const ColorWall W,
              const typename S::T* __restrict__ fin, typename S::T* __restrict__ fout,
              const double2* __restrict__ dens, const double* __restrict__ phid, Macros mo, const int out,
              uint32_t* __restrict__ err)
{
    using R = typename S::R;
    // Blocks run in descending node order: pass 1 has just read the
    // populations in ascending order, so the highest nodes' lines are the
    // ones still in L2, and the next step's pass 1 starts with the lowest
    // nodes, the last ones written here.
    const uint32_t i = (gridDim.x - 1 - blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= g.nf) return;
    int x, y, z;
    unpack(__ldg(&g.coord[i]), x, y, z);
    R gr[3], norm;
    color_gradient_dense<L, R>(g, W, phid, i, x, y, z, gr, norm);
    if constexpr (FILM) {
        R f0[L::Q], f1[L::Q];
        uint32_t nbr[L::Q];
        color_gather<L, S, PULL, FILM>(g, film, fin, i, x, y, z, f0, f1, nbr, R(P.rho_ref[0]));
        color_update<L, S, COLL>(g, F, P, fout, gr, norm, mo, out, err, i, f0, f1);
    } else {
        const double2 d = dens[i];
        R fT[L::Q];
        color_pull<L, S, PULL>(g, fin, i, x, y, z, R(P.rho_ref[0]),
                               [&](int q, R a, R b, uint32_t) { fT[q] = a + b; });
        color_update_total<L, S, COLL>(g, F, P, fout, gr, norm, mo, out, err, i, R(d.x), R(d.y), fT);
    }
}

// ---- two-phase Zou-He boundaries ------------------------------------------------
// ColorFluid::zouHeBoundary (colorfluid.cpp:638-734) runs after streaming and
// bounce-back: the single-phase rule applied to the total distribution
// f0 + f1, with the rebuilt unknowns given to the label's phase and the other
// phase's unknowns cleared.  Its density and velocity are intermediates --
// calcMacroVar (whose node set includes PB/VB) recomputes both from the
// populations -- except in the adjacent-step history of a report, which the
// reference copies between the two: the velocity there is the boundary's
// prescribed one and the phase indicator is the previous step's rho0 - rho1
// over this step's boundary density (colorfluid.cpp:162-167).
// The step runs as: pass 1 -> boundary phase pass (phi of the boundary nodes
// from their rebuilt populations) -> pass 2 -> boundary collision pass (the
// boundary nodes again, overwriting what pass 2 wrote for them).
// Non-contracted operations in the reference's order.
template <class L, class R, int DIR>
__device__ __forceinline__ void color_zou_he_node(R (&f0)[L::Q], R (&f1)[L::Q], uint32_t kind, int phs,
                                                  double val, R& dens, R& ua)
{
    constexpr int A = ZouHeDir<L, DIR>::A, SG = ZouHeDir<L, DIR>::SG;
    R sum = R(0);
#pragma unroll
    for (int q = 1; q < L::Q; ++q)
        if (comp<L>(q, A) == -SG) sum = xadd(sum, xadd(xadd(xadd(f0[q], f0[q]), f1[q]), f1[q]));
#pragma unroll
    for (int q = 0; q < L::Q; ++q)
        if (comp<L>(q, A) == 0) sum = xadd(sum, xadd(f0[q], f1[q]));
    if (kind == kZouHeVB) {
        const double vel = SG > 0 ? val : -val;
        ua = R(vel);
        dens = xmul(sum, R(1.0 / (1.0 - vel)));
    } else {
        dens = R(val);
        const R s = xsub(sum / R(val), R(1));
        ua = SG > 0 ? -s : s;
    }
    R fq[L::Q];
#pragma unroll
    for (int q = 1; q < L::Q; ++q) {
        if (comp<L>(q, A) != SG) continue;
        R fT = xadd(f0[L::op(q)], f1[L::op(q)]);
        fT = xadd(fT, xmul(xmul(xmul(R(SG), R(6.0 * w<L>(q))), dens), ua));
        R t = R(0);
#pragma unroll
        for (int n = 1; n < L::Q; ++n) {
            if (comp<L>(n, A) != 0) continue;
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                if (d == A || comp<L>(n, d) == 0 || comp<L>(q, d) == 0) continue;
                if (comp<L>(n, d) == comp<L>(q, d)) t = xadd(t, xadd(f0[n], f1[n]));
                else t = xsub(t, xadd(f0[n], f1[n]));
            }
        }
        fq[q] = xsub(fT, xmul(t, R(0.5)));
    }
#pragma unroll
    for (int q = 1; q < L::Q; ++q) {
        if (comp<L>(q, A) != SG) continue;
        f0[q] = phs == 0 ? fq[q] : R(0);
        f1[q] = phs == 0 ? R(0) : fq[q];
    }
}

// Gather a boundary node and apply the rule; returns the boundary density and
// axial velocity (ua on axis *axis).
template <class L, class S, bool FILM>
__device__ __forceinline__ void color_zou_he_gather(const Grid& g, const Film& film, const ZouHe& z, const uint32_t k,
                                                    const typename S::T* __restrict__ fin, uint32_t& i,
                                                    typename S::R (&f0)[L::Q], typename S::R (&f1)[L::Q],
                                                    uint32_t (&nbr)[L::Q], typename S::R& dens,
                                                    typename S::R& ua, int& axis, typename S::R rho_bar)
{
    i = __ldg(&z.node[k]);
    const uint32_t code = __ldg(&z.code[k]);
    const double val = __ldg(&z.value[k]);
    int x, y, zc;
    unpack(__ldg(&g.coord[i]), x, y, zc);
    color_gather<L, S, true, FILM>(g, film, fin, i, x, y, zc, f0, f1, nbr, rho_bar);
    const uint32_t kind = (code >> 8) & 0xffu;
    const int phs = (int)(code >> 16);
    const int dir = (int)(code & 0xffu);
    axis = L::ex(dir) != 0 ? 0 : (L::ey(dir) != 0 ? 1 : 2);
    switch (dir) {
    case 1: color_zou_he_node<L, typename S::R, 1>(f0, f1, kind, phs, val, dens, ua); break;
    case 2: color_zou_he_node<L, typename S::R, 2>(f0, f1, kind, phs, val, dens, ua); break;
    case 3: color_zou_he_node<L, typename S::R, 3>(f0, f1, kind, phs, val, dens, ua); break;
    case 4: color_zou_he_node<L, typename S::R, 4>(f0, f1, kind, phs, val, dens, ua); break;
    default:
        if constexpr (L::D == 3) {
            if (dir == 5) color_zou_he_node<L, typename S::R, 5>(f0, f1, kind, phs, val, dens, ua);
            else color_zou_he_node<L, typename S::R, 6>(f0, f1, kind, phs, val, dens, ua);
        }
        break;
    }
}

// Boundary phase pass: phi of the boundary nodes from their rebuilt populations.
template <class L, class S, bool FILM>
__global__ void __launch_bounds__(128)
color_zou_he_phase(const Grid g, const Film film, const ZouHe z, const typename S::T* __restrict__ fin,
                   double* __restrict__ phid, uint32_t* __restrict__ err, const double rho_bar)
{
    using R = typename S::R;
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= z.n) return;
    uint32_t i;
    R f0[L::Q], f1[L::Q], dens, ua;
    uint32_t nbr[L::Q];
    int axis;
    color_zou_he_gather<L, S, FILM>(g, film, z, k, fin, i, f0, f1, nbr, dens, ua, axis, R(rho_bar));
    R d0 = f0[0], d1 = f1[0];
#pragma unroll
    for (int q = 1; q < L::Q; ++q) { d0 += f0[q]; d1 += f1[q]; }
    const R dt = d0 + d1;
    if (!isfinite(d0) || !isfinite(d1) || !isfinite(dt) || !(dt > R(0))) atomicOr(err, kErrDensity);
    const R tol = sizeof(R) == 8 ? R(1e-10) : (IsPacked<S>::value ? R(1e-3) : R(2.7e-5));
    if (d0 < -tol * dt || d1 < -tol * dt) atomicOr(err, kErrComponent);
    // Only the dense phase field: the boundary node's pass-2 result is
    // replaced by color_zou_he_collide, which sums its own densities.
    int vx, vy, vz;
    unpack(__ldg(&g.coord[i]), vx, vy, vz);
    phid[((size_t)vz * g.ny + vy) * g.nx + vx] = (double)((d0 - d1) / dt);
}

// Boundary collision pass (after pass 2); also keeps the report's adjacent
// history of the boundary nodes as the reference forms it.  z.num[k] holds
// rho0 - rho1 of the last step that asked for the adjacent history.
template <class L, class S, int COLL, bool FILM>
__global__ void __launch_bounds__(128)
color_zou_he_collide(const Grid g, const Film film, const Force F, const ColorParams P, const ColorWall W,
                     const ZouHe z,
                     const typename S::T* __restrict__ fin, typename S::T* __restrict__ fout,
                     const double* __restrict__ phid, Macros mo, const int out, uint32_t* __restrict__ err)
{
    using R = typename S::R;
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= z.n) return;
    uint32_t i;
    R f0[L::Q], f1[L::Q], dens, ua;
    uint32_t nbr[L::Q];
    int axis;
    color_zou_he_gather<L, S, FILM>(g, film, z, k, fin, i, f0, f1, nbr, dens, ua, axis, R(P.rho_ref[0]));
    R d0 = f0[0], d1 = f1[0];
#pragma unroll
    for (int q = 1; q < L::Q; ++q) { d0 += f0[q]; d1 += f1[q]; }
    R gr[3], norm;
    {
        int gx, gy, gz;
        unpack(__ldg(&g.coord[i]), gx, gy, gz);
        color_gradient_dense<L, R>(g, W, phid, i, gx, gy, gz, gr, norm);
    }
    color_update<L, S, COLL>(g, F, P, fout, gr, norm, mo, out, err, i, f0, f1);
    if (out & kOutMacros) {
        const double prev = z.num[k];
        mo.indadj[i] = (double)dens > 0.0 ? prev / (double)dens : 0.0;
#pragma unroll
        for (int a = 0; a < 3; ++a) mo.uadj[(size_t)a * g.nfp + i] = a == axis ? (double)ua : 0.0;
    }
    if (out & kOutAdjacent) z.num[k] = (double)(d0 - d1);
}

// The adjacent-history numerator at t = 0 (no boundary rule at t = 0; the
// reference's initial calcMacroVar covers PB/VB).
template <class L, class S>
__global__ void __launch_bounds__(128)
color_zou_he_record(const Grid g, const ZouHe z, const typename S::T* __restrict__ fin, const double rho_bar)
{
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= z.n) return;
    const uint32_t i = __ldg(&z.node[k]);
    double d0 = 0.0, d1 = 0.0;
    {
        using R = typename S::R;
        R a = R(0), b = R(0);
#pragma unroll
        for (int q = 0; q < L::Q; ++q) {
            R p0, p1;
            if constexpr (IsPacked<S>::value)
                S::load_pair(fin, (uint32_t)q * g.nfp + i, (uint32_t)L::Q * g.nfp, q, R(rho_bar), p0, p1);
            else {
                p0 = S::load(fin + (size_t)q * g.nfp + i, q, R(0));
                p1 = S::load(fin + ((size_t)L::Q + q) * g.nfp + i, q, R(0));
            }
            a = q == 0 ? p0 : a + p0;
            b = q == 0 ? p1 : b + p1;
        }
        d0 = (double)a;
        d1 = (double)b;
    }
    z.num[k] = d0 - d1;
}

// t = 0 populations of ColorFluid::initialize (colorfluid.cpp:214-236):
// the node's phase gets ai_k,q rho_k - 1.5 w_q (e.F), the other phase 0.
template <class L, class S>
__global__ void color_init(const Grid g, const Force F, const ColorParams P,
                           const uint8_t* __restrict__ phase, typename S::T* __restrict__ f)
{
    using R = typename S::R;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.nf) return;
    double Fv[3];
    if (F.uniform) { Fv[0] = F.fx; Fv[1] = F.fy; Fv[2] = F.fz; }
    else { const double* lf = F.label_force + 3 * F.label[i]; Fv[0] = lf[0]; Fv[1] = lf[1]; Fv[2] = lf[2]; }
    const int ph = phase[i];
#pragma unroll
    for (int q = 0; q < L::Q; ++q) {
        double ef = 0.0;
        if (L::D == 3) ef = L::ez(q) * Fv[2];
        ef += L::ey(q) * Fv[1];
        ef += L::ex(q) * Fv[0];
        double v = P.ai[ph][q] * P.rho_ref[ph];
        v -= 1.5 * (L::w36f(q) / 36.0) * ef;
        if constexpr (IsPacked<S>::value) {
            S::store_pair(f, (uint32_t)q * g.nfp + i, (uint32_t)L::Q * g.nfp, q, R(P.rho_ref[0]),
                          ph == 0 ? R(v) : R(0), R(v), false, 0u, 0u);
        } else {
            S::store(f + ((size_t)ph * L::Q + q) * g.nfp + i, R(v), q, R(0));
            S::store(f + ((size_t)(1 - ph) * L::Q + q) * g.nfp + i, R(0), q, R(0));
        }
    }
}

}  // namespace lbf
