// Host side of the C ABI (include/lbflow.h): geometry packing, link
// classification, device state and the step / reduction drivers.
#include "../../include/lbflow.h"
#include "internal.h"
#include "reduce.cuh"

#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <string>
#include <utility>
#include <vector>

using namespace lbf;

struct lbf_engine {
    lbf_config cfg;
    lbf_label labels[256];
    int D = 3, Q = 19, phases = 1;
    int nx = 0, ny = 0, nz = 0, W = 0;
    size_t N = 0;
    uint32_t nf = 0, nfp = 0;
    std::vector<uint32_t> vox;      // voxel index of each fluid node
    size_t elem = 8;                // bytes per stored population
    void* f[2] = {nullptr, nullptr};
    int8_t* ex[2] = {nullptr, nullptr};   // block exponents (block-scaled storage)
    int cur = 0;
    uint2* occ = nullptr;
    uint32_t* coord = nullptr;
    uint8_t* node_label = nullptr;
    uint8_t* node_phase = nullptr;
    double* label_force = nullptr;
    double *rho0 = nullptr, *rho1 = nullptr, *u = nullptr, *uprev = nullptr, *uadj = nullptr;
    double *ind = nullptr, *indprev = nullptr, *indadj = nullptr;
    double2* dens = nullptr;   // two-phase: component densities of the step (pass 1 -> pass 2)
    double* phid = nullptr;         // color: phase field per voxel [N], solid voxels kSolidPhi
    uint16_t* angle_id = nullptr;
    double* angles = nullptr;
    double* tib = nullptr;
    uint32_t* err = nullptr;
    double* partial = nullptr;
    double* dense_tmp = nullptr;    // FP64 copy of reduced-precision populations (dense output)
    double* stage = nullptr;        // device staging of dense outputs bound for host memory
    double* solid_f[2] = {nullptr, nullptr};   // populations of solid voxels (lbf_keep_solid_populations)
    int scur = 0;
    size_t ns = 0;                  // solid voxels (N - nf)
    double* red = nullptr;
    double* h_red = nullptr;        // pinned
    cudaStream_t stream = nullptr;
    Force force{};
    ZouHe zh{};                     // PB/VB boundary nodes (single phase)
    uint32_t *zh_node = nullptr, *zh_code = nullptr;
    double *zh_value = nullptr, *zh_num = nullptr;
    uint32_t* film_bits[2] = {nullptr, nullptr};   // half-film voxels of phase 0 / 1 (color)
    ScspParams sp{};
    ColorParams cp{};
    bool initialized = false;
    uint32_t steps = 0;             // pull steps launched (seeds the 16-bit stochastic rounding)
    uint32_t pulls = 0;             // pull steps launched (alternates the step kernel's node order)
    uint64_t bytes = 0;
    std::string last_error;
};

namespace {

thread_local std::string g_create_error;

int fail(lbf_engine* e, int code, const std::string& msg)
{
    if (e) e->last_error = msg;
    else g_create_error = msg;
    return code;
}

#define LBF_CK(e, call)                                                                  \
    do {                                                                                 \
        cudaError_t err_ = (call);                                                       \
        if (err_ != cudaSuccess)                                                         \
            return fail(e, LBF_ECUDA, std::string(#call) + ": " + cudaGetErrorString(err_)); \
    } while (0)

// Engine state comes from one stream-ordered memory pool per device that
// keeps up to kPoolKeepBytes reserved after frees, so that destroying an
// engine and creating the next one (a sequence of runs, or a run after a
// throwaway warm-up engine) reuses mapped device memory instead of mapping
// gigabytes again; larger reservations are returned to the driver when a
// stream synchronises.
constexpr uint64_t kPoolKeepBytes = 8ull << 30;
std::mutex g_pool_mu;
cudaMemPool_t g_pool[64] = {};

}  // namespace

cudaError_t lbf::device_pool(int device, cudaMemPool_t* pool)
{
    if (device < 0 || device >= 64) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_pool_mu);
    if (!g_pool[device]) {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = device;
        cudaMemPool_t p = nullptr;
        cudaError_t r = cudaMemPoolCreate(&p, &props);
        if (r != cudaSuccess) return r;
        uint64_t keep = kPoolKeepBytes;
        r = cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep);
        if (r != cudaSuccess) { cudaMemPoolDestroy(p); return r; }
        g_pool[device] = p;
    }
    *pool = g_pool[device];
    return cudaSuccess;
}

namespace {

cudaError_t engine_pool(int device, cudaMemPool_t* pool) { return lbf::device_pool(device, pool); }

template <class T>
int dalloc(lbf_engine* e, T** p, size_t count)
{
    *p = nullptr;
    if (count == 0) count = 1;
    cudaMemPool_t pool = nullptr;
    cudaError_t r = engine_pool(e->cfg.device, &pool);
    if (r == cudaSuccess)
        r = cudaMallocFromPoolAsync(reinterpret_cast<void**>(p), count * sizeof(T), pool, e->stream);
    if (r != cudaSuccess)
        return fail(e, r == cudaErrorMemoryAllocation ? LBF_ENOMEM : LBF_ECUDA,
                    std::string("cudaMalloc: ") + cudaGetErrorString(r));
    e->bytes += count * sizeof(T);
    return LBF_OK;
}

// Reference lattice tables in reference component order ({y,x} / {z,y,x}),
// used for host-side classification exactly as Simulator::buildIb does.
const int kE9[9][3] = {{0,0,0},{0,1,0},{1,0,0},{0,-1,0},{-1,0,0},{1,1,0},{1,-1,0},{-1,-1,0},{-1,1,0}};
const int kE19[19][3] = {{0,0,0},{0,0,1},{0,0,-1},{0,1,0},{0,-1,0},{1,0,0},{-1,0,0},
    {0,1,1},{0,1,-1},{0,-1,1},{0,-1,-1},{1,0,1},{1,0,-1},{-1,0,1},{-1,0,-1},
    {1,1,0},{1,-1,0},{-1,1,0},{-1,-1,0}};

// Voxels that carry populations: the fluid sets of SCSP::initialize /
// collision and Simulator::buildIb (scsp.cpp:116-134, 374-464;
// simulator.cpp:399-415; ColorFluid's initialize / calcMacroVar / collision
// sets, colorfluid.cpp:220, 244, 323).
bool is_fluid(int t) { return t == LBF_VD || t == LBF_GV || t == LBF_PB || t == LBF_VB || t == LBF_HF; }
bool is_solid(int t) { return t == LBF_BB || t == LBF_SD; }

// e_q component a (0 = x, 1 = y, 2 = z) of the reference tables.
int ecomp(int D, int q, int a)
{
    if (D == 2) return a == 0 ? kE9[q][1] : (a == 1 ? kE9[q][0] : 0);
    return kE19[q][2 - a];
}

// Two-rate form of the collision: SRT -> s+ = s- = 1/tau; MRT (legacy
// spectrum, simulator.cpp:199-216) -> s+ = 1/tau, s- = 8 (2 - s+) / (8 - s+).
Trt rates(bool mrt, double tau)
{
    Trt r;
    r.sp = 1.0 / tau;
    r.sm = mrt ? 8.0 * (2.0 - r.sp) / (8.0 - r.sp) : r.sp;
    return r;
}

// RotateTx3D / RotateTz3D / RotateT2D (fn.cpp:118-166) and
// ColorFluid::calcTibNorm (colorfluid.cpp:1111-1129), reference arithmetic.
void rot_cs(double o, double a, double* c, double* s)
{
    const double h = std::sqrt(o * o + a * a);
    *c = 1; *s = 0;
    if (h != 0) { *c = a / h; *s = o / h; }
}
void tib3(const double n[3], double* T)
{
    double c, s, tx[9], tz[9];
    rot_cs(n[0], n[1], &c, &s);
    const double txv[9] = {c, -s, 0, s, c, 0, 0, 0, 1};
    std::memcpy(tx, txv, sizeof tx);
    const double val = std::sqrt(n[0] * n[0] + n[1] * n[1]);
    rot_cs(val, n[2], &c, &s);
    const double tzv[9] = {1, 0, 0, 0, c, -s, 0, s, c};
    std::memcpy(tz, tzv, sizeof tz);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            double acc = 0.0;
            for (int k = 0; k < 3; ++k) acc += tz[3 * i + k] * tx[3 * k + j];
            T[3 * i + j] = acc;
        }
}
void tib2(const double n[2], double* T)
{
    double c, s;
    rot_cs(n[0], n[1], &c, &s);
    T[0] = c; T[1] = -s; T[2] = s; T[3] = c;
}

int setdev(lbf_engine* e)
{
    LBF_CK(e, cudaSetDevice(e->cfg.device));
    return LBF_OK;
}

Grid grid_of(const lbf_engine* e)
{
    Grid g;
    g.nx = e->nx; g.ny = e->ny; g.nz = e->nz; g.W = e->W;
    g.nf = e->nf; g.nfp = e->nfp;
    g.occ = e->occ; g.coord = e->coord;
    return g;
}

Macros macros_of(const lbf_engine* e)
{
    Macros m;
    m.rho0 = e->rho0; m.rho1 = e->rho1; m.u = e->u; m.uadj = e->uadj;
    m.ind = e->ind; m.indadj = e->indadj;
    return m;
}

unsigned dense_blocks(size_t N);
template <class L>
__global__ void solid_stream(const lbf::Grid g, int phases, const double* __restrict__ fin,
                             const double* __restrict__ sin, double* __restrict__ sout, size_t ns, size_t N);

void launch_step(lbf_engine* e, bool pull, int out)
{
    const void* fin = e->f[e->cur];
    void* fout = e->f[e->cur ^ 1];
    if (pull && e->solid_f[0]) {
        const Grid g = grid_of(e);
        if (e->D == 3)
            solid_stream<D3Q19><<<dense_blocks(e->N), 256, 0, e->stream>>>(
                g, e->phases, static_cast<const double*>(fin), e->solid_f[e->scur], e->solid_f[e->scur ^ 1], e->ns, e->N);
        else
            solid_stream<D2Q9><<<dense_blocks(e->N), 256, 0, e->stream>>>(
                g, e->phases, static_cast<const double*>(fin), e->solid_f[e->scur], e->solid_f[e->scur ^ 1], e->ns, e->N);
        e->scur ^= 1;
    }
    if (e->cfg.model == LBF_MODEL_SCSP) {
        // FP16 / BF16 storage rounds stochastically, with a fresh seed every
        // step (deterministic for a given run); the t = 0 collision rounds to
        // nearest.
        const bool dither = e->cfg.storage == LBF_STORE_FP16 || e->cfg.storage == LBF_STORE_BF16;
        e->sp.seed = dither && pull ? (++e->steps * 2654435761u) | 1u : 0u;
        e->sp.reverse = pull ? (int)(++e->pulls & 1u) : 0;
        ScspLaunch a{grid_of(e), e->force, e->sp, fin, fout, macros_of(e), e->err, e->stream,
                     e->ex[e->cur], e->ex[e->cur ^ 1], out};
        launch_scsp(e->D, (int)e->cfg.storage, e->cfg.collision == LBF_MRT, pull, out, a);
        // At t = 0 (no pull) the boundary nodes hold rho0 at rest, which the
        // main kernel reproduces from their initial populations.
        if (pull && e->zh.n) launch_scsp_zou_he(e->D, (int)e->cfg.storage, a, e->zh);
    } else {
        // 16-bit storage rounds stochastically with a fresh seed every pull
        // step, as the single-phase path does.
        const bool dither = e->cfg.storage == LBF_STORE_FP16 || e->cfg.storage == LBF_STORE_BF16;
        e->cp.seed = dither && pull ? (++e->steps * 2654435761u) | 1u : 0u;
        ColorWall W{e->angle_id, e->angles, e->tib};
        ColorLaunch a{grid_of(e), e->force, e->cp, W, fin, fout, e->dens, e->phid, macros_of(e), e->err,
                      e->stream, e->zh, Film{{e->film_bits[0], e->film_bits[1]}}};
        launch_color(e->D, (int)e->cfg.storage, (int)e->cfg.collision, pull, out, a);
    }
    e->cur ^= 1;
}

template <class Fn>
int run_reduce(lbf_engine* e, const Fn& fn, double* out)
{
    reduce_pass1<Fn><<<kReduceBlocks, kReduceThreads, 0, e->stream>>>(fn, e->nf, e->partial);
    reduce_pass2<Fn><<<1, kReduceThreads, 0, e->stream>>>(e->partial, kReduceBlocks, e->red);
    LBF_CK(e, cudaGetLastError());
    LBF_CK(e, cudaMemcpyAsync(e->h_red, e->red, Fn::K * sizeof(double), cudaMemcpyDeviceToHost, e->stream));
    LBF_CK(e, cudaStreamSynchronize(e->stream));
    std::memcpy(out, e->h_red, Fn::K * sizeof(double));
    return LBF_OK;
}

// Stored populations <-> dense-per-node FP64 ([phase][q][nfp]).
template <class L, class S>
__global__ void expand_kernel(const typename S::T* __restrict__ in, double* __restrict__ out,
                              uint32_t nf, uint32_t nfp, int phases, double rho0)
{
    using R = typename S::R;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nf) return;
    for (int p = 0; p < phases; ++p)
#pragma unroll
        for (int q = 0; q < L::Q; ++q) {
            const size_t j = ((size_t)p * L::Q + q) * nfp + i;
            const R v = S::load(in + j, q, R(rho0));
            out[j] = S::shifted ? (L::w36f(q) / 36.0) * rho0 + (double)v : (double)v;
        }
}

template <class L, class S>
__global__ void compress_kernel(const double* __restrict__ in, typename S::T* __restrict__ out,
                                uint32_t nf, uint32_t nfp, int phases, double rho0)
{
    using R = typename S::R;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nf) return;
    for (int p = 0; p < phases; ++p)
#pragma unroll
        for (int q = 0; q < L::Q; ++q) {
            const size_t j = ((size_t)p * L::Q + q) * nfp + i;
            const double v = in[j];
            S::store(out + j, S::shifted ? R(v - (L::w36f(q) / 36.0) * rho0) : R(v), q, R(rho0));
        }
}

// Block-scaled storage <-> FP64 (exact decode; encode as StoreBFP16::store_blk
// but from FP64 deviations).
template <class L>
__global__ void expand_blk_kernel(const int16_t* __restrict__ in, const int8_t* __restrict__ ex,
                                  double* __restrict__ out, uint32_t nf, uint32_t nfp, double rho0)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nf) return;
    const int e = ex[i];
#pragma unroll
    for (int q = 0; q < L::Q; ++q) {
        const double w = L::w36f(q) / 36.0;
        out[(size_t)q * nfp + i] = w * rho0 + w * ldexp((double)in[(size_t)q * nfp + i], e - 15);
    }
}

template <class L>
__global__ void compress_blk_kernel(const double* __restrict__ in, int16_t* __restrict__ out,
                                    int8_t* __restrict__ ex, uint32_t nf, uint32_t nfp, double rho0)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nf) return;
    double x[L::Q];
    double m = 0.0;
#pragma unroll
    for (int q = 0; q < L::Q; ++q) {
        const double w = L::w36f(q) / 36.0;
        x[q] = (in[(size_t)q * nfp + i] - w * rho0) / w;
        m = fmax(m, fabs(x[q]));
    }
    const int e = StoreBFP16<L>::exponent((float)m * 1.0000001f);
#pragma unroll
    for (int q = 0; q < L::Q; ++q) {
        double v = rint(ldexp(x[q], 15 - e));
        v = v > 32767.0 ? 32767.0 : (v < -32767.0 ? -32767.0 : v);
        out[(size_t)q * nfp + i] = (int16_t)v;
    }
    ex[i] = (int8_t)e;
}

// Two-phase 16-bit storage (total + component-0 share) <-> FP64 components.
template <class L, class S>
__global__ void expand_packed_kernel(const uint16_t* __restrict__ in, double* __restrict__ out, uint32_t nf,
                                     uint32_t nfp, float rho_bar)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nf) return;
#pragma unroll
    for (int q = 0; q < L::Q; ++q) {
        float f0, f1;
        S::load_pair(in, (uint32_t)q * nfp + i, (uint32_t)L::Q * nfp, q, rho_bar, f0, f1);
        out[(size_t)q * nfp + i] = (double)f0;
        out[((size_t)L::Q + q) * nfp + i] = (double)f1;
    }
}

template <class L, class S>
__global__ void compress_packed_kernel(const double* __restrict__ in, uint16_t* __restrict__ out, uint32_t nf,
                                       uint32_t nfp, float rho_bar)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nf) return;
#pragma unroll
    for (int q = 0; q < L::Q; ++q) {
        const double a = in[(size_t)q * nfp + i], b = in[((size_t)L::Q + q) * nfp + i];
        S::store_pair(out, (uint32_t)q * nfp + i, (uint32_t)L::Q * nfp, q, rho_bar, (float)a, (float)(a + b), false,
                      0u, 0u);
    }
}

template <class L>
void convert(const lbf_engine* e, bool expand, void* f, double* tmp)
{
    if (e->cfg.storage == LBF_STORE_BFP16) {
        const unsigned t = 256, b = blocks_for(e->nf, t);
        if (!b) return;
        if (expand)
            expand_blk_kernel<L><<<b, t, 0, e->stream>>>((const int16_t*)f, e->ex[e->cur], tmp, e->nf, e->nfp, e->cfg.rho[0]);
        else
            compress_blk_kernel<L><<<b, t, 0, e->stream>>>(tmp, (int16_t*)f, e->ex[e->cur], e->nf, e->nfp, e->cfg.rho[0]);
        return;
    }
    const unsigned t = 256, b = blocks_for(e->nf, t);
    if (!b) return;
    const double r0 = e->cfg.rho[0];
#define LBF_CONV(S, T)                                                                         \
    do {                                                                                       \
        if (expand) expand_kernel<L, S><<<b, t, 0, e->stream>>>((const T*)f, tmp, e->nf, e->nfp, e->phases, r0); \
        else compress_kernel<L, S><<<b, t, 0, e->stream>>>(tmp, (T*)f, e->nf, e->nfp, e->phases, r0); \
    } while (0)
    if (e->cfg.model == LBF_MODEL_COLOR && (e->cfg.storage == LBF_STORE_FP16 || e->cfg.storage == LBF_STORE_BF16)) {
        const float rb = (float)e->cp.rho_ref[0];
#define LBF_PACKED(H)                                                                          \
        do {                                                                                   \
            using S = ColorPacked<L, H>;                                                       \
            if (expand) expand_packed_kernel<L, S><<<b, t, 0, e->stream>>>((const uint16_t*)f, tmp, e->nf, e->nfp, rb); \
            else compress_packed_kernel<L, S><<<b, t, 0, e->stream>>>(tmp, (uint16_t*)f, e->nf, e->nfp, rb); \
        } while (0)
        if (e->cfg.storage == LBF_STORE_FP16) LBF_PACKED(__half);
        else LBF_PACKED(__nv_bfloat16);
#undef LBF_PACKED
    }
    else if (e->cfg.model == LBF_MODEL_COLOR) LBF_CONV(StoreF32Full, float);
    else if (e->cfg.storage == LBF_STORE_FP16) LBF_CONV(StoreF16<L>, __half);
    else if (e->cfg.storage == LBF_STORE_BF16) LBF_CONV(StoreBF16<L>, __nv_bfloat16);
    else LBF_CONV(StoreF32<L>, float);
#undef LBF_CONV
}

// Link mask of a voxel from the occupancy map (what the kernels see).
template <class L>
__global__ void link_mask_kernel(const Grid g, uint32_t* __restrict__ out, size_t N)
{
    const size_t v = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= N) return;
    const int x = (int)(v % g.nx);
    const int y = (int)((v / g.nx) % g.ny);
    const int z = (int)(v / ((size_t)g.nx * g.ny));
    bool fluid;
    lookup(g, x, y, z, fluid);
    uint32_t m = 0;
    if (fluid) {
#pragma unroll
        for (int q = 1; q < L::Q; ++q) {
            bool nf;
            lookup(g, wrap(x + L::ex(q), g.nx), wrap(y + L::ey(q), g.ny),
                   L::D == 3 ? wrap(z + L::ez(q), g.nz) : 0, nf);
            if (!nf) m |= 1u << (q - 1);
        }
    }
    out[v] = m;
}

int expand_to_host(lbf_engine* e, std::vector<double>& compact)
{
    const size_t count = (size_t)e->phases * e->Q * e->nfp;
    compact.assign(count, 0.0);
    if (e->cfg.storage == LBF_STORE_FP64) {
        LBF_CK(e, cudaMemcpyAsync(compact.data(), e->f[e->cur], count * sizeof(double),
                                  cudaMemcpyDeviceToHost, e->stream));
        LBF_CK(e, cudaStreamSynchronize(e->stream));
        return LBF_OK;
    }
    double* tmp = nullptr;
    LBF_CK(e, cudaMalloc(&tmp, count * sizeof(double)));
    if (e->D == 3) convert<D3Q19>(e, true, e->f[e->cur], tmp);
    else convert<D2Q9>(e, true, e->f[e->cur], tmp);
    cudaError_t r = cudaGetLastError();
    if (r == cudaSuccess) r = cudaMemcpyAsync(compact.data(), tmp, count * sizeof(double), cudaMemcpyDeviceToHost, e->stream);
    if (r == cudaSuccess) r = cudaStreamSynchronize(e->stream);
    cudaFree(tmp);
    if (r != cudaSuccess) return fail(e, LBF_ECUDA, std::string("expand populations: ") + cudaGetErrorString(r));
    return LBF_OK;
}

}  // namespace

namespace lbf {
void set_global_error(const std::string& msg) { g_create_error = msg; }
}  // namespace lbf

namespace {
// Populations of solid voxels (checkpoint compatibility).  The reference
// streams every voxel, fluid or solid (Simulator::streaming,
// simulator.cpp:73-101), collides only fluid ones, and bounce-back overwrites
// every population a fluid voxel receives from a solid one
// (simulator.cpp:103-111), so solid voxels carry values that never reach the
// fluid but do appear in its checkpoints (scsp.cpp:277-302).  They are kept in
// their own array [phase][q][solid index]; the solid index of voxel v is v
// minus the number of fluid voxels before it.  One pull step: a solid voxel's
// q population comes from x - e_q, the post-collision value of the previous
// step (fin for a fluid source, the old solid array for a solid one); the
// rest population is never streamed and stays as initialised (0).
template <class L>
__global__ void solid_stream(const lbf::Grid g, int phases, const double* __restrict__ fin,
                             const double* __restrict__ sin, double* __restrict__ sout, size_t ns, size_t N)
{
    for (size_t v = (size_t)blockIdx.x * blockDim.x + threadIdx.x; v < N; v += (size_t)gridDim.x * blockDim.x) {
        const int x = (int)(v % g.nx);
        const int y = (int)((v / g.nx) % g.ny);
        const int z = (int)(v / ((size_t)g.nx * g.ny));
        bool fluid;
        const uint32_t before = lbf::lookup(g, x, y, z, fluid);
        if (fluid) continue;
        const size_t si = v - before;
        for (int p = 0; p < phases; ++p) {
            const size_t b0 = (size_t)p * L::Q;
            sout[b0 * ns + si] = sin[b0 * ns + si];
#pragma unroll
            for (int q = 1; q < L::Q; ++q) {
                const int sx = lbf::wrap(x - L::ex(q), g.nx), sy = lbf::wrap(y - L::ey(q), g.ny);
                const int sz = L::D == 3 ? lbf::wrap(z - L::ez(q), g.nz) : 0;
                bool sf;
                const uint32_t j = lbf::lookup(g, sx, sy, sz, sf);
                const size_t sv = ((size_t)sz * g.ny + sy) * g.nx + sx;
                sout[(b0 + q) * ns + si] = sf ? fin[(b0 + q) * g.nfp + j] : sin[(b0 + q) * ns + (sv - j)];
            }
        }
    }
}

// Solid entries of a dense [block][voxel] array into the solid array.
__global__ void solid_from_dense(const lbf::Grid g, int blocks, const double* __restrict__ dense,
                                 double* __restrict__ s, size_t ns, size_t N)
{
    for (size_t v = (size_t)blockIdx.x * blockDim.x + threadIdx.x; v < N; v += (size_t)gridDim.x * blockDim.x) {
        const int x = (int)(v % g.nx);
        const int y = (int)((v / g.nx) % g.ny);
        const int z = (int)(v / ((size_t)g.nx * g.ny));
        bool fluid;
        const uint32_t before = lbf::lookup(g, x, y, z, fluid);
        if (fluid) continue;
        for (int b = 0; b < blocks; ++b) s[(size_t)b * ns + (v - before)] = dense[(size_t)b * N + v];
    }
}

// Dense outputs of voxels [v0, v0 + r), one thread per voxel (grid-stride),
// x fastest, so that a warp writes consecutive addresses of every array.
// Fields: out = [rho0 r][rho1 r (color)][velocity r x D interleaved];
// populations: out = [block][r].  With v0 = 0 and r = N these are the file
// layouts themselves.
__global__ void fields_range_kernel(const lbf::Grid g, const double* __restrict__ rho0,
                                    const double* __restrict__ rho1, const double* __restrict__ u, int D,
                                    size_t v0, size_t r, double* __restrict__ out)
{
    for (size_t j = (size_t)blockIdx.x * blockDim.x + threadIdx.x; j < r; j += (size_t)gridDim.x * blockDim.x) {
        const size_t v = v0 + j;
        const int x = (int)(v % g.nx);
        const int y = (int)((v / g.nx) % g.ny);
        const int z = (int)(v / ((size_t)g.nx * g.ny));
        bool fluid;
        const uint32_t k = lbf::lookup(g, x, y, z, fluid);
        out[j] = fluid ? rho0[k] : 0.0;
        size_t o = r;
        if (rho1) {
            out[r + j] = fluid ? rho1[k] : 0.0;
            o += r;
        }
        for (int c = 0; c < D; ++c) out[o + j * D + c] = fluid ? u[(size_t)c * g.nfp + k] : 0.0;
    }
}

__global__ void populations_range_kernel(const lbf::Grid g, const double* __restrict__ in, int blocks, size_t v0,
                                         size_t r, double* __restrict__ out, uint32_t* __restrict__ err,
                                         const double* __restrict__ solid, size_t ns)
{
    bool bad = false;
    for (size_t j = (size_t)blockIdx.x * blockDim.x + threadIdx.x; j < r; j += (size_t)gridDim.x * blockDim.x) {
        const size_t v = v0 + j;
        const int x = (int)(v % g.nx);
        const int y = (int)((v / g.nx) % g.ny);
        const int z = (int)(v / ((size_t)g.nx * g.ny));
        bool fluid;
        const uint32_t k = lbf::lookup(g, x, y, z, fluid);
        for (int b = 0; b < blocks; ++b) {
            const double val = fluid ? in[(size_t)b * g.nfp + k] : (solid ? solid[(size_t)b * ns + (v - k)] : 0.0);
            bad |= !isfinite(val);
            out[(size_t)b * r + j] = val;
        }
    }
    if (bad) atomicOr(err, lbf::kErrOutput);
}

// Where a dense output goes: device memory of the engine's device or managed
// memory (written in place by the kernel), or page-locked host memory (written
// through a device staging buffer and copied by DMA: direct kernel stores to
// host memory cross PCIe as small transactions and run several times slower).
enum class Dest { kNone, kDevice, kHost };
Dest destination(lbf_engine* e, double* p)
{
    cudaPointerAttributes pa{};
    if (cudaPointerGetAttributes(&pa, p) != cudaSuccess) {
        cudaGetLastError();
        return Dest::kNone;
    }
    if (pa.type == cudaMemoryTypeDevice) return pa.device == e->cfg.device ? Dest::kDevice : Dest::kNone;
    if (pa.type == cudaMemoryTypeManaged) return Dest::kDevice;
    if (pa.type == cudaMemoryTypeHost) return Dest::kHost;
    return Dest::kNone;
}

// Device staging buffer for host destinations (allocated on first use, kept).
constexpr size_t kStageBytes = (size_t)256 << 20;
int stage_buffer(lbf_engine* e, double** out)
{
    if (!e->stage) {
        const int rc = dalloc(e, &e->stage, kStageBytes / sizeof(double));
        if (rc) return rc;
    }
    *out = e->stage;
    return LBF_OK;
}

__global__ void fill_value(double* __restrict__ p, size_t n, double v)
{
    for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) p[k] = v;
}

unsigned dense_blocks(size_t N)
{
    const size_t b = (N + 255) / 256;
    return (unsigned)(b < (size_t)148 * 16 ? b : (size_t)148 * 16);
}
}  // namespace

namespace {
// ---- geometry classification on the device ---------------------------------
// One warp per 32-voxel occupancy word of an x-row (words in z, y, x-word
// order): lane b reads voxel x = 32 w + b, the warp's ballot of "carries
// populations" is the word's fluid bits.  Also records which labels occur
// (an 8-word bitmap) and each word's fluid count for the prefix scan.
__global__ void classify_words(const uint8_t* __restrict__ geom, const uint8_t* __restrict__ fluid_label, int nx,
                               int W, size_t words, uint2* __restrict__ occ, unsigned long long* __restrict__ counts,
                               uint32_t* __restrict__ used)
{
    __shared__ uint32_t s_used[8];
    if (threadIdx.x < 8) s_used[threadIdx.x] = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const size_t warps = ((size_t)gridDim.x * blockDim.x) >> 5;
    for (size_t wd = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; wd < words; wd += warps) {
        const size_t r = wd / (size_t)W;
        const int x = (int)(wd - r * W) * 32 + lane;
        bool fl = false;
        uint32_t word = 8, bit = 0;
        if (x < nx) {
            const uint8_t l = geom[r * (size_t)nx + x];
            fl = fluid_label[l] != 0;
            word = l >> 5;
            bit = 1u << (l & 31);
        }
        const uint32_t bits = __ballot_sync(0xffffffffu, fl);
#pragma unroll
        for (uint32_t k = 0; k < 8; ++k) {
            const uint32_t m = __reduce_or_sync(0xffffffffu, word == k ? bit : 0u);
            if (lane == 0 && m) atomicOr(&s_used[k], m);
        }
        if (lane == 0) {
            occ[wd].x = bits;
            counts[wd] = (unsigned long long)__popc(bits);
        }
    }
    __syncthreads();
    if (threadIdx.x < 8 && s_used[threadIdx.x]) atomicOr(&used[threadIdx.x], s_used[threadIdx.x]);
}

// Prefix counts into the words; total[0] = number of fluid voxels.
__global__ void finish_words(const unsigned long long* __restrict__ counts,
                             const unsigned long long* __restrict__ prefix, size_t words, uint2* __restrict__ occ,
                             unsigned long long* __restrict__ total)
{
    for (size_t w = (size_t)blockIdx.x * blockDim.x + threadIdx.x; w < words; w += (size_t)gridDim.x * blockDim.x) {
        occ[w].y = (uint32_t)prefix[w];
        if (w + 1 == words) total[0] = prefix[w] + counts[w];
    }
}

// Node records in voxel order: packed coordinates, and where needed the
// node's label (per-label forces) and phase (two-phase initialisation).
__global__ void fill_nodes(const uint8_t* __restrict__ geom, const uint2* __restrict__ occ, int nx, int ny, int W,
                           size_t words, const uint8_t* __restrict__ phase_of, uint32_t* __restrict__ coord,
                           uint8_t* __restrict__ nlabel, uint8_t* __restrict__ nphase)
{
    const int lane = threadIdx.x & 31;
    const size_t warps = ((size_t)gridDim.x * blockDim.x) >> 5;
    for (size_t wd = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; wd < words; wd += warps) {
        const uint2 e = occ[wd];
        if (!((e.x >> lane) & 1u)) continue;
        const size_t r = wd / (size_t)W;
        const uint32_t x = (uint32_t)(wd - r * W) * 32 + lane;
        const uint32_t y = (uint32_t)(r % (size_t)ny), z = (uint32_t)(r / (size_t)ny);
        const uint32_t k = e.y + __popc(e.x & ((1u << lane) - 1u));
        coord[k] = x | (y << 11) | (z << 22);
        const uint8_t l = geom[r * (size_t)nx + x];
        if (nlabel) nlabel[k] = l;
        if (nphase) nphase[k] = phase_of[l];
    }
}

// Voxel index of every node from the device coordinates (host copy, built on
// the first call that needs it: dense host transfers and set-up lists).
int ensure_vox(lbf_engine* e)
{
    if (e->vox.size() == e->nf) return LBF_OK;
    std::vector<uint32_t> c(e->nf);
    if (e->nf) {
        LBF_CK(e, cudaMemcpyAsync(c.data(), e->coord, (size_t)e->nf * sizeof(uint32_t), cudaMemcpyDeviceToHost,
                                  e->stream));
        LBF_CK(e, cudaStreamSynchronize(e->stream));
    }
    e->vox.resize(e->nf);
    for (uint32_t k = 0; k < e->nf; ++k) {
        const uint32_t x = c[k] & 2047u, y = (c[k] >> 11) & 2047u, z = c[k] >> 22;
        e->vox[k] = (uint32_t)(((size_t)z * e->ny + y) * e->nx + x);
    }
    return LBF_OK;
}

// Label checks (ValidateSimulation subset, fileprm.cpp:274-294) over the
// labels that occur, and the fluid/solid type sets of buildIb
// (simulator.cpp:399-415).
int validate_labels(const lbf_config& c, const lbf_label* labels, const bool (&used)[256], int Q, int D,
                    int phases, std::string& msg)
{
    for (int l = 0; l < 256; ++l) {
        if (!used[l]) continue;
        const lbf_label& L = labels[l];
        msg.clear();
        if (L.type == 0) msg = "geometry label " + std::to_string(l) + " is not defined";
        else if (!is_fluid(L.type) && !is_solid(L.type))
            msg = "label " + std::to_string(l) + ": only VD, GV, PB, VB, HF, BB and SD labels are supported";
        else if (L.type == LBF_HF && c.model != LBF_MODEL_COLOR)
            msg = "label " + std::to_string(l) + ": half-permeable films (HF) need the color model";
        else if ((L.type == LBF_PB || L.type == LBF_VB) && !std::isfinite(L.value)) msg = "Non-finite boundary value.";
        else if ((L.type == LBF_PB || L.type == LBF_VB) && (L.dir <= 0 || L.dir >= Q))
            msg = "Boundary direction must be a non-rest lattice direction.";
        else if (L.type == LBF_PB && L.value <= 0.0) msg = "Pressure-boundary density must be positive.";
        else if ((L.type == LBF_PB || L.type == LBF_VB) && L.dir > 2 * D)
            msg = "Pressure and velocity boundaries require an axial direction.";
        else if (is_fluid(L.type) && (L.phase < 0 || L.phase >= phases))
            msg = "Boundary phase is outside the configured fluid model.";
        else if (L.type == LBF_GV && (L.dir <= 0 || L.dir >= Q || !std::isfinite(L.value)))
            msg = "Invalid body-force direction or magnitude.";
        if (!msg.empty()) return LBF_EINVAL;
    }
    return LBF_OK;
}
}  // namespace

extern "C" {

int lbf_create(const lbf_config* cfg, const lbf_label labels[256], const uint8_t* geometry, lbf_engine** out)
{
    if (!out) return fail(nullptr, LBF_EINVAL, "lbf_create: out is NULL");
    *out = nullptr;
    if (!cfg || !labels || !geometry) return fail(nullptr, LBF_EINVAL, "lbf_create: NULL argument");
    const lbf_config& c = *cfg;
    if (!((c.dims == 2 && c.nz == 1) || c.dims == 3))
        return fail(nullptr, LBF_EINVAL, "dims must be 2 (with nz = 1) or 3");
    if (c.nx == 0 || c.ny == 0 || c.nz == 0 || c.nx > 2048 || c.ny > 2048 || c.nz > 1024)
        return fail(nullptr, LBF_EINVAL, "grid dimensions must be 1..2048 (x, y) and 1..1024 (z)");
    if (c.model != LBF_MODEL_SCSP && c.model != LBF_MODEL_COLOR)
        return fail(nullptr, LBF_EINVAL, "unknown fluid model");
    if (c.collision != LBF_SRT && c.collision != LBF_MRT)
        return fail(nullptr, LBF_EINVAL, "unknown collision model");
    if (c.storage > LBF_STORE_BFP16) return fail(nullptr, LBF_EINVAL, "unknown storage");
    if (c.model == LBF_MODEL_COLOR && c.storage == LBF_STORE_BFP16)
        return fail(nullptr, LBF_EINVAL, "two-phase storage must be FP64, FP32, FP16 or BF16");
    const int phases = c.model == LBF_MODEL_COLOR ? 2 : 1;
    for (int k = 0; k < phases; ++k)
        if (!std::isfinite(c.tau[k]) || c.tau[k] <= 0.5 || !std::isfinite(c.rho[k]) || c.rho[k] <= 0.0)
            return fail(nullptr, LBF_EINVAL, "Densities must be positive; relaxation times must exceed 0.5.");

    lbf_engine* e = new (std::nothrow) lbf_engine();
    if (!e) return fail(nullptr, LBF_ENOMEM, "host allocation failed");
    e->cfg = c;
    std::memcpy(e->labels, labels, sizeof e->labels);
    e->D = (int)c.dims;
    e->Q = c.dims == 2 ? 9 : 19;
    e->phases = phases;
    e->nx = (int)c.nx; e->ny = (int)c.ny; e->nz = (int)c.nz;
    e->W = (e->nx + 31) / 32;
    e->N = (size_t)c.nx * c.ny * c.nz;
    e->elem = c.storage == LBF_STORE_FP64 ? 8 : (c.storage == LBF_STORE_FP32 ? 4 : 2);
    const bool blocked = c.storage == LBF_STORE_BFP16;
    auto bail = [&](int code, const std::string& m) { lbf_destroy(e); return fail(nullptr, code, m); };

    // Which labels occur, the occupancy words and the fluid count come from
    // the device (classify_words); without a usable device the labels are
    // still checked on the host so that a bad geometry is reported as such.
    bool used[256] = {};
    const size_t rows = (size_t)e->nz * e->ny;
    const size_t words = rows * (size_t)e->W;
    int rc = setdev(e);
    if (rc) {
        for (size_t v = 0; v < e->N; ++v) used[geometry[v]] = true;
        std::string m;
        if (validate_labels(c, labels, used, e->Q, e->D, phases, m) != LBF_OK) return bail(LBF_EINVAL, m);
        m = e->last_error;
        lbf_destroy(e);
        return fail(nullptr, rc, m);
    }
#define LBF_ALLOC(p, n)                                                  \
    do {                                                                 \
        int r_ = dalloc(e, &(p), (n));                                   \
        if (r_) { std::string m_ = e->last_error; lbf_destroy(e); return fail(nullptr, r_, m_); } \
    } while (0)
#define LBF_CUDA(call)                                                   \
    do {                                                                 \
        cudaError_t r_ = (call);                                         \
        if (r_ != cudaSuccess) { lbf_destroy(e); return fail(nullptr, LBF_ECUDA, std::string(#call) + ": " + cudaGetErrorString(r_)); } \
    } while (0)
    LBF_CUDA(cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking));
    LBF_CUDA(cudaMallocHost(&e->h_red, kReduceMaxK * sizeof(double)));
    // Set-up scratch, freed before returning: the geometry, per-label tables
    // (fluid flag, phase), word counts and their prefix, the label bitmap and
    // the fluid total.
    uint8_t* d_geom = nullptr;
    uint8_t* d_ltab = nullptr;
    unsigned long long* d_cnt = nullptr;
    void* d_scan_tmp = nullptr;
    size_t scan_bytes = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, (unsigned long long*)nullptr, (unsigned long long*)nullptr,
                                  (int64_t)words);
    struct Scratch {
        void* p[4] = {nullptr, nullptr, nullptr, nullptr};
        cudaStream_t s = nullptr;
        ~Scratch() { for (void* q : p) if (q) cudaFreeAsync(q, s); }
    } scratch;
    scratch.s = e->stream;
    cudaMemPool_t pool = nullptr;
    LBF_CUDA(engine_pool((int)c.device, &pool));
    auto salloc = [&](void** p, size_t bytes, int slot) -> cudaError_t {
        const cudaError_t r = cudaMallocFromPoolAsync(p, bytes ? bytes : 1, pool, e->stream);
        if (r == cudaSuccess) scratch.p[slot] = *p;
        return r;
    };
    LBF_CUDA(salloc((void**)&d_geom, e->N, 0));
    LBF_CUDA(salloc((void**)&d_ltab, 512, 1));
    LBF_CUDA(salloc((void**)&d_cnt, (2 * words + 2) * sizeof(unsigned long long) + 8 * sizeof(uint32_t), 2));
    LBF_CUDA(salloc(&d_scan_tmp, scan_bytes, 3));
    unsigned long long* d_prefix = d_cnt + words;
    unsigned long long* d_total = d_prefix + words;
    uint32_t* d_used = reinterpret_cast<uint32_t*>(d_total + 2);
    uint8_t ltab[512];
    for (int l = 0; l < 256; ++l) {
        ltab[l] = is_fluid(labels[l].type) ? 1 : 0;
        ltab[256 + l] = (uint8_t)(is_fluid(labels[l].type) && labels[l].phase >= 0 && labels[l].phase < 2
                                  ? labels[l].phase : 0);
    }
    LBF_ALLOC(e->occ, words);
    LBF_CUDA(cudaMemcpyAsync(d_geom, geometry, e->N, cudaMemcpyHostToDevice, e->stream));
    LBF_CUDA(cudaMemcpyAsync(d_ltab, ltab, sizeof ltab, cudaMemcpyHostToDevice, e->stream));
    LBF_CUDA(cudaMemsetAsync(d_total, 0, 2 * sizeof(unsigned long long) + 8 * sizeof(uint32_t), e->stream));
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, (int)c.device);
    const unsigned cls_blocks = (unsigned)std::min<size_t>((words + 7) / 8, (size_t)sms * 16);
    classify_words<<<cls_blocks, 256, 0, e->stream>>>(d_geom, d_ltab, e->nx, e->W, words, e->occ, d_cnt, d_used);
    LBF_CUDA(cudaGetLastError());
    LBF_CUDA(cub::DeviceScan::ExclusiveSum(d_scan_tmp, scan_bytes, d_cnt, d_prefix, (int64_t)words, e->stream));
    finish_words<<<(unsigned)std::min<size_t>((words + 255) / 256, (size_t)sms * 16), 256, 0, e->stream>>>(
        d_cnt, d_prefix, words, e->occ, d_total);
    LBF_CUDA(cudaGetLastError());
    static_assert(kReduceMaxK * sizeof(double) >= 8 + 8 * sizeof(uint32_t), "pinned staging too small");
    LBF_CUDA(cudaMemcpyAsync(e->h_red, d_total, 8 + 8 * sizeof(uint32_t), cudaMemcpyDeviceToHost, e->stream));
    // d_total + 1 is unused padding; the bitmap follows it.
    LBF_CUDA(cudaMemcpyAsync(reinterpret_cast<char*>(e->h_red) + 8, d_used, 8 * sizeof(uint32_t),
                             cudaMemcpyDeviceToHost, e->stream));
    LBF_CUDA(cudaStreamSynchronize(e->stream));
    uint64_t count = 0;
    uint32_t used_bits[8];
    std::memcpy(&count, e->h_red, 8);
    std::memcpy(used_bits, reinterpret_cast<char*>(e->h_red) + 8, sizeof used_bits);
    for (int l = 0; l < 256; ++l) used[l] = (used_bits[l >> 5] >> (l & 31)) & 1u;
    {
        std::string m;
        if (validate_labels(c, labels, used, e->Q, e->D, phases, m) != LBF_OK) return bail(LBF_EINVAL, m);
    }
    // Element offsets inside a population buffer are 32-bit in the kernels.
    if ((count + 64) * (uint64_t)phases * (uint64_t)e->Q >= 0xffffffffull)
        return bail(LBF_EINVAL, "too many fluid nodes for one engine (phases * Q * nodes must stay below 2^32)");
    e->nf = (uint32_t)count;
    e->nfp = (uint32_t)((count + 63) / 64 * 64);
    if (e->nfp == 0) e->nfp = 64;

    // Body force per label, x/y/z (Simulator::forceForIndex, simulator.cpp:218-228:
    // Qp[dir] * value, Qp = e / |e|).
    const double sq = std::sqrt(2) / 2;
    std::vector<double> lforce(256 * 3, 0.0);
    for (int l = 0; l < 256; ++l) {
        const lbf_label& L = labels[l];
        if (L.type != LBF_GV || L.dir <= 0 || L.dir >= e->Q) continue;
        int nzc = 0;
        for (int a = 0; a < 3; ++a) nzc += ecomp(e->D, L.dir, a) != 0;
        for (int a = 0; a < 3; ++a) {
            const int ea = ecomp(e->D, L.dir, a);
            const double qp = nzc == 2 ? ea * sq : (double)ea;
            lforce[3 * l + a] = qp * L.value;
        }
    }
    bool uniform = true, first = true;
    double F0[3] = {0, 0, 0};
    for (int l = 0; l < 256 && uniform; ++l) {
        if (!used[l] || !is_fluid(labels[l].type)) continue;
        if (first) { for (int a = 0; a < 3; ++a) F0[a] = lforce[3 * l + a]; first = false; }
        else for (int a = 0; a < 3; ++a) if (lforce[3 * l + a] != F0[a]) uniform = false;
    }
    bool boundaries = false;
    for (int l = 0; l < 256; ++l) boundaries |= used[l] && (labels[l].type == LBF_PB || labels[l].type == LBF_VB);

    const size_t fcount = (size_t)phases * e->Q * e->nfp;
    for (int b = 0; b < 2; ++b) {
        char* p = nullptr;
        LBF_ALLOC(p, fcount * e->elem);
        e->f[b] = p;
        LBF_CUDA(cudaMemsetAsync(p, 0, fcount * e->elem, e->stream));
        if (blocked) {
            LBF_ALLOC(e->ex[b], e->nfp);
            LBF_CUDA(cudaMemsetAsync(e->ex[b], 0, e->nfp, e->stream));
        }
    }
    LBF_ALLOC(e->coord, e->nfp);
    LBF_ALLOC(e->label_force, 256 * 3);
    if (!uniform) LBF_ALLOC(e->node_label, e->nfp);
    if (c.model == LBF_MODEL_COLOR) LBF_ALLOC(e->node_phase, e->nfp);
    fill_nodes<<<cls_blocks, 256, 0, e->stream>>>(d_geom, e->occ, e->nx, e->ny, e->W, words, d_ltab + 256,
                                                   e->coord, e->node_label, e->node_phase);
    LBF_CUDA(cudaGetLastError());
    LBF_CUDA(cudaMemcpyAsync(e->label_force, lforce.data(), lforce.size() * sizeof(double), cudaMemcpyHostToDevice, e->stream));
    if (boundaries || c.model == LBF_MODEL_COLOR) {
        if ((rc = ensure_vox(e))) { std::string m = e->last_error; lbf_destroy(e); return fail(nullptr, rc, m); }
    }

    // Zou-He boundary nodes in compact order (SCSP::zouHeBoundary, scsp.cpp:188-275).
    std::vector<uint32_t> zh_node, zh_code;
    std::vector<double> zh_value;
    if (boundaries)
        for (uint32_t k = 0; k < e->nf; ++k) {
            const lbf_label& L = labels[geometry[e->vox[k]]];
            if (L.type != LBF_PB && L.type != LBF_VB) continue;
            zh_node.push_back(k);
            zh_code.push_back(((uint32_t)L.phase << 16) | ((L.type == LBF_VB ? kZouHeVB : kZouHePB) << 8) |
                              (uint32_t)L.dir);
            zh_value.push_back(L.value);
        }

    // Half-film bitmaps in the occupancy word layout (simulator.cpp:418-421).
    bool films = false;
    for (int l = 0; l < 256; ++l) films |= used[l] && labels[l].type == LBF_HF;
    if (films && (c.storage == LBF_STORE_FP16 || c.storage == LBF_STORE_BF16))
        return bail(LBF_EINVAL, "half-permeable films (HF) need FP64 or FP32 storage");
    if (films) {
        std::vector<uint32_t> fb[2] = {std::vector<uint32_t>(rows * e->W, 0u), std::vector<uint32_t>(rows * e->W, 0u)};
        for (size_t v = 0; v < e->N; ++v) {
            const lbf_label& L = labels[geometry[v]];
            if (L.type != LBF_HF) continue;
            const size_t r = v / e->nx, x = v % e->nx;
            fb[L.phase][r * e->W + (x >> 5)] |= 1u << (x & 31);
        }
        for (int k = 0; k < 2; ++k) {
            LBF_ALLOC(e->film_bits[k], fb[k].size());
            LBF_CUDA(cudaMemcpyAsync(e->film_bits[k], fb[k].data(), fb[k].size() * sizeof(uint32_t),
                                     cudaMemcpyHostToDevice, e->stream));
        }
    }
    if (!zh_node.empty()) {
        LBF_ALLOC(e->zh_node, zh_node.size());
        LBF_ALLOC(e->zh_code, zh_code.size());
        LBF_ALLOC(e->zh_value, zh_value.size());
        LBF_CUDA(cudaMemcpyAsync(e->zh_node, zh_node.data(), zh_node.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, e->stream));
        LBF_CUDA(cudaMemcpyAsync(e->zh_code, zh_code.data(), zh_code.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, e->stream));
        LBF_CUDA(cudaMemcpyAsync(e->zh_value, zh_value.data(), zh_value.size() * sizeof(double), cudaMemcpyHostToDevice, e->stream));
        if (c.model == LBF_MODEL_COLOR) {
            LBF_ALLOC(e->zh_num, zh_node.size());
            LBF_CUDA(cudaMemsetAsync(e->zh_num, 0, zh_node.size() * sizeof(double), e->stream));
        }
        e->zh.n = (uint32_t)zh_node.size();
        e->zh.num = e->zh_num;
        e->zh.node = e->zh_node;
        e->zh.code = e->zh_code;
        e->zh.value = e->zh_value;
    }
    LBF_ALLOC(e->rho0, e->nfp);
    LBF_ALLOC(e->u, 3 * (size_t)e->nfp);
    LBF_ALLOC(e->uprev, 3 * (size_t)e->nfp);
    LBF_ALLOC(e->uadj, 3 * (size_t)e->nfp);
    LBF_CUDA(cudaMemsetAsync(e->rho0, 0, e->nfp * sizeof(double), e->stream));
    LBF_CUDA(cudaMemsetAsync(e->u, 0, 3 * (size_t)e->nfp * sizeof(double), e->stream));
    LBF_CUDA(cudaMemsetAsync(e->uprev, 0, 3 * (size_t)e->nfp * sizeof(double), e->stream));
    LBF_CUDA(cudaMemsetAsync(e->uadj, 0, 3 * (size_t)e->nfp * sizeof(double), e->stream));
    LBF_ALLOC(e->err, 1);
    LBF_CUDA(cudaMemsetAsync(e->err, 0, sizeof(uint32_t), e->stream));
    LBF_ALLOC(e->partial, (size_t)kReduceBlocks * kReduceMaxK);
    LBF_ALLOC(e->red, kReduceMaxK);

    e->force.uniform = uniform ? 1 : 0;
    e->force.fx = F0[0]; e->force.fy = F0[1]; e->force.fz = F0[2];
    e->force.label = e->node_label;
    e->force.label_force = e->label_force;

    if (c.model == LBF_MODEL_SCSP) {
        e->sp.rho0 = c.rho[0];
        e->sp.inv_rho0 = 1.0 / c.rho[0];
        e->sp.rate = rates(c.collision == LBF_MRT, c.tau[0]);
        e->sp.mrt = c.collision == LBF_MRT ? 1 : 0;
    } else {
        // ColorFluid::initPhi (colorfluid.cpp:1131-1150).
        double alpha[2];
        alpha[0] = c.alpha0;
        alpha[1] = 1 - c.rho[0] / c.rho[1] * (1 - alpha[0]);
        for (int ph = 0; ph < 2; ++ph)
            for (int q = 0; q < e->Q; ++q) {
                double a, b;
                if (e->Q == 9) { a = (1 - alpha[ph]) / 5; b = (1 - alpha[ph]) / 20; }
                else { a = (1 - alpha[ph]) / 12; b = (1 - alpha[ph]) / 24; }
                int nzc = 0;
                for (int d = 0; d < 3; ++d) nzc += ecomp(e->D, q, d) != 0;
                e->cp.ai[ph][q] = q == 0 ? alpha[ph] : (nzc == 1 ? a : b);
            }
        e->cp.rho_ref[0] = c.rho[0]; e->cp.rho_ref[1] = c.rho[1];
        e->cp.relax0 = c.tau[0] / 2.0;
        e->cp.relax1 = c.tau[1] / 2.0;
        e->cp.uniform_tau = c.tau[0] == c.tau[1];
        e->cp.rate = rates(true, c.tau[0]);
        e->cp.ak = 2.25 * c.sigma;
        e->cp.beta = c.beta;

        // Wall data: mean contact angle per wall node (simulator.cpp:399-430),
        // deduplicated into a small table, and TibNorm per wall-normal code.
        static const double pi = 3.1415926535897932384626433832795;
        std::vector<uint16_t> aid(e->nf, 0);
        std::map<std::pair<uint64_t, uint64_t>, uint16_t> ids;
        std::vector<double> ang(2, 0.0);  // id 0 unused
        for (uint32_t k = 0; k < e->nf; ++k) {
            const size_t v = e->vox[k];
            const int x = (int)(v % e->nx), y = (int)((v / e->nx) % e->ny), z = (int)(v / ((size_t)e->nx * e->ny));
            double ca = 0;
            int nCA = 0;
            for (int q = 1; q < e->Q; ++q) {
                const int ax = (x + ecomp(e->D, q, 0) + e->nx) % e->nx;
                const int ay = (y + ecomp(e->D, q, 1) + e->ny) % e->ny;
                const int az = (z + ecomp(e->D, q, 2) + e->nz) % e->nz;
                const lbf_label& nb = labels[geometry[((size_t)az * e->ny + ay) * e->nx + ax]];
                if (is_solid(nb.type)) { ca += nb.type == LBF_SD ? nb.value : 0.0; nCA++; }
            }
            if (!nCA) continue;
            ca /= nCA;
            const double cs = std::cos(ca / 180.0 * pi), sn = std::sin(ca / 180.0 * pi);
            uint64_t bc, bs;
            std::memcpy(&bc, &cs, 8); std::memcpy(&bs, &sn, 8);
            auto key = std::make_pair(bc, bs);
            auto it = ids.find(key);
            if (it == ids.end()) {
                if (ids.size() >= 65535) return bail(LBF_EINVAL, "too many distinct wall contact angles");
                const uint16_t id = (uint16_t)(ids.size() + 1);
                it = ids.emplace(key, id).first;
                ang.push_back(cs); ang.push_back(sn);
            }
            aid[k] = it->second;
        }
        const int ncodes = e->D == 3 ? normal_codes<D3Q19>() : normal_codes<D2Q9>();
        const int tsz = e->D == 3 ? 9 : 4;
        std::vector<double> tib((size_t)ncodes * tsz, 0.0);
        if (e->D == 3) {
            for (int a = -5; a <= 5; ++a)
                for (int b = -5; b <= 5; ++b)
                    for (int cc = -5; cc <= 5; ++cc) {
                        const double n[3] = {(double)a, (double)b, (double)cc};
                        tib3(n, &tib[(size_t)normal_code<D3Q19>(a, b, cc) * 9]);
                    }
        } else {
            for (int a = -3; a <= 3; ++a)
                for (int b = -3; b <= 3; ++b) {
                    const double n[2] = {(double)a, (double)b};
                    tib2(n, &tib[(size_t)normal_code<D2Q9>(a, b, 0) * 4]);
                }
        }
        LBF_ALLOC(e->rho1, e->nfp);
        LBF_ALLOC(e->ind, e->nfp);
        LBF_ALLOC(e->indprev, e->nfp);
        LBF_ALLOC(e->indadj, e->nfp);
        LBF_ALLOC(e->dens, e->nfp);
        LBF_ALLOC(e->phid, e->N);
        fill_value<<<dense_blocks(e->N), 256, 0, e->stream>>>(e->phid, e->N, kSolidPhi);
        LBF_CUDA(cudaGetLastError());
        LBF_ALLOC(e->angle_id, e->nfp);
        LBF_ALLOC(e->angles, ang.size());
        LBF_ALLOC(e->tib, tib.size());
        LBF_CUDA(cudaMemsetAsync(e->rho1, 0, e->nfp * sizeof(double), e->stream));
        LBF_CUDA(cudaMemsetAsync(e->ind, 0, e->nfp * sizeof(double), e->stream));
        LBF_CUDA(cudaMemsetAsync(e->indprev, 0, e->nfp * sizeof(double), e->stream));
        LBF_CUDA(cudaMemsetAsync(e->indadj, 0, e->nfp * sizeof(double), e->stream));
        LBF_CUDA(cudaMemcpyAsync(e->angle_id, aid.data(), aid.size() * sizeof(uint16_t), cudaMemcpyHostToDevice, e->stream));
        LBF_CUDA(cudaMemcpyAsync(e->angles, ang.data(), ang.size() * sizeof(double), cudaMemcpyHostToDevice, e->stream));
        LBF_CUDA(cudaMemcpyAsync(e->tib, tib.data(), tib.size() * sizeof(double), cudaMemcpyHostToDevice, e->stream));
        LBF_CUDA(cudaStreamSynchronize(e->stream));
    }
    LBF_CUDA(cudaStreamSynchronize(e->stream));
#undef LBF_ALLOC
#undef LBF_CUDA
    *out = e;
    return LBF_OK;
}

void lbf_destroy(lbf_engine* e)
{
    if (!e) return;
    cudaSetDevice(e->cfg.device);
    if (e->stream) cudaStreamSynchronize(e->stream);
    void* ptrs[] = {e->f[0], e->f[1], e->ex[0], e->ex[1], e->occ, e->coord, e->node_label, e->node_phase, e->label_force,
                    e->rho0, e->rho1, e->u, e->uprev, e->uadj, e->ind, e->indprev, e->indadj,
                    e->dens, e->angle_id, e->angles, e->tib, e->err, e->partial, e->red,
                    e->zh_node, e->zh_code, e->zh_value, e->zh_num, e->dense_tmp, e->film_bits[0], e->film_bits[1],
                    e->stage, e->phid, e->solid_f[0], e->solid_f[1]};
    for (void* p : ptrs) if (p) cudaFreeAsync(p, e->stream);
    if (e->stream) cudaStreamSynchronize(e->stream);
    if (e->h_red) cudaFreeHost(e->h_red);
    if (e->stream) cudaStreamDestroy(e->stream);
    delete e;
}

int lbf_keep_solid_populations(lbf_engine* e)
{
    if (!e) return fail(e, LBF_EINVAL, "NULL engine");
    if (e->cfg.storage != LBF_STORE_FP64)
        return fail(e, LBF_EINVAL, "solid-voxel populations are kept with FP64 storage only");
    if (e->solid_f[0]) return LBF_OK;
    int rc = setdev(e);
    if (rc) return rc;
    e->ns = e->N - e->nf;
    const size_t count = (size_t)e->phases * e->Q * (e->ns ? e->ns : 1);
    for (int b = 0; b < 2; ++b) {
        if ((rc = dalloc(e, &e->solid_f[b], count))) return rc;
        LBF_CK(e, cudaMemsetAsync(e->solid_f[b], 0, count * sizeof(double), e->stream));
    }
    e->scur = 0;
    if ((rc = ensure_vox(e))) return rc;
    LBF_CK(e, cudaStreamSynchronize(e->stream));
    return LBF_OK;
}

int lbf_initialize(lbf_engine* e)
{
    if (!e) return fail(e, LBF_EINVAL, "NULL engine");
    int rc = setdev(e);
    if (rc) return rc;
    // A fresh t = 0 state starts with a clear device error word (and solid
    // voxels at 0, as the reference's initialisation leaves them).
    LBF_CK(e, cudaMemsetAsync(e->err, 0, sizeof(uint32_t), e->stream));
    if (e->solid_f[0])
        LBF_CK(e, cudaMemsetAsync(e->solid_f[e->scur], 0, (size_t)e->phases * e->Q * e->ns * sizeof(double), e->stream));
    const Grid g = grid_of(e);
    if (e->cfg.model == LBF_MODEL_SCSP)
        launch_scsp_init(e->D, (int)e->cfg.storage, g, e->force, e->cfg.rho[0], e->f[e->cur], e->ex[e->cur],
                         e->stream);
    else
        launch_color_init(e->D, (int)e->cfg.storage, g, e->force, e->cp, e->node_phase, e->f[e->cur], e->stream);
    launch_step(e, false, kOutMacros | kOutAdjacent);
    LBF_CK(e, cudaGetLastError());
    e->initialized = true;
    return LBF_OK;
}

int lbf_initialize_equilibrium(lbf_engine* e, const float* fields, uint32_t ld, uint32_t flags)
{
    if (!e) return fail(e, LBF_EINVAL, "NULL engine");
    if (!fields || ld < 4 || flags != 0) return fail(e, LBF_EINVAL, "fields must be non-NULL with ld >= 4; flags 0");
    if (e->cfg.model != LBF_MODEL_SCSP) return fail(e, LBF_EINVAL, "equilibrium initialisation is single-phase only");
    int rc = setdev(e);
    if (rc) return rc;
    // The fields usually come from another stream (an inference framework's,
    // or a copy from pageable memory that returns before its DMA lands):
    // wait for all queued device work so the read below sees them complete.
    LBF_CK(e, cudaDeviceSynchronize());
    cudaPointerAttributes pa{};
    if (cudaPointerGetAttributes(&pa, fields) != cudaSuccess || pa.type != cudaMemoryTypeDevice ||
        pa.device != e->cfg.device) {
        cudaGetLastError();
        return fail(e, LBF_EINVAL, "fields must be device memory of the engine's device");
    }
    LBF_CK(e, cudaMemsetAsync(e->err, 0, sizeof(uint32_t), e->stream));
    const Grid g = grid_of(e);
    launch_scsp_init_eq(e->D, (int)e->cfg.storage, g, e->force, e->cfg.rho[0], fields, ld, e->f[e->cur],
                        e->ex[e->cur], e->stream);
    launch_step(e, false, kOutMacros | kOutAdjacent);
    LBF_CK(e, cudaGetLastError());
    e->initialized = true;
    return LBF_OK;
}

namespace {
// Sums of the macroscopic fields over block^3 cubes: one thread per cube
// walks its voxels in (z, y, x) order (deterministic).  out[cube * 5 + k] =
// {sum rho, sum u_x, sum u_y, sum u_z, fluid voxels}.
__global__ void block_sums_kernel(const lbf::Grid g, const double* __restrict__ rho, const double* __restrict__ u,
                                  int b, int bx, int by, int bz, double* __restrict__ out)
{
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= (uint32_t)(bx * by * bz)) return;
    const int X0 = (int)(k % bx) * b, Y0 = (int)((k / bx) % by) * b, Z0 = (int)(k / ((uint32_t)bx * by)) * b;
    double s[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    for (int z = Z0; z < Z0 + b; ++z)
        for (int y = Y0; y < Y0 + b; ++y)
            for (int x = X0; x < X0 + b; ++x) {
                bool fluid;
                const uint32_t j = lbf::lookup(g, x, y, z, fluid);
                if (!fluid) continue;
                s[0] += rho[j];
                s[1] += u[j];
                s[2] += u[(size_t)g.nfp + j];
                s[3] += u[2 * (size_t)g.nfp + j];
                s[4] += 1.0;
            }
    for (int c = 0; c < 5; ++c) out[(size_t)k * 5 + c] = s[c];
}

}  // namespace

int lbf_block_sums(lbf_engine* e, uint32_t block, double* out, size_t n)
{
    if (!e || !out || block == 0) return fail(e, LBF_EINVAL, "NULL argument or zero block");
    if (e->cfg.model != LBF_MODEL_SCSP) return fail(e, LBF_EINVAL, "block sums are single-phase only");
    const uint32_t bzs = e->D == 2 ? 1u : block;
    if (e->nx % block || e->ny % block || e->nz % bzs) return fail(e, LBF_EINVAL, "grid is not a multiple of block");
    const int bx = e->nx / (int)block, by = e->ny / (int)block, bz = e->nz / (int)bzs;
    const size_t nb = (size_t)bx * by * bz;
    if (n != nb * 5) return fail(e, LBF_EINVAL, "out must hold 5 doubles per block");
    if (!e->initialized) return fail(e, LBF_ESTATE, "block sums before initialisation");
    int rc = setdev(e);
    if (rc) return rc;
    // out may be device memory of the engine's device (written in place) or host memory.
    cudaPointerAttributes pa{};
    const bool on_device = cudaPointerGetAttributes(&pa, out) == cudaSuccess && pa.type == cudaMemoryTypeDevice;
    cudaGetLastError();
    if (on_device && pa.device != e->cfg.device) return fail(e, LBF_EINVAL, "out is device memory of another device");
    double* d = on_device ? out : nullptr;
    if (!on_device) LBF_CK(e, cudaMalloc(&d, nb * 5 * sizeof(double)));
    const Grid g = grid_of(e);
    if (e->D == 2) {
        // 2-D: cubes are block x block squares of the single layer.
        block_sums_kernel<<<blocks_for((uint32_t)nb, 128), 128, 0, e->stream>>>(g, e->rho0, e->u, (int)block, bx, by,
                                                                                 1, d);
    } else {
        block_sums_kernel<<<blocks_for((uint32_t)nb, 128), 128, 0, e->stream>>>(g, e->rho0, e->u, (int)block, bx, by,
                                                                                 bz, d);
    }
    cudaError_t r = cudaGetLastError();
    if (!on_device && r == cudaSuccess)
        r = cudaMemcpyAsync(out, d, nb * 5 * sizeof(double), cudaMemcpyDeviceToHost, e->stream);
    if (r == cudaSuccess) r = cudaStreamSynchronize(e->stream);
    if (!on_device) cudaFree(d);
    if (r != cudaSuccess) return fail(e, LBF_ECUDA, std::string("block sums: ") + cudaGetErrorString(r));
    return LBF_OK;
}

int lbf_add_density(lbf_engine* e, const float* drho)
{
    if (!e || !drho) return fail(e, LBF_EINVAL, "NULL argument");
    if (e->cfg.model != LBF_MODEL_SCSP) return fail(e, LBF_EINVAL, "density increments are single-phase only");
    if (!e->initialized) return fail(e, LBF_ESTATE, "density increment before initialisation");
    int rc = setdev(e);
    if (rc) return rc;
    LBF_CK(e, cudaDeviceSynchronize());
    cudaPointerAttributes pa{};
    if (cudaPointerGetAttributes(&pa, drho) != cudaSuccess || pa.type != cudaMemoryTypeDevice ||
        pa.device != e->cfg.device) {
        cudaGetLastError();
        return fail(e, LBF_EINVAL, "drho must be device memory of the engine's device");
    }
    launch_scsp_add_density(e->D, (int)e->cfg.storage, grid_of(e), drho, e->f[e->cur], e->ex[e->cur],
                            e->cfg.rho[0], e->stream);
    LBF_CK(e, cudaGetLastError());
    return LBF_OK;
}

int lbf_step(lbf_engine* e, uint32_t nsteps, uint32_t flags)
{
    if (!e) return fail(e, LBF_EINVAL, "NULL engine");
    if (!e->initialized) return fail(e, LBF_ESTATE, "lbf_step before lbf_initialize or lbf_set_populations");
    int rc = setdev(e);
    if (rc) return rc;
    const int out = (flags & LBF_STEP_MACROS ? kOutMacros : 0) | (flags & LBF_STEP_ADJACENT ? kOutAdjacent : 0);
    for (uint32_t s = 0; s < nsteps; ++s) launch_step(e, true, s + 1 == nsteps ? out : 0);
    LBF_CK(e, cudaGetLastError());
    return LBF_OK;
}

int lbf_get_populations(lbf_engine* e, double* host, size_t n)
{
    if (!e || !host) return fail(e, LBF_EINVAL, "NULL argument");
    const size_t need = (size_t)e->phases * e->Q * e->N;
    if (n != need) return fail(e, LBF_EINVAL, "population buffer must hold phases*Q*N doubles");
    int rc = setdev(e);
    if (rc) return rc;
    if ((rc = ensure_vox(e))) return rc;
    std::vector<double> compact;
    rc = expand_to_host(e, compact);
    if (rc) return rc;
    std::memset(host, 0, n * sizeof(double));
    for (int p = 0; p < e->phases; ++p)
        for (int q = 0; q < e->Q; ++q) {
            const double* src = compact.data() + ((size_t)p * e->Q + q) * e->nfp;
            double* dst = host + ((size_t)p * e->Q + q) * e->N;
            for (uint32_t k = 0; k < e->nf; ++k) dst[e->vox[k]] = src[k];
        }
    if (e->solid_f[0]) {
        // Solid voxels' streamed populations (lbf_keep_solid_populations).
        const size_t blocks = (size_t)e->phases * e->Q;
        std::vector<double> sv(blocks * e->ns);
        if (!sv.empty()) {
            LBF_CK(e, cudaMemcpyAsync(sv.data(), e->solid_f[e->scur], sv.size() * sizeof(double),
                                      cudaMemcpyDeviceToHost, e->stream));
            LBF_CK(e, cudaStreamSynchronize(e->stream));
        }
        size_t k = 0, si = 0;
        for (size_t v = 0; v < e->N; ++v) {
            if (k < e->nf && e->vox[k] == v) { ++k; continue; }
            for (size_t b = 0; b < blocks; ++b) host[b * e->N + v] = sv[b * e->ns + si];
            ++si;
        }
    }
    return LBF_OK;
}

int lbf_set_populations(lbf_engine* e, const double* host, size_t n)
{
    if (!e || !host) return fail(e, LBF_EINVAL, "NULL argument");
    const size_t need = (size_t)e->phases * e->Q * e->N;
    if (n != need) return fail(e, LBF_EINVAL, "population buffer must hold phases*Q*N doubles");
    int rc = setdev(e);
    if (rc) return rc;
    if ((rc = ensure_vox(e))) return rc;
    const size_t count = (size_t)e->phases * e->Q * e->nfp;
    std::vector<double> compact(count, 0.0);
    for (int p = 0; p < e->phases; ++p)
        for (int q = 0; q < e->Q; ++q) {
            const double* src = host + ((size_t)p * e->Q + q) * e->N;
            double* dst = compact.data() + ((size_t)p * e->Q + q) * e->nfp;
            for (uint32_t k = 0; k < e->nf; ++k) dst[k] = src[e->vox[k]];
        }
    if (e->solid_f[0]) {
        // Solid voxels' values of the checkpoint (scsp.cpp:277-302 writes them).
        const size_t blocks = (size_t)e->phases * e->Q;
        std::vector<double> sv(blocks * e->ns);
        size_t k = 0, si = 0;
        for (size_t v = 0; v < e->N; ++v) {
            if (k < e->nf && e->vox[k] == v) { ++k; continue; }
            for (size_t b = 0; b < blocks; ++b) sv[b * e->ns + si] = host[b * e->N + v];
            ++si;
        }
        if (!sv.empty())
            LBF_CK(e, cudaMemcpyAsync(e->solid_f[e->scur], sv.data(), sv.size() * sizeof(double),
                                      cudaMemcpyHostToDevice, e->stream));
    }
    if (e->cfg.storage == LBF_STORE_FP64) {
        LBF_CK(e, cudaMemcpyAsync(e->f[e->cur], compact.data(), count * sizeof(double), cudaMemcpyHostToDevice, e->stream));
        LBF_CK(e, cudaStreamSynchronize(e->stream));
    } else {
        double* tmp = nullptr;
        LBF_CK(e, cudaMalloc(&tmp, count * sizeof(double)));
        cudaError_t r = cudaMemcpyAsync(tmp, compact.data(), count * sizeof(double), cudaMemcpyHostToDevice, e->stream);
        if (r == cudaSuccess) {
            if (e->D == 3) convert<D3Q19>(e, false, e->f[e->cur], tmp);
            else convert<D2Q9>(e, false, e->f[e->cur], tmp);
            r = cudaGetLastError();
        }
        if (r == cudaSuccess) r = cudaStreamSynchronize(e->stream);
        cudaFree(tmp);
        if (r != cudaSuccess) return fail(e, LBF_ECUDA, std::string("set populations: ") + cudaGetErrorString(r));
    }
    e->initialized = true;
    return LBF_OK;
}


int lbf_fields_dense_async(lbf_engine* e, double* out, size_t n)
{
    if (!e || !out) return fail(e, LBF_EINVAL, "NULL argument");
    const bool color = e->cfg.model == LBF_MODEL_COLOR;
    const int per = 1 + (color ? 1 : 0) + e->D;
    if (n != (size_t)per * e->N)
        return fail(e, LBF_EINVAL, "fields buffer must hold (1 + color + dims) * nx*ny*nz doubles");
    int rc = setdev(e);
    if (rc) return rc;
    const Dest dst = destination(e, out);
    if (dst == Dest::kNone)
        return fail(e, LBF_EINVAL, "out must be device memory of the engine's device or page-locked host memory");
    if (e->N == 0) return LBF_OK;
    const Grid g = grid_of(e);
    const double* r1 = color ? e->rho1 : nullptr;
    if (dst == Dest::kDevice) {
        fields_range_kernel<<<dense_blocks(e->N), 256, 0, e->stream>>>(g, e->rho0, r1, e->u, e->D, 0, e->N, out);
        LBF_CK(e, cudaGetLastError());
        return LBF_OK;
    }
    double* st = nullptr;
    if ((rc = stage_buffer(e, &st))) return rc;
    const size_t chunk = kStageBytes / (sizeof(double) * per);
    const size_t vec = (size_t)(1 + (color ? 1 : 0)) * e->N;   // offset of the velocity array in out
    for (size_t v0 = 0; v0 < e->N; v0 += chunk) {
        const size_t r = std::min(chunk, e->N - v0);
        fields_range_kernel<<<dense_blocks(r), 256, 0, e->stream>>>(g, e->rho0, r1, e->u, e->D, v0, r, st);
        LBF_CK(e, cudaGetLastError());
        LBF_CK(e, cudaMemcpyAsync(out + v0, st, r * sizeof(double), cudaMemcpyDeviceToHost, e->stream));
        if (color)
            LBF_CK(e, cudaMemcpyAsync(out + e->N + v0, st + r, r * sizeof(double), cudaMemcpyDeviceToHost, e->stream));
        LBF_CK(e, cudaMemcpyAsync(out + vec + (size_t)e->D * v0, st + (size_t)(1 + (color ? 1 : 0)) * r,
                                  (size_t)e->D * r * sizeof(double), cudaMemcpyDeviceToHost, e->stream));
    }
    return LBF_OK;
}

int lbf_populations_dense_async(lbf_engine* e, double* out, size_t n)
{
    if (!e || !out) return fail(e, LBF_EINVAL, "NULL argument");
    const size_t blocks = (size_t)e->phases * e->Q;
    if (n != blocks * e->N) return fail(e, LBF_EINVAL, "population buffer must hold phases*Q*N doubles");
    int rc = setdev(e);
    if (rc) return rc;
    const Dest dst = destination(e, out);
    if (dst == Dest::kNone)
        return fail(e, LBF_EINVAL, "out must be device memory of the engine's device or page-locked host memory");
    const double* src = static_cast<const double*>(e->f[e->cur]);
    if (e->cfg.storage != LBF_STORE_FP64) {
        if (!e->dense_tmp && (rc = dalloc(e, &e->dense_tmp, blocks * e->nfp))) return rc;
        if (e->D == 3) convert<D3Q19>(e, true, e->f[e->cur], e->dense_tmp);
        else convert<D2Q9>(e, true, e->f[e->cur], e->dense_tmp);
        LBF_CK(e, cudaGetLastError());
        src = e->dense_tmp;
    }
    if (e->N == 0) return LBF_OK;
    const Grid g = grid_of(e);
    if (dst == Dest::kDevice) {
        populations_range_kernel<<<dense_blocks(e->N), 256, 0, e->stream>>>(g, src, (int)blocks, 0, e->N, out, e->err,
                                                                            e->solid_f[e->scur], e->ns);
        LBF_CK(e, cudaGetLastError());
        return LBF_OK;
    }
    double* st = nullptr;
    if ((rc = stage_buffer(e, &st))) return rc;
    const size_t chunk = kStageBytes / (sizeof(double) * blocks);
    for (size_t v0 = 0; v0 < e->N; v0 += chunk) {
        const size_t r = std::min(chunk, e->N - v0);
        populations_range_kernel<<<dense_blocks(r), 256, 0, e->stream>>>(g, src, (int)blocks, v0, r, st, e->err,
                                                                         e->solid_f[e->scur], e->ns);
        LBF_CK(e, cudaGetLastError());
        // [block][r] in the stage -> [block][N] at voxel v0 in out.
        LBF_CK(e, cudaMemcpy2DAsync(out + v0, e->N * sizeof(double), st, r * sizeof(double), r * sizeof(double),
                                    blocks, cudaMemcpyDeviceToHost, e->stream));
    }
    return LBF_OK;
}

int lbf_host_alloc(size_t bytes, void** out)
{
    if (!out) return fail(nullptr, LBF_EINVAL, "lbf_host_alloc: out is NULL");
    *out = nullptr;
    const cudaError_t r = cudaHostAlloc(out, bytes ? bytes : 1, cudaHostAllocPortable | cudaHostAllocMapped);
    if (r != cudaSuccess) {
        *out = nullptr;
        return fail(nullptr, r == cudaErrorMemoryAllocation ? LBF_ENOMEM : LBF_ECUDA,
                    std::string("cudaHostAlloc: ") + cudaGetErrorString(r));
    }
    return LBF_OK;
}

void lbf_host_free(void* p)
{
    if (p) cudaFreeHost(p);
}

int lbf_get_macros(lbf_engine* e, double* rho0, double* rho1, double* u)
{
    if (!e) return fail(e, LBF_EINVAL, "NULL engine");
    int rc = setdev(e);
    if (rc) return rc;
    if ((rc = ensure_vox(e))) return rc;
    std::vector<double> buf((size_t)e->nfp * 3);
    auto scatter = [&](const double* dsrc, double* dst, int comps) -> int {
        LBF_CK(e, cudaMemcpyAsync(buf.data(), dsrc, (size_t)comps * e->nfp * sizeof(double), cudaMemcpyDeviceToHost, e->stream));
        LBF_CK(e, cudaStreamSynchronize(e->stream));
        std::memset(dst, 0, (size_t)comps * e->N * sizeof(double));
        for (int c = 0; c < comps; ++c)
            for (uint32_t k = 0; k < e->nf; ++k) dst[(size_t)c * e->N + e->vox[k]] = buf[(size_t)c * e->nfp + k];
        return LBF_OK;
    };
    if (rho0 && (rc = scatter(e->rho0, rho0, 1))) return rc;
    if (rho1) {
        if (e->rho1) { if ((rc = scatter(e->rho1, rho1, 1))) return rc; }
        else std::memset(rho1, 0, e->N * sizeof(double));
    }
    if (u && (rc = scatter(e->u, u, 3))) return rc;
    return LBF_OK;
}

int lbf_convergence(lbf_engine* e, int first, double out[6])
{
    if (!e || !out) return fail(e, LBF_EINVAL, "NULL argument");
    int rc = setdev(e);
    if (rc) return rc;
    for (int k = 0; k < 6; ++k) out[k] = 0.0;
    const bool color = e->cfg.model == LBF_MODEL_COLOR;
    if (!first) {
        ConvergenceFn fn{e->u, e->uprev, e->uadj, e->ind, e->indprev, e->indadj, e->nfp, color ? 1 : 0};
        double r[ConvergenceFn::K];
        if ((rc = run_reduce(e, fn, r))) return rc;
        for (int k = 0; k < ConvergenceFn::K; ++k) out[k] = r[k];
    }
    LBF_CK(e, cudaMemcpyAsync(e->uprev, e->u, 3 * (size_t)e->nfp * sizeof(double), cudaMemcpyDeviceToDevice, e->stream));
    if (color)
        LBF_CK(e, cudaMemcpyAsync(e->indprev, e->ind, (size_t)e->nfp * sizeof(double), cudaMemcpyDeviceToDevice, e->stream));
    LBF_CK(e, cudaStreamSynchronize(e->stream));
    return LBF_OK;
}

int lbf_report_sums(lbf_engine* e, uint32_t axis, uint32_t lo, uint32_t hi, double out[10])
{
    if (!e || !out || axis > 2) return fail(e, LBF_EINVAL, "invalid argument");
    int rc = setdev(e);
    if (rc) return rc;
    ReportFn fn{e->coord, e->u, e->rho0, e->rho1, e->nfp, (int)axis, (int)lo, (int)hi};
    return run_reduce(e, fn, out);
}

int lbf_flux_sums(lbf_engine* e, double out[9])
{
    if (!e || !out) return fail(e, LBF_EINVAL, "NULL argument");
    int rc = setdev(e);
    if (rc) return rc;
    FluxFn fn{e->u, e->rho0, e->rho1, e->nfp};
    return run_reduce(e, fn, out);
}

int lbf_link_mask(lbf_engine* e, uint32_t* host, size_t n)
{
    if (!e || !host || n != e->N) return fail(e, LBF_EINVAL, "mask buffer must hold nx*ny*nz entries");
    int rc = setdev(e);
    if (rc) return rc;
    uint32_t* d = nullptr;
    LBF_CK(e, cudaMalloc(&d, e->N * sizeof(uint32_t)));
    const unsigned t = 256;
    const unsigned b = (unsigned)((e->N + t - 1) / t);
    if (e->D == 3) link_mask_kernel<D3Q19><<<b, t, 0, e->stream>>>(grid_of(e), d, e->N);
    else link_mask_kernel<D2Q9><<<b, t, 0, e->stream>>>(grid_of(e), d, e->N);
    cudaError_t r = cudaGetLastError();
    if (r == cudaSuccess) r = cudaMemcpyAsync(host, d, e->N * sizeof(uint32_t), cudaMemcpyDeviceToHost, e->stream);
    if (r == cudaSuccess) r = cudaStreamSynchronize(e->stream);
    cudaFree(d);
    if (r != cudaSuccess) return fail(e, LBF_ECUDA, std::string("link mask: ") + cudaGetErrorString(r));
    return LBF_OK;
}

int lbf_status(lbf_engine* e, uint32_t* bits)
{
    if (!e || !bits) return fail(e, LBF_EINVAL, "NULL argument");
    int rc = setdev(e);
    if (rc) return rc;
    LBF_CK(e, cudaStreamSynchronize(e->stream));
    LBF_CK(e, cudaMemcpy(bits, e->err, sizeof(uint32_t), cudaMemcpyDeviceToHost));
    return LBF_OK;
}

int lbf_synchronize(lbf_engine* e)
{
    if (!e) return fail(e, LBF_EINVAL, "NULL engine");
    int rc = setdev(e);
    if (rc) return rc;
    LBF_CK(e, cudaStreamSynchronize(e->stream));
    return LBF_OK;
}

uint64_t lbf_fluid_nodes(const lbf_engine* e) { return e ? e->nf : 0; }
void* lbf_stream(const lbf_engine* e) { return e ? (void*)e->stream : nullptr; }
uint64_t lbf_device_bytes(const lbf_engine* e) { return e ? e->bytes : 0; }

const char* lbf_last_error(const lbf_engine* e)
{
    return e ? e->last_error.c_str() : g_create_error.c_str();
}

}  // extern "C"
