// Many independent geometries in one launch (the batched form).
//
// All geometries' fluid nodes are packed into one node list: geometry g owns
// nodes [node_base_g, node_base_g + nf_g), in its own voxel order.  Each
// geometry keeps its own occupancy words, whose prefix counts start at
// node_base_g, so the single-geometry pull lookup returns global node
// indices unchanged.  The node list is cut into tiles of consecutive nodes of
// one geometry (all-solid regions produce no nodes and so no tiles); a grid of
// resident blocks walks the tile list of the still-active geometries every
// step, reading each tile's geometry size and collision rates.  Steps are
// replayed from a captured CUDA graph.  FP16 storage rounds stochastically
// with the single engine's per-step seeds: the step count lives in device
// memory (a pair of words indexed by the buffer parity: a step reads one and
// its first thread writes the next count into the other), so graph replays
// see a new seed every step without any host involvement.  Per-geometry reductions write one
// partial per tile and then sum each geometry's tiles in order
// (deterministic), so every geometry can be tested for convergence and
// retired on its own.  lbf_batch_autotune picks the tile size and grid shape
// by timing candidates on the batch itself.
#include "../../include/lbflow.h"
#include "internal.h"
#include "reduce.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

using namespace lbf;

namespace {

struct BatchGeom {
    int nx, ny, nz, W;
    uint32_t occ_base;      // first occupancy word of the geometry
    uint32_t node_base;     // first global node
    uint32_t nf;            // fluid nodes
    double sp, sm;          // collision rates
};

struct Tile { uint32_t geom, first, count; };

thread_local std::string g_batch_error;

int bfail(lbf_batch* b, int code, const std::string& m);

template <class L, class S, bool PULL>
__global__ void __launch_bounds__(256)
batch_step(const BatchGeom* __restrict__ geoms, const Tile* __restrict__ tiles, uint32_t ntiles,
           const uint2* __restrict__ occ, const uint32_t* __restrict__ coord, uint32_t nfp,
           const Force F, const double rho0, const typename S::T* __restrict__ fin,
           typename S::T* __restrict__ fout, Macros mo, const int out, uint32_t* __restrict__ err,
           uint32_t* __restrict__ step_count, const int parity)
{
    // Stochastic rounding seed of this step (16-bit float storage, pull
    // steps): count k = 1, 2, ... of pull steps, as the single engine seeds
    // them.  This launch reads step_count[parity] and publishes k into
    // step_count[parity ^ 1] for the next launch, never the word it reads.
    uint32_t seed = 0;
    if (S::dither && PULL && step_count) {
        const uint32_t k = step_count[parity] + 1u;
        seed = (k * 2654435761u) | 1u;
        if (blockIdx.x == 0 && threadIdx.x == 0) step_count[parity ^ 1] = k;
    }
    for (uint32_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const Tile tl = tiles[t];
        const BatchGeom G = geoms[tl.geom];
        Grid g;
        g.nx = G.nx; g.ny = G.ny; g.nz = G.nz; g.W = G.W;
        g.nf = G.node_base + G.nf;
        g.nfp = nfp;
        g.occ = occ + G.occ_base;
        g.coord = coord;
        ScspParams P;
        P.rho0 = rho0;
        P.inv_rho0 = 1.0 / rho0;
        P.rate.sp = G.sp;
        P.rate.sm = G.sm;
        P.seed = seed;
        P.node0 = G.node_base;
        for (uint32_t k = threadIdx.x; k < tl.count; k += blockDim.x)
            scsp_update<L, S, PULL, true>(g, F, P, fin, fout, tl.first + k, mo, out, err, nullptr, nullptr);
    }
}

// Per-tile partial sums of a reduction functor (one block per tile).
template <class Fn>
__global__ void __launch_bounds__(256)
tile_sums(const Fn fn, const Tile* __restrict__ tiles, double* __restrict__ partial)
{
    constexpr int K = Fn::K;
    const Tile tl = tiles[blockIdx.x];
    double acc[K];
#pragma unroll
    for (int k = 0; k < K; ++k) acc[k] = 0.0;
    for (uint32_t j = threadIdx.x; j < tl.count; j += blockDim.x) fn(tl.first + j, acc);
    __shared__ double sm[K][8];
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
    if (threadIdx.x < K) {
        const int k = threadIdx.x;
        double v = sm[k][0];
        for (int w = 1; w < (int)(blockDim.x / 32); ++w) v = Fn::is_max(k) ? fmax(v, sm[k][w]) : v + sm[k][w];
        partial[(size_t)blockIdx.x * K + k] = v;
    }
}

// Sum each geometry's tile partials in tile order (one thread per geometry).
template <class Fn>
__global__ void geom_sums(const double* __restrict__ partial, const uint32_t* __restrict__ tile_first,
                          const uint32_t* __restrict__ tile_count, uint32_t ngeom, double* __restrict__ out)
{
    constexpr int K = Fn::K;
    const uint32_t gi = blockIdx.x * blockDim.x + threadIdx.x;
    if (gi >= ngeom) return;
    for (int k = 0; k < K; ++k) {
        double v = 0.0;
        for (uint32_t t = 0; t < tile_count[gi]; ++t) {
            const double p = partial[(size_t)(tile_first[gi] + t) * K + k];
            v = Fn::is_max(k) ? fmax(v, p) : v + p;
        }
        out[(size_t)gi * K + k] = v;
    }
}

}  // namespace

struct lbf_batch {
    uint32_t count = 0;
    int device = 0;
    uint32_t storage = LBF_STORE_FP64;
    double rho0 = 1.0;
    size_t elem = 8;
    uint32_t nf = 0, nfp = 0;
    std::vector<BatchGeom> geoms;
    std::vector<std::vector<uint32_t>> vox;   // per geometry: voxel of each local node
    std::vector<uint8_t> active;
    // device
    BatchGeom* d_geoms = nullptr;
    uint2* d_occ = nullptr;
    uint32_t* d_coord = nullptr;
    uint8_t* d_label = nullptr;
    double* d_label_force = nullptr;
    void* f[2] = {nullptr, nullptr};
    int cur = 0;
    double *rho = nullptr, *u = nullptr, *uprev = nullptr, *uadj = nullptr;
    uint32_t* err = nullptr;
    Tile* d_tiles_all = nullptr;      // every tile, geometry order
    Tile* d_tiles_active = nullptr;   // the schedule of active geometries
    uint32_t* d_tile_first = nullptr;
    uint32_t* d_tile_count = nullptr;
    double* d_partial = nullptr;
    double* d_out = nullptr;
    uint32_t* d_step = nullptr;       // pull-step count, two words by buffer parity (FP16 rounding seeds)
    uint32_t ntiles_all = 0, ntiles_active = 0;
    size_t tile_cap = 0;              // capacity of the device tile arrays
    std::vector<Tile> tiles_all;
    std::vector<uint32_t> tile_first, tile_count;
    Force force{};
    cudaStream_t stream = nullptr;
    // launch shape (autotuned)
    unsigned threads = 128, tile_nodes = 256, grid = 0;
    // CUDA graph of `graph_steps` plain steps
    cudaGraphExec_t graph = nullptr;
    uint32_t graph_steps = 0;
    int graph_cur = 0;     // buffer parity the graph was captured with
    bool initialized = false;
    std::string last_error;
};

namespace {

int bfail(lbf_batch* b, int code, const std::string& m)
{
    if (b) b->last_error = m;
    else g_batch_error = m;
    return code;
}

#define BCK(b, call)                                                                      \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess) return bfail(b, LBF_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

Macros batch_macros(const lbf_batch* b)
{
    Macros m{};
    m.rho0 = b->rho; m.u = b->u; m.uadj = b->uadj;
    return m;
}

template <class S>
void launch_batch(lbf_batch* b, bool pull, int out, const Tile* tiles, uint32_t ntiles, unsigned grid)
{
    using T = typename S::T;
    if (!ntiles) return;
    const T* fin = (const T*)b->f[b->cur];
    T* fout = (T*)b->f[b->cur ^ 1];
    if (pull)
        batch_step<D3Q19, S, true><<<grid, b->threads, 0, b->stream>>>(
            b->d_geoms, tiles, ntiles, b->d_occ, b->d_coord, b->nfp, b->force, b->rho0, fin, fout,
            batch_macros(b), out, b->err, b->d_step, b->cur);
    else
        batch_step<D3Q19, S, false><<<grid, b->threads, 0, b->stream>>>(
            b->d_geoms, tiles, ntiles, b->d_occ, b->d_coord, b->nfp, b->force, b->rho0, fin, fout,
            batch_macros(b), out, b->err, b->d_step, b->cur);
}

void batch_launch(lbf_batch* b, bool pull, int out, bool all_tiles = false)
{
    const Tile* tiles = all_tiles ? b->d_tiles_all : b->d_tiles_active;
    const uint32_t n = all_tiles ? b->ntiles_all : b->ntiles_active;
    const unsigned grid = std::max(1u, std::min(b->grid, n));
    switch (b->storage) {
    case LBF_STORE_FP64: launch_batch<StoreF64>(b, pull, out, tiles, n, grid); break;
    case LBF_STORE_FP16: launch_batch<StoreF16<D3Q19>>(b, pull, out, tiles, n, grid); break;
    default: launch_batch<StoreF32<D3Q19>>(b, pull, out, tiles, n, grid); break;
    }
    b->cur ^= 1;
}

void drop_graph(lbf_batch* b)
{
    if (b->graph) cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
    b->graph_steps = 0;
}

// Build the tile list for the current tile size and upload it.
int build_tiles(lbf_batch* b)
{
    b->tiles_all.clear();
    b->tile_first.assign(b->count, 0);
    b->tile_count.assign(b->count, 0);
    for (uint32_t g = 0; g < b->count; ++g) {
        b->tile_first[g] = (uint32_t)b->tiles_all.size();
        const BatchGeom& G = b->geoms[g];
        for (uint32_t k = 0; k < G.nf; k += b->tile_nodes)
            b->tiles_all.push_back(Tile{g, G.node_base + k, std::min(b->tile_nodes, G.nf - k)});
        b->tile_count[g] = (uint32_t)b->tiles_all.size() - b->tile_first[g];
    }
    b->ntiles_all = (uint32_t)b->tiles_all.size();
    // Device tile arrays grow only (retiring geometries inside a run, which
    // rebuilds the active schedule, then makes no allocation).
    const size_t nt = std::max<size_t>(1, b->ntiles_all);
    if (nt > b->tile_cap) {
        cudaFree(b->d_tiles_all); cudaFree(b->d_tiles_active); cudaFree(b->d_partial);
        b->d_tiles_all = b->d_tiles_active = nullptr;
        b->d_partial = nullptr;
        b->tile_cap = 0;
        BCK(b, cudaMalloc(&b->d_tiles_all, nt * sizeof(Tile)));
        BCK(b, cudaMalloc(&b->d_tiles_active, nt * sizeof(Tile)));
        BCK(b, cudaMalloc(&b->d_partial, nt * kReduceMaxK * sizeof(double)));
        b->tile_cap = nt;
    }
    if (!b->d_tile_first) {
        BCK(b, cudaMalloc(&b->d_tile_first, std::max<size_t>(1, b->count) * sizeof(uint32_t)));
        BCK(b, cudaMalloc(&b->d_tile_count, std::max<size_t>(1, b->count) * sizeof(uint32_t)));
    }
    BCK(b, cudaMemcpyAsync(b->d_tiles_all, b->tiles_all.data(), b->ntiles_all * sizeof(Tile), cudaMemcpyHostToDevice, b->stream));
    BCK(b, cudaMemcpyAsync(b->d_tile_first, b->tile_first.data(), b->count * sizeof(uint32_t), cudaMemcpyHostToDevice, b->stream));
    BCK(b, cudaMemcpyAsync(b->d_tile_count, b->tile_count.data(), b->count * sizeof(uint32_t), cudaMemcpyHostToDevice, b->stream));
    // Active schedule: interleave geometries' tiles round-robin so that the
    // resident blocks share out large and small geometries evenly.
    std::vector<Tile> act;
    act.reserve(b->ntiles_all);
    uint32_t round = 0;
    bool more = true;
    while (more) {
        more = false;
        for (uint32_t g = 0; g < b->count; ++g) {
            if (!b->active[g] || round >= b->tile_count[g]) continue;
            act.push_back(b->tiles_all[b->tile_first[g] + round]);
            more = true;
        }
        ++round;
    }
    b->ntiles_active = (uint32_t)act.size();
    if (!act.empty())
        BCK(b, cudaMemcpyAsync(b->d_tiles_active, act.data(), act.size() * sizeof(Tile), cudaMemcpyHostToDevice, b->stream));
    BCK(b, cudaStreamSynchronize(b->stream));
    drop_graph(b);
    return LBF_OK;
}

int capture_graph(lbf_batch* b, uint32_t steps)
{
    drop_graph(b);
    cudaGraph_t g = nullptr;
    const int cur0 = b->cur;
    BCK(b, cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    for (uint32_t s = 0; s < steps; ++s) batch_launch(b, true, 0);
    cudaError_t r = cudaStreamEndCapture(b->stream, &g);
    b->cur = cur0;   // capture does not execute; the buffers are back where they were
    if (r != cudaSuccess) return bfail(b, LBF_ECUDA, std::string("graph capture: ") + cudaGetErrorString(r));
    r = cudaGraphInstantiate(&b->graph, g, 0);
    cudaGraphDestroy(g);
    if (r != cudaSuccess) { b->graph = nullptr; return bfail(b, LBF_ECUDA, std::string("graph instantiate: ") + cudaGetErrorString(r)); }
    b->graph_steps = steps;
    b->graph_cur = cur0;
    return LBF_OK;
}

template <class Fn>
int batch_reduce(lbf_batch* b, const Fn& fn, double* out)
{
    if (!b->ntiles_all) { std::memset(out, 0, sizeof(double) * Fn::K * b->count); return LBF_OK; }
    tile_sums<Fn><<<b->ntiles_all, 256, 0, b->stream>>>(fn, b->d_tiles_all, b->d_partial);
    geom_sums<Fn><<<(b->count + 127) / 128, 128, 0, b->stream>>>(b->d_partial, b->d_tile_first, b->d_tile_count,
                                                                 b->count, b->d_out);
    BCK(b, cudaGetLastError());
    BCK(b, cudaMemcpyAsync(out, b->d_out, sizeof(double) * Fn::K * b->count, cudaMemcpyDeviceToHost, b->stream));
    BCK(b, cudaStreamSynchronize(b->stream));
    return LBF_OK;
}

}  // namespace

extern "C" {

int lbf_batch_create(const lbf_batch_geometry* geoms, uint32_t count, const lbf_label labels[256],
                     uint32_t collision, uint32_t storage, int32_t device, double rho0, lbf_batch** out)
{
    if (!out) return bfail(nullptr, LBF_EINVAL, "out is NULL");
    *out = nullptr;
    if (!geoms || !labels || count == 0) return bfail(nullptr, LBF_EINVAL, "no geometries");
    if (collision != LBF_SRT && collision != LBF_MRT) return bfail(nullptr, LBF_EINVAL, "unknown collision model");
    if (storage != LBF_STORE_FP64 && storage != LBF_STORE_FP32 && storage != LBF_STORE_FP16)
        return bfail(nullptr, LBF_EINVAL, "batch storage must be FP64, FP32 or FP16");
    if (!(rho0 > 0.0)) return bfail(nullptr, LBF_EINVAL, "rho0 must be positive");
    lbf_batch* b = new lbf_batch();
    b->count = count;
    b->device = device;
    b->storage = storage;
    b->rho0 = rho0;
    b->elem = storage == LBF_STORE_FP64 ? 8 : (storage == LBF_STORE_FP32 ? 4 : 2);
    auto bail = [&](int code, const std::string& m) { lbf_batch_destroy(b); return bfail(nullptr, code, m); };

    // Forces per label (x, y, z): Qp[dir] * value (simulator.cpp:218-228).
    const double sq = std::sqrt(2) / 2;
    std::vector<double> lforce(256 * 3, 0.0);
    for (int l = 0; l < 256; ++l) {
        const lbf_label& L = labels[l];
        if (L.type != LBF_GV) continue;
        if (L.dir <= 0 || L.dir >= 19 || !std::isfinite(L.value))
            return bail(LBF_EINVAL, "Invalid body-force direction or magnitude.");
        const int e[3] = {D3Q19::ex(L.dir), D3Q19::ey(L.dir), D3Q19::ez(L.dir)};
        const int nzc = (e[0] != 0) + (e[1] != 0) + (e[2] != 0);
        for (int a = 0; a < 3; ++a) lforce[3 * l + a] = (nzc == 2 ? e[a] * sq : (double)e[a]) * L.value;
    }
    auto fluid = [&](uint8_t v) { return labels[v].type == LBF_VD || labels[v].type == LBF_GV; };
    auto solid = [&](uint8_t v) { return labels[v].type == LBF_BB || labels[v].type == LBF_SD; };

    std::vector<uint2> occ;
    std::vector<uint32_t> coord;
    std::vector<uint8_t> nlabel;
    bool used[256] = {};
    uint64_t base = 0;
    b->geoms.resize(count);
    b->vox.resize(count);
    for (uint32_t gi = 0; gi < count; ++gi) {
        const lbf_batch_geometry& G = geoms[gi];
        if (G.nx == 0 || G.ny == 0 || G.nz == 0 || G.nx > 2048 || G.ny > 2048 || G.nz > 1024 || !G.labels)
            return bail(LBF_EINVAL, "geometry " + std::to_string(gi) + ": invalid dimensions");
        if (!std::isfinite(G.tau) || G.tau <= 0.5)
            return bail(LBF_EINVAL, "geometry " + std::to_string(gi) + ": relaxation time must exceed 0.5");
        const int W = (int)((G.nx + 31) / 32);
        BatchGeom& B = b->geoms[gi];
        B.nx = (int)G.nx; B.ny = (int)G.ny; B.nz = (int)G.nz; B.W = W;
        B.occ_base = (uint32_t)occ.size();
        B.node_base = (uint32_t)base;
        const double sp = 1.0 / G.tau;
        B.sp = sp;
        B.sm = collision == LBF_MRT ? 8.0 * (2.0 - sp) / (8.0 - sp) : sp;
        const size_t rows = (size_t)G.nz * G.ny;
        for (size_t r = 0; r < rows; ++r)
            for (int w = 0; w < W; ++w) {
                uint32_t bits = 0;
                for (int k = 0; k < 32; ++k) {
                    const uint32_t x = (uint32_t)(w * 32 + k);
                    if (x >= G.nx) break;
                    const uint8_t v = G.labels[r * G.nx + x];
                    if (labels[v].type == 0) return bail(LBF_EINVAL, "geometry label " + std::to_string(v) + " is not defined");
                    if (!fluid(v) && !solid(v))
                        return bail(LBF_EINVAL, "label " + std::to_string(v) + ": only VD, GV, BB and SD labels are supported");
                    if (fluid(v)) { bits |= 1u << k; used[v] = true; }
                }
                occ.push_back(make_uint2(bits, (uint32_t)base));
                base += (uint64_t)__builtin_popcount(bits);
            }
        B.nf = (uint32_t)(base - B.node_base);
        b->vox[gi].reserve(B.nf);
        const size_t N = rows * G.nx;
        for (size_t v = 0; v < N; ++v) {
            const uint8_t l = G.labels[v];
            if (!fluid(l)) continue;
            const uint32_t x = (uint32_t)(v % G.nx), y = (uint32_t)((v / G.nx) % G.ny), z = (uint32_t)(v / ((size_t)G.nx * G.ny));
            b->vox[gi].push_back((uint32_t)v);
            coord.push_back(x | (y << 11) | (z << 22));
            nlabel.push_back(l);
        }
        if ((base + 64) * 19ull >= 0xffffffffull) return bail(LBF_EINVAL, "too many fluid nodes in the batch");
    }
    b->nf = (uint32_t)base;
    b->nfp = (uint32_t)((base + 63) / 64 * 64);
    if (b->nfp == 0) b->nfp = 64;
    bool uniform = true, first = true;
    double F0[3] = {0, 0, 0};
    for (int l = 0; l < 256 && uniform; ++l) {
        if (!used[l]) continue;
        if (first) { for (int a = 0; a < 3; ++a) F0[a] = lforce[3 * l + a]; first = false; }
        else for (int a = 0; a < 3; ++a) if (lforce[3 * l + a] != F0[a]) uniform = false;
    }
    b->active.assign(count, 1);

    cudaError_t r = cudaSetDevice(device);
    if (r != cudaSuccess) return bail(LBF_ECUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(r));
#define BALLOC(p, n) do { r = cudaMalloc((void**)&(p), std::max<size_t>(1, (n))); \
        if (r != cudaSuccess) return bail(r == cudaErrorMemoryAllocation ? LBF_ENOMEM : LBF_ECUDA, std::string("cudaMalloc: ") + cudaGetErrorString(r)); } while (0)
#define BCUDA(call) do { r = (call); if (r != cudaSuccess) return bail(LBF_ECUDA, std::string(#call) + ": " + cudaGetErrorString(r)); } while (0)
    BCUDA(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
    BALLOC(b->d_geoms, count * sizeof(BatchGeom));
    BALLOC(b->d_occ, occ.size() * sizeof(uint2));
    BALLOC(b->d_coord, (size_t)b->nfp * sizeof(uint32_t));
    BALLOC(b->d_label_force, 256 * 3 * sizeof(double));
    for (int k = 0; k < 2; ++k) {
        BALLOC(b->f[k], (size_t)19 * b->nfp * b->elem);
        BCUDA(cudaMemsetAsync(b->f[k], 0, (size_t)19 * b->nfp * b->elem, b->stream));
    }
    BALLOC(b->rho, (size_t)b->nfp * sizeof(double));
    BALLOC(b->u, (size_t)3 * b->nfp * sizeof(double));
    BALLOC(b->uprev, (size_t)3 * b->nfp * sizeof(double));
    BALLOC(b->uadj, (size_t)3 * b->nfp * sizeof(double));
    BALLOC(b->err, sizeof(uint32_t));
    BALLOC(b->d_out, (size_t)count * kReduceMaxK * sizeof(double));
    BALLOC(b->d_step, 2 * sizeof(uint32_t));
    BCUDA(cudaMemsetAsync(b->d_step, 0, 2 * sizeof(uint32_t), b->stream));
    BCUDA(cudaMemsetAsync(b->rho, 0, (size_t)b->nfp * sizeof(double), b->stream));
    BCUDA(cudaMemsetAsync(b->u, 0, (size_t)3 * b->nfp * sizeof(double), b->stream));
    BCUDA(cudaMemsetAsync(b->uprev, 0, (size_t)3 * b->nfp * sizeof(double), b->stream));
    BCUDA(cudaMemsetAsync(b->uadj, 0, (size_t)3 * b->nfp * sizeof(double), b->stream));
    BCUDA(cudaMemsetAsync(b->err, 0, sizeof(uint32_t), b->stream));
    BCUDA(cudaMemcpyAsync(b->d_geoms, b->geoms.data(), count * sizeof(BatchGeom), cudaMemcpyHostToDevice, b->stream));
    BCUDA(cudaMemcpyAsync(b->d_occ, occ.data(), occ.size() * sizeof(uint2), cudaMemcpyHostToDevice, b->stream));
    BCUDA(cudaMemcpyAsync(b->d_coord, coord.data(), coord.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, b->stream));
    BCUDA(cudaMemcpyAsync(b->d_label_force, lforce.data(), lforce.size() * sizeof(double), cudaMemcpyHostToDevice, b->stream));
    if (!uniform) {
        BALLOC(b->d_label, (size_t)b->nfp);
        BCUDA(cudaMemcpyAsync(b->d_label, nlabel.data(), nlabel.size(), cudaMemcpyHostToDevice, b->stream));
    }
#undef BALLOC
#undef BCUDA
    b->force.uniform = uniform ? 1 : 0;
    b->force.fx = F0[0]; b->force.fy = F0[1]; b->force.fz = F0[2];
    b->force.label = b->d_label;
    b->force.label_force = b->d_label_force;
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    b->grid = (unsigned)sms * 8;
    if (int rc = build_tiles(b)) { std::string m = b->last_error; lbf_batch_destroy(b); return bfail(nullptr, rc, m); }
    *out = b;
    return LBF_OK;
}

void lbf_batch_destroy(lbf_batch* b)
{
    if (!b) return;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    drop_graph(b);
    void* ptrs[] = {b->d_geoms, b->d_occ, b->d_coord, b->d_label, b->d_label_force, b->f[0], b->f[1],
                    b->rho, b->u, b->uprev, b->uadj, b->err, b->d_tiles_all, b->d_tiles_active,
                    b->d_tile_first, b->d_tile_count, b->d_partial, b->d_out, b->d_step};
    for (void* p : ptrs) if (p) cudaFree(p);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
}

int lbf_batch_initialize(lbf_batch* b)
{
    if (!b) return bfail(b, LBF_EINVAL, "NULL batch");
    BCK(b, cudaSetDevice(b->device));
    Grid g{};
    g.nf = b->nf;
    g.nfp = b->nfp;
    const unsigned t = 256, n = blocks_for(b->nf, t);
    if (n) {
        if (b->storage == LBF_STORE_FP64) scsp_init<D3Q19, StoreF64><<<n, t, 0, b->stream>>>(g, b->force, b->rho0, (double*)b->f[b->cur], nullptr);
        else if (b->storage == LBF_STORE_FP16) scsp_init<D3Q19, StoreF16<D3Q19>><<<n, t, 0, b->stream>>>(g, b->force, b->rho0, (__half*)b->f[b->cur], nullptr);
        else scsp_init<D3Q19, StoreF32<D3Q19>><<<n, t, 0, b->stream>>>(g, b->force, b->rho0, (float*)b->f[b->cur], nullptr);
    }
    batch_launch(b, false, kOutMacros | kOutAdjacent, true);
    BCK(b, cudaGetLastError());
    b->initialized = true;
    return LBF_OK;
}

int lbf_batch_step(lbf_batch* b, uint32_t nsteps, uint32_t flags)
{
    if (!b) return bfail(b, LBF_EINVAL, "NULL batch");
    if (!b->initialized) return bfail(b, LBF_ESTATE, "lbf_batch_step before lbf_batch_initialize");
    BCK(b, cudaSetDevice(b->device));
    const int out = (flags & LBF_STEP_MACROS ? kOutMacros : 0) | (flags & LBF_STEP_ADJACENT ? kOutAdjacent : 0);
    uint32_t plain = nsteps ? nsteps - 1 : 0;
    // Whole graph replays (an even step count, so the buffers end where they began).
    const uint32_t G = 64;
    if (plain >= G) {
        if (b->graph && b->graph_cur != b->cur) drop_graph(b);
        if (!b->graph) { int rc = capture_graph(b, G); if (rc) return rc; }
        while (plain >= G) {
            BCK(b, cudaGraphLaunch(b->graph, b->stream));
            plain -= G;
        }
    }
    for (uint32_t s = 0; s < plain; ++s) batch_launch(b, true, 0);
    if (nsteps) batch_launch(b, true, out);
    BCK(b, cudaGetLastError());
    return LBF_OK;
}

int lbf_batch_convergence(lbf_batch* b, int first, double* out)
{
    if (!b || !out) return bfail(b, LBF_EINVAL, "NULL argument");
    BCK(b, cudaSetDevice(b->device));
    std::vector<double> r((size_t)b->count * ConvergenceFn::K, 0.0);
    if (!first) {
        ConvergenceFn fn{b->u, b->uprev, b->uadj, nullptr, nullptr, nullptr, b->nfp, 0};
        if (int rc = batch_reduce(b, fn, r.data())) return rc;
    }
    for (uint32_t g = 0; g < b->count; ++g) {
        for (int k = 0; k < 5; ++k) out[(size_t)g * 6 + k] = r[(size_t)g * 5 + k];
        out[(size_t)g * 6 + 5] = 0.0;
    }
    BCK(b, cudaMemcpyAsync(b->uprev, b->u, (size_t)3 * b->nfp * sizeof(double), cudaMemcpyDeviceToDevice, b->stream));
    BCK(b, cudaStreamSynchronize(b->stream));
    return LBF_OK;
}

int lbf_batch_flux_sums(lbf_batch* b, double* out)
{
    if (!b || !out) return bfail(b, LBF_EINVAL, "NULL argument");
    BCK(b, cudaSetDevice(b->device));
    FluxFn fn{b->u, b->rho, nullptr, b->nfp};
    return batch_reduce(b, fn, out);
}

int lbf_batch_set_active(lbf_batch* b, const uint8_t* active)
{
    if (!b || !active) return bfail(b, LBF_EINVAL, "NULL argument");
    BCK(b, cudaSetDevice(b->device));
    for (uint32_t g = 0; g < b->count; ++g) b->active[g] = active[g] ? 1 : 0;
    return build_tiles(b);
}

int lbf_batch_autotune(lbf_batch* b, uint32_t steps, double out[4])
{
    if (!b || !out) return bfail(b, LBF_EINVAL, "NULL argument");
    if (!b->initialized) return bfail(b, LBF_ESTATE, "autotune before lbf_batch_initialize");
    BCK(b, cudaSetDevice(b->device));
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device);
    if (steps < 2) steps = 2;
    steps += steps & 1;   // even: the populations end in the buffer they started in
    const unsigned threads_c[] = {128, 256};
    const unsigned tile_mult[] = {1, 2, 4};
    const unsigned per_sm[] = {4, 8, 16};
    double best = 1e300;
    unsigned bt = b->threads, btile = b->tile_nodes, bgrid = b->grid;
    // Trials advance the populations; keep a copy and put it back afterwards
    // so that tuning leaves the simulation where it was.
    const size_t fbytes = (size_t)19 * b->nfp * b->elem;
    void* snap = nullptr;
    BCK(b, cudaMalloc(&snap, fbytes + 2 * sizeof(uint32_t)));
    BCK(b, cudaMemcpyAsync(snap, b->f[b->cur], fbytes, cudaMemcpyDeviceToDevice, b->stream));
    BCK(b, cudaMemcpyAsync((char*)snap + fbytes, b->d_step, 2 * sizeof(uint32_t), cudaMemcpyDeviceToDevice, b->stream));
    const int cur0 = b->cur;
    cudaEvent_t e0, e1;
    BCK(b, cudaEventCreate(&e0));
    BCK(b, cudaEventCreate(&e1));
    for (unsigned th : threads_c)
        for (unsigned tm : tile_mult)
            for (unsigned ps : per_sm) {
                b->threads = th;
                b->tile_nodes = th * tm;
                b->grid = (unsigned)sms * ps * 128 / th;
                if (int rc = build_tiles(b)) return rc;
                batch_launch(b, true, 0);          // warm
                batch_launch(b, true, 0);
                cudaEventRecord(e0, b->stream);
                for (uint32_t s = 0; s < steps; ++s) batch_launch(b, true, 0);
                cudaEventRecord(e1, b->stream);
                BCK(b, cudaEventSynchronize(e1));
                float ms = 0;
                cudaEventElapsedTime(&ms, e0, e1);
                if (ms < best) { best = ms; bt = th; btile = th * tm; bgrid = b->grid; }
            }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    BCK(b, cudaMemcpyAsync(b->f[b->cur], snap, fbytes, cudaMemcpyDeviceToDevice, b->stream));
    BCK(b, cudaMemcpyAsync(b->d_step, (char*)snap + fbytes, 2 * sizeof(uint32_t), cudaMemcpyDeviceToDevice, b->stream));
    BCK(b, cudaStreamSynchronize(b->stream));
    cudaFree(snap);
    if (b->cur != cur0) return bfail(b, LBF_ESTATE, "autotune: buffer parity changed");
    b->threads = bt;
    b->tile_nodes = btile;
    b->grid = bgrid;
    if (int rc = build_tiles(b)) return rc;
    out[0] = bt; out[1] = btile; out[2] = (double)bgrid / sms; out[3] = best / steps;
    BCK(b, cudaGetLastError());
    return LBF_OK;
}

int lbf_batch_get_macros(lbf_batch* b, uint32_t geometry, double* rho, double* u)
{
    if (!b || geometry >= b->count) return bfail(b, LBF_EINVAL, "invalid geometry");
    BCK(b, cudaSetDevice(b->device));
    const BatchGeom& G = b->geoms[geometry];
    const size_t N = (size_t)G.nx * G.ny * G.nz;
    std::vector<double> buf((size_t)std::max<uint32_t>(1, G.nf));
    if (rho) {
        BCK(b, cudaMemcpyAsync(buf.data(), b->rho + G.node_base, G.nf * sizeof(double), cudaMemcpyDeviceToHost, b->stream));
        BCK(b, cudaStreamSynchronize(b->stream));
        std::memset(rho, 0, N * sizeof(double));
        for (uint32_t k = 0; k < G.nf; ++k) rho[b->vox[geometry][k]] = buf[k];
    }
    if (u) {
        std::memset(u, 0, 3 * N * sizeof(double));
        for (int c = 0; c < 3; ++c) {
            BCK(b, cudaMemcpyAsync(buf.data(), b->u + (size_t)c * b->nfp + G.node_base, G.nf * sizeof(double), cudaMemcpyDeviceToHost, b->stream));
            BCK(b, cudaStreamSynchronize(b->stream));
            for (uint32_t k = 0; k < G.nf; ++k) u[(size_t)c * N + b->vox[geometry][k]] = buf[k];
        }
    }
    return LBF_OK;
}

int lbf_batch_status(lbf_batch* b, uint32_t* bits)
{
    if (!b || !bits) return bfail(b, LBF_EINVAL, "NULL argument");
    BCK(b, cudaSetDevice(b->device));
    BCK(b, cudaStreamSynchronize(b->stream));
    BCK(b, cudaMemcpy(bits, b->err, sizeof(uint32_t), cudaMemcpyDeviceToHost));
    return LBF_OK;
}

int lbf_batch_synchronize(lbf_batch* b)
{
    if (!b) return bfail(b, LBF_EINVAL, "NULL batch");
    BCK(b, cudaStreamSynchronize(b->stream));
    return LBF_OK;
}

uint64_t lbf_batch_fluid_nodes(const lbf_batch* b, uint32_t geometry)
{
    if (!b) return 0;
    if (geometry == 0xffffffffu) return b->nf;
    return geometry < b->count ? b->geoms[geometry].nf : 0;
}

uint32_t lbf_batch_active_tiles(const lbf_batch* b) { return b ? b->ntiles_active : 0; }
void* lbf_batch_stream(const lbf_batch* b) { return b ? (void*)b->stream : nullptr; }
const char* lbf_batch_last_error(const lbf_batch* b) { return b ? b->last_error.c_str() : g_batch_error.c_str(); }

}  // extern "C"
