// Implicit-GEMM 3D convolutions of the learned warm start on tcgen05 tensor
// cores (BF16 operands, FP32 accumulators in tensor memory).
//
// Two kernels cover every convolution of the operator and its gradients:
//
//  igemm  out[row][n] = act(sum_k A[row][k] W[n][k] + bias)
//         A is gathered on the fly from one or two channels-last sources
//         (periodic 3x3x3 taps, 2x2x2 stride-2 cells or single voxels), W is
//         a K-major weight matrix.  Epilogues: bf16 or fp32 rows, or a
//         scatter into the 8 fine voxels of each 2x2x2 cell (transposed
//         convolution and the data gradient of the strided one).
//         Forward convolutions and data gradients (flipped, transposed
//         weights) run here.
//  wgrad  out[i][j] = sum_row A[row][i] B[row][j], both operands MN-major
//         (channels contiguous), the long reduction over rows split across
//         CTAs with fixed-order partial sums.  Weight gradients run here.
//
// Block: 160 threads, warp-specialised.  Warps 0-3 (128 producer threads)
// gather 16-byte pieces with cp.async into a 2-stage ring of
// 128-byte-swizzled operand tiles; each producer's copies of a stage arrive
// on the stage's `full` mbarrier (cp.async.mbarrier.arrive, 128 arrivals), so
// no producer waits for its own loads.  One thread of warp 4 waits for
// `full`, issues four M=128 x N x K=16 MMAs per 64-wide K stage and commits
// them to the stage's `empty` mbarrier, which the producers wait on before
// refilling the slot; its last commit arrives on `done`.  The epilogue (warps
// 0-3) reads the accumulator rows back with tcgen05.ld (warp w owns TMEM
// lanes 32w..32w+31 = tile rows).  Every wait is bounded: on timeout the
// kernel sets LBF_ERR_MMA_TIMEOUT, stops issuing and still releases its
// tensor memory.
#include "../../include/lbflow.h"
#include "../../include/lbflow_operator.h"
#include "internal.h"
#include "umma.cuh"

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <string>

namespace {

using namespace lbf::umma;

constexpr int kProducers = 128;        // warps 0-3: operand gathers, then the epilogue
constexpr int kThreads = kProducers + 32;   // + warp 4: the MMA issuer
constexpr int kBM = 128;             // tile rows = UMMA M
constexpr int kBK = 64;              // K per stage: one 128-byte swizzle row of bf16
// Two stages: with the producers decoupled from the MMA issue, the number of
// CTAs an SM holds (set by shared memory: 4 at 49 KB each) matters more than
// the ring depth (measured on the heaviest launch: 2 stages 390 TFLOP/s,
// 3 stages 348, 4 stages 282, 5 stages 177).
constexpr int kStages = 2;
constexpr uint32_t kTileA = kBM * kBK * 2;
constexpr long long kWaitCycles = 4000000000LL;   // about 2 s at the boost clock

struct Gather {
    const uint16_t* src0;
    const uint16_t* src1;
    uint32_t c0, c1, ct;
    uint32_t in_d, in_h, in_w;
    uint32_t out_d, out_h, out_w;
    uint32_t ks, stride;
    int pad;
    uint32_t taps;
    uint32_t rows;
};

struct Coord {
    int b, z, y, x;   // GEMM-row voxel
};

__device__ __forceinline__ Coord row_coord(const Gather& g, uint32_t m) {
    Coord c;
    c.x = int(m % g.out_w);
    uint32_t t = m / g.out_w;
    c.y = int(t % g.out_h);
    t /= g.out_h;
    c.z = int(t % g.out_d);
    c.b = int(t / g.out_d);
    return c;
}

__device__ __forceinline__ int wrap(int v, int n) {
    return v < 0 ? v + n : (v >= n ? v - n : v);
}

__device__ __forceinline__ void tap_offsets(const Gather& g, uint32_t tap, int& dz, int& dy, int& dx) {
    const uint32_t k2 = g.ks * g.ks;
    dz = int(tap / k2);
    const uint32_t r = tap - uint32_t(dz) * k2;
    dy = int(r / g.ks);
    dx = int(r - uint32_t(dy) * g.ks);
}

__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<const uint32_t*>(&h);
}

struct SmemRing {
    uint32_t a0, b0, b_bytes, full0, empty0, done, tmem_slot;
    __device__ uint32_t a(int s) const { return a0 + uint32_t(s) * kTileA; }
    __device__ uint32_t b(int s) const { return b0 + uint32_t(s) * b_bytes; }
    __device__ uint32_t full(int s) const { return full0 + uint32_t(s) * 8u; }
    __device__ uint32_t empty(int s) const { return empty0 + uint32_t(s) * 8u; }
};

__device__ __forceinline__ SmemRing carve(uint8_t* raw, uint32_t b_bytes) {
    SmemRing r;
    const uint32_t base = (smem_u32(raw) + 1023u) & ~1023u;
    r.a0 = base;
    r.b0 = base + kStages * kTileA;
    r.b_bytes = b_bytes;
    r.full0 = r.b0 + kStages * b_bytes;
    r.empty0 = r.full0 + kStages * 8u;
    r.done = r.empty0 + kStages * 8u;
    r.tmem_slot = r.done + 8u;
    return r;
}

constexpr size_t smem_bytes(uint32_t b_bytes) {
    return 1024 + kStages * (kTileA + b_bytes) + (2 * kStages + 1) * 8 + 16;
}

// Allocation of `cols` TMEM columns by warp 0 and the barrier set-up.
__device__ __forceinline__ uint32_t prologue(const SmemRing& r, uint32_t cols) {
    if (threadIdx.x < 32) {
        tmem_alloc(r.tmem_slot, cols);
        tmem_relinquish();
    }
    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; ++s) {
            mbar_init(r.full(s), kProducers);
            mbar_init(r.empty(s), 1);
        }
        mbar_init(r.done, 1);
        mbar_init_fence();
    }
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    uint32_t t;
    asm volatile("ld.shared.b32 %0, [%1];" : "=r"(t) : "r"(r.tmem_slot) : "memory");
    return t;
}

__device__ __forceinline__ void release(uint32_t tmem, uint32_t cols) {
    fence_before_sync();
    __syncthreads();
    if (threadIdx.x < 32) tmem_dealloc(tmem, cols);
}

// The shared producer / MMA pipeline.  Loader provides (producer threads)
//   load(chunk, stage)   cp.async the chunk's A and B tiles into the stage
//   adesc/bdesc(stage, kk)  descriptors of the kk-th K=16 slice
// Returns, in the producer threads, whether the accumulator is complete
// (every wait succeeded and `done` fired); false elsewhere or on a timeout.
template <class Loader>
__device__ bool mainloop(Loader& ld, const SmemRing& r, uint32_t nch, uint32_t tmem, uint32_t idesc) {
    const uint32_t warp = threadIdx.x >> 5;
    if (warp < uint32_t(kProducers / 32)) {
        bool ok = true;
        for (uint32_t c = 0; c < nch; ++c) {
            const int s = int(c % kStages);
            if (c >= uint32_t(kStages)) {
                // The slot's previous chunk must have been consumed by its MMAs.
                const bool w = mbar_wait(r.empty(s), ((c / kStages) - 1u) & 1u, kWaitCycles);
                ok = __all_sync(0xffffffffu, w);      // the warp leaves together (loads shuffle)
                if (!ok) break;
            }
            ld.load(c, s);
            cp_async_arrive(r.full(s));
        }
        cp_async_commit();          // wait_group only waits for committed copies
        cp_async_wait<0>();
        const bool d = mbar_wait(r.done, 0u, kWaitCycles);
        fence_after_sync();
        return ok && d;
    }
    if (threadIdx.x == uint32_t(kProducers)) {
        bool ok = true;
        for (uint32_t c = 0; c < nch; ++c) {
            const int s = int(c % kStages);
            ok = mbar_wait(r.full(s), (c / kStages) & 1u, kWaitCycles);
            if (!ok) break;
            // The producers' cp.async writes, made visible to the tensor
            // core's (async-proxy) reads of the stage.
            fence_async_shared();
            fence_after_sync();
#pragma unroll
            for (int kk = 0; kk < kBK / 16; ++kk)
                mma_bf16(tmem, ld.adesc(s, kk), ld.bdesc(s, kk), idesc, (c | uint32_t(kk)) != 0u);
            commit(r.empty(s));
        }
        // `done` fires once every MMA issued above has completed (at once
        // when none was issued), also after a timeout, so the tensor memory
        // is never released under a running MMA.
        commit(r.done);
    }
    return false;
}

// ---------------------------------------------------------------- igemm ----

struct IgemmArgs {
    Gather g;
    const uint16_t* w;
    uint32_t n, k_pad;
    const float* bias;
    void* out;
    uint32_t mode, ld;
    uint32_t act;
    float slope;
    uint32_t* err;
};

// Voxel index of tap (dz, dy, dx) of row voxel c, and the address of channels
// [ch, ch + 8) of that voxel in whichever source holds them.
__device__ __forceinline__ size_t gather_vox(const Gather& g, const Coord& c, int dz, int dy, int dx) {
    const int z = wrap(int(g.stride) * c.z + dz - g.pad, int(g.in_d));
    const int y = wrap(int(g.stride) * c.y + dy - g.pad, int(g.in_h));
    const int x = wrap(int(g.stride) * c.x + dx - g.pad, int(g.in_w));
    return ((size_t(c.b) * g.in_d + z) * g.in_h + y) * g.in_w + x;
}
__device__ __forceinline__ const uint16_t* chan_ptr(const Gather& g, size_t vox, uint32_t ch) {
    return ch < g.c0 ? g.src0 + vox * g.c0 + ch : g.src1 + vox * g.c1 + (ch - g.c0);
}

// A tile: thread t owns tile row t and copies its 8 16-byte pieces of each
// 64-wide K stage.  When a stage lies inside one tap of one source (channel
// counts multiples of 64) the row's 128 bytes are contiguous in memory: one
// address per stage.  Otherwise the tap and channel advance piece by piece.
template <int BN>
struct IgemmLoader {
    const IgemmArgs& p;
    SmemRing r;
    Coord rc;
    bool rv;
    bool uniform;
    uint32_t n0;
    uint32_t sw;          // swizzle of the thread's row (row mod 8)
    uint32_t poff_b;      // swizzled byte offset of the thread's B piece
    // Uniform path: the K position of the next chunk (chunks come in order)
    // as tap (dz, dy, dx) and channel, advanced incrementally instead of by
    // divisions, and the row's unwrapped source origin stride * voxel - pad.
    uint32_t u_tap, u_ch;
    int u_dz, u_dy, u_dx;
    int oz, oy, ox;

    __device__ IgemmLoader(const IgemmArgs& a, const SmemRing& ring, uint32_t m0, uint32_t n0_)
        : p(a), r(ring), n0(n0_) {
        const uint32_t t = threadIdx.x;
        const uint32_t m = m0 + t;
        rv = m < p.g.rows;
        rc = row_coord(p.g, rv ? m : 0u);
        sw = t & 7u;
        poff_b = (((t & 7u) ^ ((t >> 3) & 7u)) << 4);
        uniform = (p.g.ct % kBK == 0) && (p.g.c1 == 0 || p.g.c0 % kBK == 0);
        u_tap = 0; u_ch = 0;
        u_dz = u_dy = u_dx = 0;
        oz = int(p.g.stride) * rc.z - p.g.pad;
        oy = int(p.g.stride) * rc.y - p.g.pad;
        ox = int(p.g.stride) * rc.x - p.g.pad;
    }

    __device__ void load(uint32_t chunk, int s) {
        const uint32_t t = threadIdx.x;
        const uint32_t a = r.a(s) + t * 128u;
        if (uniform) {
            // Each thread finds its row's 128 contiguous bytes; the copies are
            // then spread so that lanes 8q..8q+7 move the 8 pieces of one row
            // (coalesced), the row addresses passed by warp shuffles (a null
            // address marks a row past the end or a K position past the taps).
            const bool v = rv && u_tap < p.g.taps;
            const uint16_t* src = nullptr;
            if (v) {
                const int z = wrap(oz + u_dz, int(p.g.in_d));
                const int y = wrap(oy + u_dy, int(p.g.in_h));
                const int x = wrap(ox + u_dx, int(p.g.in_w));
                const size_t vox = ((size_t(rc.b) * p.g.in_d + z) * p.g.in_h + y) * p.g.in_w + x;
                src = chan_ptr(p.g, vox, u_ch);
            }
            // Next chunk: 64 channels further, carrying into the next tap.
            u_ch += kBK;
            if (u_ch >= p.g.ct) {
                u_ch = 0;
                ++u_tap;
                if (++u_dx == int(p.g.ks)) {
                    u_dx = 0;
                    if (++u_dy == int(p.g.ks)) { u_dy = 0; ++u_dz; }
                }
            }
            const uint32_t lane = t & 31u, wbase = t & ~31u, j = lane & 7u;
            const unsigned long long sp = reinterpret_cast<unsigned long long>(src);
#pragma unroll
            for (uint32_t i = 0; i < 8; ++i) {
                const uint32_t rw = 4u * i + (lane >> 3);              // row within the warp
                const unsigned long long q = __shfl_sync(0xffffffffu, sp, int(rw));
                const uint32_t row = wbase + rw;
                const uint32_t dst = r.a(s) + row * 128u + ((j ^ (row & 7u)) << 4);
                cp_async16(dst, q ? reinterpret_cast<const uint16_t*>(q) + 8u * j : p.g.src0, q ? 16u : 0u);
            }
        } else {
            uint32_t k = chunk * kBK;
            uint32_t tap = k / p.g.ct;
            uint32_t ch = k - tap * p.g.ct;
            uint32_t cur = 0xffffffffu;
            size_t vox = 0;
#pragma unroll
            for (uint32_t j = 0; j < 8; ++j) {
                const bool v = rv && tap < p.g.taps;
                if (v && tap != cur) {
                    int dz, dy, dx;
                    tap_offsets(p.g, tap, dz, dy, dx);
                    vox = gather_vox(p.g, rc, dz, dy, dx);
                    cur = tap;
                }
                cp_async16(a + ((j ^ sw) << 4), v ? chan_ptr(p.g, vox, ch) : p.g.src0, v ? 16u : 0u);
                ch += 8u;
                if (ch >= p.g.ct) { ch = 0; ++tap; }
            }
        }
        const uint32_t kb = chunk * kBK + (t & 7u) * 8u;
        const uint32_t b = r.b(s) + (t >> 3) * 128u + poff_b;
#pragma unroll
        for (int i = 0; i < BN / 16; ++i) {
            const uint32_t n = (t >> 3) + 16u * i;
            cp_async16(b + uint32_t(i) * 16u * 128u, p.w + size_t(n0 + n) * p.k_pad + kb, 16u);
        }
    }
    __device__ uint64_t adesc(int s, int kk) const { return desc_sw128(r.a(s) + 32u * kk, 16u, 1024u); }
    __device__ uint64_t bdesc(int s, int kk) const { return desc_sw128(r.b(s) + 32u * kk, 16u, 1024u); }
};

template <int BN>
__global__ void __launch_bounds__(kThreads, 1) igemm_kernel(const __grid_constant__ IgemmArgs p) {
    extern __shared__ uint8_t smem_raw[];
    constexpr uint32_t kCols = BN < 32 ? 32 : BN;
    const SmemRing r = carve(smem_raw, BN * 128u);
    const uint32_t tmem = prologue(r, kCols);
    const uint32_t m0 = blockIdx.x * kBM, n0 = blockIdx.y * BN;

    IgemmLoader<BN> ld(p, r, m0, n0);
    const bool ok = mainloop(ld, r, p.k_pad / kBK, tmem, idesc_bf16(kBM, BN, false, false));
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (warp >= uint32_t(kProducers / 32)) {
        release(tmem, kCols);
        return;
    }
    if (!ok && threadIdx.x == 0) atomicOr(p.err, LBF_ERR_MMA_TIMEOUT);

    const uint32_t row = m0 + warp * 32 + lane;
    const bool rvalid = ok && row < p.g.rows;
    Coord rc = row_coord(p.g, rvalid ? row : 0u);
#pragma unroll 1
    for (int col0 = 0; col0 < BN; col0 += 16) {
        float v[16];
        tmem_ld16(tmem + ((warp * 32u) << 16) + uint32_t(col0), v);
        if (!rvalid) continue;
        const uint32_t nb = n0 + col0;
#pragma unroll
        for (int e = 0; e < 16; ++e) {
            const uint32_t n = nb + e;
            float x = v[e];
            if (p.bias && n < p.n) x += p.bias[p.mode == LBF_OUT_SCATTER2_BF16 ? n % p.ld : n];
            if (p.act) x = x > 0.f ? x : x * p.slope;
            v[e] = x;
        }
        if (p.mode == LBF_OUT_F32) {
            float* o = static_cast<float*>(p.out) + size_t(row) * p.ld;
            for (int e = 0; e < 16; ++e)
                if (nb + e < p.n) o[nb + e] = v[e];
            continue;
        }
        uint16_t* o;
        uint32_t c;
        bool vec;
        if (p.mode == LBF_OUT_BF16) {
            o = static_cast<uint16_t*>(p.out) + size_t(row) * p.ld;
            c = nb;
            vec = (p.ld % 8u == 0u) && nb + 16 <= p.n;
        } else {
            // Scatter: n = tap * ld + c into fine voxel 2 * row + tap.
            const uint32_t tap = nb / p.ld;
            c = nb - tap * p.ld;
            const int dz = int(tap >> 2), dy = int((tap >> 1) & 1u), dx = int(tap & 1u);
            const size_t fd = 2u * p.g.out_d, fh = 2u * p.g.out_h, fw = 2u * p.g.out_w;
            const size_t vox = ((size_t(rc.b) * fd + 2 * rc.z + dz) * fh + 2 * rc.y + dy) * fw + 2 * rc.x + dx;
            o = static_cast<uint16_t*>(p.out) + vox * p.ld;
            vec = (p.ld % 16u == 0u) && nb + 16 <= p.n;
            if (!vec) {
                for (int e = 0; e < 16; ++e) {
                    const uint32_t n = nb + e;
                    if (n >= p.n) break;
                    const uint32_t tp = n / p.ld, cc = n - tp * p.ld;
                    const int ez = int(tp >> 2), ey = int((tp >> 1) & 1u), ex = int(tp & 1u);
                    const size_t vx = ((size_t(rc.b) * fd + 2 * rc.z + ez) * fh + 2 * rc.y + ey) * fw +
                                      2 * rc.x + ex;
                    __nv_bfloat16 h = __float2bfloat16_rn(v[e]);
                    static_cast<uint16_t*>(p.out)[vx * p.ld + cc] = *reinterpret_cast<uint16_t*>(&h);
                }
                continue;
            }
        }
        if (vec) {
            uint4 q0, q1;
            q0.x = pack_bf16(v[0], v[1]);   q0.y = pack_bf16(v[2], v[3]);
            q0.z = pack_bf16(v[4], v[5]);   q0.w = pack_bf16(v[6], v[7]);
            q1.x = pack_bf16(v[8], v[9]);   q1.y = pack_bf16(v[10], v[11]);
            q1.z = pack_bf16(v[12], v[13]); q1.w = pack_bf16(v[14], v[15]);
            reinterpret_cast<uint4*>(o + c)[0] = q0;
            reinterpret_cast<uint4*>(o + c)[1] = q1;
        } else {
            for (int e = 0; e < 16; ++e) {
                if (nb + e >= p.n) break;
                __nv_bfloat16 h = __float2bfloat16_rn(v[e]);
                o[c + e] = *reinterpret_cast<uint16_t*>(&h);
            }
        }
    }
    release(tmem, kCols);
}

// ---------------------------------------------------------------- wgrad ----

struct WgradArgs {
    Gather g;
    const uint16_t* b;
    uint32_t cb;
    uint32_t mtot;          // taps * ct
    uint32_t cps;           // K chunks per split
    uint32_t nch;           // total K chunks = ceil(rows / 64)
    float* partial;         // [split][mtot][cb]
    uint32_t* err;
};

// Mixed-radix (x, y, z, b) advance of a row index by 64.
struct Step64 {
    int ax, ay, az, ab;
};

template <int BN>
struct WgradLoader {
    const WgradArgs& p;
    SmemRing r;
    Step64 st;
    Coord rc;             // voxel of this thread's K row of the current chunk
    uint32_t base;        // first row of the current chunk
    uint32_t m_end;
    uint32_t kr, half;    // K row (t >> 1) and which 8 of its 16 pieces (t & 1)
    uint32_t tap0, ch0;   // tap and channel of the thread's first piece
    bool uniform;         // its 8 pieces are 64 contiguous channels of one tap and source
    uint32_t aoff;        // byte offset of the thread's first A piece inside a stage
    uint32_t j0;

    __device__ WgradLoader(const WgradArgs& a, const SmemRing& ring, uint32_t i0, uint32_t j0_, uint32_t c_begin,
                           uint32_t m_end_, const Step64& s64)
        : p(a), r(ring), st(s64), m_end(m_end_), j0(j0_) {
        const uint32_t t = threadIdx.x;
        kr = t >> 1;
        half = t & 1u;
        const uint32_t i = i0 + half * 64u;
        tap0 = i / p.g.ct;
        ch0 = i - tap0 * p.g.ct;
        uniform = (p.g.ct % kBK == 0) && (p.g.c1 == 0 || p.g.c0 % kBK == 0);
        aoff = half * 1024u + (kr >> 3) * 2048u + (kr & 7u) * 128u;
        base = c_begin * kBK;
        const uint32_t m = base + kr;
        rc = row_coord(p.g, m < m_end ? m : 0u);
    }

    __device__ void advance() {
        base += kBK;
        rc.x += st.ax;
        int carry = rc.x >= int(p.g.out_w);
        if (carry) rc.x -= int(p.g.out_w);
        rc.y += st.ay + carry;
        carry = rc.y >= int(p.g.out_h);
        if (carry) rc.y -= int(p.g.out_h);
        rc.z += st.az + carry;
        carry = rc.z >= int(p.g.out_d);
        if (carry) rc.z -= int(p.g.out_d);
        rc.b += st.ab + carry;
    }

    __device__ void load(uint32_t /*chunk*/, int s) {
        const uint32_t t = threadIdx.x;
        const uint32_t a = r.a(s) + aoff;
        const uint32_t sw = kr & 7u;
        const bool rowv = base + kr < m_end;
        if (uniform) {
            // Thread (kr, half) finds 128 contiguous bytes of its K row; the
            // copies are spread so that lanes 16q..16q+15 move the 16 pieces of
            // one K row (256 contiguous bytes), addresses passed by shuffles.
            const bool v = rowv && tap0 < p.g.taps;
            const uint16_t* src = p.g.src0;
            if (v) {
                int dz, dy, dx;
                tap_offsets(p.g, tap0, dz, dy, dx);
                src = chan_ptr(p.g, gather_vox(p.g, rc, dz, dy, dx), ch0);
            }
            const uint32_t lane = t & 31u, pc = lane & 15u;
            const unsigned long long sp = reinterpret_cast<unsigned long long>(src);
#pragma unroll
            for (uint32_t i = 0; i < 8; ++i) {
                const uint32_t rw = 2u * i + (lane >> 4);              // K row within the warp's 16
                const int from = int(2u * rw + (pc >> 3));             // the thread holding that half
                const unsigned long long q = __shfl_sync(0xffffffffu, sp, from);
                const int vq = __shfl_sync(0xffffffffu, int(v), from);
                const uint32_t k = (t >> 5) * 16u + rw;                // K row within the chunk
                const uint32_t dst = r.a(s) + (pc >> 3) * 1024u + (k >> 3) * 2048u + (k & 7u) * 128u +
                                     (((pc & 7u) ^ (k & 7u)) << 4);
                cp_async16(dst, vq ? reinterpret_cast<const uint16_t*>(q) + 8u * (pc & 7u) : p.g.src0,
                           vq ? 16u : 0u);
            }
        } else {
            uint32_t tap = tap0, ch = ch0, cur = 0xffffffffu;
            size_t vox = 0;
#pragma unroll
            for (uint32_t jj = 0; jj < 8; ++jj) {
                const bool v = rowv && tap < p.g.taps;
                if (v && tap != cur) {
                    int dz, dy, dx;
                    tap_offsets(p.g, tap, dz, dy, dx);
                    vox = gather_vox(p.g, rc, dz, dy, dx);
                    cur = tap;
                }
                cp_async16(a + ((jj ^ sw) << 4), v ? chan_ptr(p.g, vox, ch) : p.g.src0, v ? 16u : 0u);
                ch += 8u;
                if (ch >= p.g.ct) { ch = 0; ++tap; }
            }
        }
        // B: BN/8 pieces per K row.
        constexpr uint32_t kPieces = BN / 8;
        constexpr uint32_t kRowsPerPass = kProducers / kPieces;
        constexpr uint32_t kSbo = (BN / 64) * 1024u;
        const uint32_t qn = t % kPieces;
        const uint32_t jn = j0 + qn * 8u;
#pragma unroll
        for (uint32_t it = 0; it < kBK / kRowsPerPass; ++it) {
            const uint32_t k = t / kPieces + kRowsPerPass * it;
            const uint32_t row = base + k;
            const bool v = row < m_end && jn < p.cb;
            const uint16_t* src = v ? p.b + size_t(row) * p.cb + jn : p.b;
            const uint32_t dst = r.b(s) + (qn >> 3) * 1024u + (k >> 3) * kSbo + (k & 7u) * 128u +
                                 (((qn & 7u) ^ (k & 7u)) << 4);
            cp_async16(dst, src, v ? 16u : 0u);
        }
        advance();
    }
    __device__ uint64_t adesc(int s, int kk) const { return desc_sw128(r.a(s) + 4096u * kk, 1024u, 2048u); }
    __device__ uint64_t bdesc(int s, int kk) const {
        constexpr uint32_t kSbo = (BN / 64) * 1024u;
        return desc_sw128(r.b(s) + 2u * kSbo * kk, 1024u, kSbo);
    }
};

template <int BN>
__global__ void __launch_bounds__(kThreads, 1) wgrad_kernel(const __grid_constant__ WgradArgs p, const Step64 st) {
    extern __shared__ uint8_t smem_raw[];
    const SmemRing r = carve(smem_raw, BN * 128u);
    const uint32_t tmem = prologue(r, BN);
    const uint32_t i0 = blockIdx.x * kBM, j0 = blockIdx.y * BN;
    const uint32_t c_begin = blockIdx.z * p.cps;
    const uint32_t c_end = min(p.nch, c_begin + p.cps);
    const uint32_t m_end = min(p.g.rows, c_end * kBK);

    WgradLoader<BN> ld(p, r, i0, j0, c_begin, m_end, st);
    const uint32_t nch = c_end > c_begin ? c_end - c_begin : 0u;
    const bool ok = mainloop(ld, r, nch, tmem, idesc_bf16(kBM, BN, true, true));
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (warp >= uint32_t(kProducers / 32)) {
        release(tmem, BN);
        return;
    }
    if (!ok && nch > 0 && threadIdx.x == 0) atomicOr(p.err, LBF_ERR_MMA_TIMEOUT);

    const uint32_t i = i0 + warp * 32 + lane;
    float* out = p.partial + (size_t(blockIdx.z) * p.mtot + i) * p.cb;
#pragma unroll 1
    for (int col0 = 0; col0 < BN; col0 += 16) {
        float v[16];
        tmem_ld16(tmem + ((warp * 32u) << 16) + uint32_t(col0), v);
        if (i >= p.mtot) continue;
        for (int e = 0; e < 16; ++e) {
            const uint32_t j = j0 + col0 + e;
            if (j < p.cb) out[j] = ok ? v[e] : 0.f;
        }
    }
    release(tmem, BN);
}

__global__ void sum_partials(const float* __restrict__ part, float* __restrict__ out, size_t n, uint32_t splits) {
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
        float s = 0.f;
        for (uint32_t k = 0; k < splits; ++k) s += part[k * n + i];
        out[i] = s;
    }
}

// ----------------------------------------------------------------- host ----

int fail(const std::string& msg, int code = LBF_EINVAL) {
    lbf::set_global_error(msg);
    return code;
}

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

// Validates the gather and fills the device form.  Every source voxel index
// stays inside the source grid: stride*row + tap - pad must lie in
// [-in, 2*in) on each axis so that one periodic wrap brings it back.
int make_gather(const lbf_gather& a, Gather& g, const char* who) {
    const std::string w(who);
    if (!a.src0 || (a.c1 && !a.src1)) return fail(w + ": null source");
    if (a.c0 == 0 || a.c0 % 8 || a.c1 % 8) return fail(w + ": gathered channel counts must be positive multiples of 8");
    if (!aligned16(a.src0) || (a.src1 && !aligned16(a.src1))) return fail(w + ": sources must be 16-byte aligned");
    if (a.ksize < 1 || a.ksize > 3 || a.stride < 1 || a.stride > 2) return fail(w + ": ksize must be 1..3, stride 1..2");
    if (!a.batch || !a.in_d || !a.in_h || !a.in_w || !a.out_d || !a.out_h || !a.out_w)
        return fail(w + ": empty grid");
    const uint32_t in[3] = {a.in_d, a.in_h, a.in_w}, out[3] = {a.out_d, a.out_h, a.out_w};
    for (int d = 0; d < 3; ++d) {
        const long long lo = -(long long)a.pad;
        const long long hi = (long long)a.stride * (out[d] - 1) + a.ksize - 1 - a.pad;
        if (lo < -(long long)in[d] || hi >= 2LL * in[d])
            return fail(w + ": gather reaches beyond one periodic image of the source");
    }
    const unsigned long long rows = (unsigned long long)a.batch * a.out_d * a.out_h * a.out_w;
    const unsigned long long vin = (unsigned long long)a.batch * a.in_d * a.in_h * a.in_w;
    if (rows >= (1ull << 31) || vin * (a.c0 + a.c1) >= (1ull << 40)) return fail(w + ": grid too large");
    g.src0 = static_cast<const uint16_t*>(a.src0);
    g.src1 = static_cast<const uint16_t*>(a.src1);
    g.c0 = a.c0;
    g.c1 = a.c1;
    g.ct = a.c0 + a.c1;
    g.in_d = a.in_d; g.in_h = a.in_h; g.in_w = a.in_w;
    g.out_d = a.out_d; g.out_h = a.out_h; g.out_w = a.out_w;
    g.ks = a.ksize;
    g.stride = a.stride;
    g.pad = a.pad;
    g.taps = a.ksize * a.ksize * a.ksize;
    g.rows = uint32_t(rows);
    return LBF_OK;
}

template <int BN>
int launch_igemm(const IgemmArgs& p, uint32_t n_pad, cudaStream_t s) {
    const size_t sm = smem_bytes(BN * 128u);
    cudaError_t e = cudaFuncSetAttribute(igemm_kernel<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm));
    if (e != cudaSuccess) return fail(std::string("lbf_igemm_run: ") + cudaGetErrorString(e), LBF_ECUDA);
    dim3 grid((p.g.rows + kBM - 1) / kBM, n_pad / BN);
    igemm_kernel<BN><<<grid, kThreads, sm, s>>>(p);
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail(std::string("lbf_igemm_run: ") + cudaGetErrorString(e), LBF_ECUDA);
    return LBF_OK;
}

struct WgradPlan {
    uint32_t bn, tiles_m, tiles_n, nch, cps, splits;
    size_t bytes;
};

WgradPlan plan_wgrad(const Gather& g, uint32_t cb) {
    WgradPlan pl{};
    pl.bn = cb <= 64 ? 64 : 128;
    const uint32_t mtot = g.taps * g.ct;
    pl.tiles_m = (mtot + kBM - 1) / kBM;
    pl.tiles_n = (cb + pl.bn - 1) / pl.bn;
    pl.nch = (g.rows + kBK - 1) / kBK;
    const uint32_t tiles = pl.tiles_m * pl.tiles_n;
    // About two waves of 148 SMs, at least 8 K stages per split.
    uint32_t want = (2u * 148u + tiles - 1) / tiles;
    want = std::max(1u, std::min(want, (pl.nch + 7) / 8));
    pl.cps = (pl.nch + want - 1) / want;
    pl.splits = (pl.nch + pl.cps - 1) / pl.cps;
    pl.bytes = size_t(pl.splits) * mtot * cb * sizeof(float);
    return pl;
}

}  // namespace

extern "C" {

int lbf_igemm_run(const lbf_igemm* d, void* stream) {
    if (!d) return fail("lbf_igemm_run: null descriptor");
    IgemmArgs p{};
    int rc = make_gather(d->a, p.g, "lbf_igemm_run");
    if (rc) return rc;
    const uint32_t np = d->n_pad;
    if (!(np == 16 || np == 32 || np == 64 || (np % 128 == 0 && np > 0)))
        return fail("lbf_igemm_run: n_pad must be 16, 32, 64 or a multiple of 128");
    if (d->n == 0 || d->n > np) return fail("lbf_igemm_run: n must be in 1..n_pad");
    if (d->k_pad == 0 || d->k_pad % kBK || d->k_pad < p.g.taps * p.g.ct)
        return fail("lbf_igemm_run: k_pad must be a multiple of 64 covering ksize^3 * channels");
    if (!d->weight || !aligned16(d->weight) || !d->out || !d->err) return fail("lbf_igemm_run: null or misaligned pointer");
    if (d->out_mode > LBF_OUT_SCATTER2_BF16 || d->out_ld == 0) return fail("lbf_igemm_run: bad output mode");
    if (d->out_mode == LBF_OUT_SCATTER2_BF16 && d->n > 8u * d->out_ld)
        return fail("lbf_igemm_run: scatter output needs n <= 8 * out_ld");
    if (d->out_mode != LBF_OUT_SCATTER2_BF16 && d->n > d->out_ld) return fail("lbf_igemm_run: n exceeds out_ld");
    if (d->out_mode != LBF_OUT_F32 && !aligned16(d->out)) return fail("lbf_igemm_run: out must be 16-byte aligned");
    p.w = static_cast<const uint16_t*>(d->weight);
    p.n = d->n;
    p.k_pad = d->k_pad;
    p.bias = d->bias;
    p.out = d->out;
    p.mode = d->out_mode;
    p.ld = d->out_ld;
    p.act = d->act;
    p.slope = d->slope;
    p.err = d->err;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    switch (np) {
        case 16: return launch_igemm<16>(p, np, s);
        case 32: return launch_igemm<32>(p, np, s);
        case 64: return launch_igemm<64>(p, np, s);
        default: return launch_igemm<128>(p, np, s);
    }
}

size_t lbf_wgrad_workspace(const lbf_wgrad* w) {
    if (!w) return 0;
    Gather g{};
    if (make_gather(w->a, g, "lbf_wgrad_workspace")) return 0;
    return plan_wgrad(g, w->cb).bytes;
}

int lbf_wgrad_run(const lbf_wgrad* w, void* stream) {
    if (!w) return fail("lbf_wgrad_run: null descriptor");
    WgradArgs p{};
    int rc = make_gather(w->a, p.g, "lbf_wgrad_run");
    if (rc) return rc;
    if (!w->b || !aligned16(w->b) || w->cb == 0 || w->cb % 8 || !w->out || !w->err)
        return fail("lbf_wgrad_run: b must be 16-byte aligned with cb a positive multiple of 8; out and err non-null");
    const WgradPlan pl = plan_wgrad(p.g, w->cb);
    if (!w->workspace || w->workspace_bytes < pl.bytes)
        return fail("lbf_wgrad_run: workspace smaller than lbf_wgrad_workspace()");
    p.b = static_cast<const uint16_t*>(w->b);
    p.cb = w->cb;
    p.mtot = p.g.taps * p.g.ct;
    p.cps = pl.cps;
    p.nch = pl.nch;
    p.partial = static_cast<float*>(w->workspace);
    p.err = w->err;
    Step64 st;
    uint32_t q = kBK;
    st.ax = int(q % p.g.out_w); q /= p.g.out_w;
    st.ay = int(q % p.g.out_h); q /= p.g.out_h;
    st.az = int(q % p.g.out_d); q /= p.g.out_d;
    st.ab = int(q);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    dim3 grid(pl.tiles_m, pl.tiles_n, pl.splits);
    cudaError_t e;
    if (pl.bn == 64) {
        const size_t sm = smem_bytes(64 * 128u);
        e = cudaFuncSetAttribute(wgrad_kernel<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm));
        if (e == cudaSuccess) wgrad_kernel<64><<<grid, kThreads, sm, s>>>(p, st);
    } else {
        const size_t sm = smem_bytes(128 * 128u);
        e = cudaFuncSetAttribute(wgrad_kernel<128>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm));
        if (e == cudaSuccess) wgrad_kernel<128><<<grid, kThreads, sm, s>>>(p, st);
    }
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e == cudaSuccess) {
        const size_t n = size_t(p.mtot) * p.cb;
        const unsigned blocks = unsigned(std::min<size_t>((n + 255) / 256, 148u * 8u));
        sum_partials<<<blocks, 256, 0, s>>>(p.partial, w->out, n, pl.splits);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) return fail(std::string("lbf_wgrad_run: ") + cudaGetErrorString(e), LBF_ECUDA);
    return LBF_OK;
}

void lbf_operator_info(uint32_t out[4]) {
    out[0] = kBM;
    out[1] = kBK;
    out[2] = kStages;
    out[3] = kThreads;
}

}  // extern "C"
