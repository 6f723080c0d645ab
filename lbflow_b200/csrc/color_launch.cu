// Template instantiation and dispatch of the two-phase kernels.
#include "internal.h"
#include "../../include/lbflow.h"

namespace lbf {

namespace {
template <class L, class S, int COLL, bool FILM>
void run_step(bool pull, int out, const ColorLaunch& a)
{
    using T = typename S::T;
    const T* fin = static_cast<const T*>(a.fin);
    T* fout = static_cast<T*>(a.fout);
    const unsigned threads = 128, blocks = blocks_for(a.g.nf, threads);
    if (blocks == 0) return;
    const unsigned zb = blocks_for(a.zh.n, threads);
    const double rb = a.P.rho_ref[0];
    if (pull)
        color_phase<L, S, true, FILM><<<blocks, threads, 0, a.stream>>>(a.g, a.film, fin, a.dens, a.phid, a.err, rb);
    else
        color_phase<L, S, false, false><<<blocks, threads, 0, a.stream>>>(a.g, a.film, fin, a.dens, a.phid, a.err, rb);
    // Zou-He boundary nodes (PB/VB): their phase from the rebuilt populations
    // before pass 2 reads it, and their collision after pass 2 (overwriting).
    if (pull && zb)
        color_zou_he_phase<L, S, FILM><<<zb, threads, 0, a.stream>>>(a.g, a.film, a.zh, fin, a.phid, a.err, rb);
    if (!pull && zb && (out & kOutAdjacent))
        color_zou_he_record<L, S><<<zb, threads, 0, a.stream>>>(a.g, a.zh, fin, rb);
    if (pull)
        color_collide<L, S, COLL, true, FILM><<<blocks, threads, 0, a.stream>>>(
            a.g, a.film, a.F, a.P, a.W, fin, fout, a.dens, a.phid, a.mo, out, a.err);
    else
        color_collide<L, S, COLL, false, false><<<blocks, threads, 0, a.stream>>>(
            a.g, a.film, a.F, a.P, a.W, fin, fout, a.dens, a.phid, a.mo, out, a.err);
    if (pull && zb)
        color_zou_he_collide<L, S, COLL, FILM><<<zb, threads, 0, a.stream>>>(a.g, a.film, a.F, a.P, a.W, a.zh, fin,
                                                                            fout, a.phid, a.mo, out, a.err);
}

template <class L, class S, int COLL>
void dispatch(bool pull, int out, const ColorLaunch& a)
{
    // Half films: the film-aware gathers only where the geometry has films
    // (FP64 and FP32 storage; the engine refuses films with 16-bit storage).
    if constexpr (IsPacked<S>::value) run_step<L, S, COLL, false>(pull, out, a);
    else if (a.film.bits[0]) run_step<L, S, COLL, true>(pull, out, a);
    else run_step<L, S, COLL, false>(pull, out, a);
}

template <class L, class S>
void dispatch_coll(int collision, bool pull, int out, const ColorLaunch& a)
{
    if (collision == LBF_MRT) dispatch<L, S, 1>(pull, out, a);
    else dispatch<L, S, 0>(pull, out, a);
}
}  // namespace

void launch_color(int dims, int storage, int collision, bool pull, int out, const ColorLaunch& a)
{
    // The two-phase path stores full populations (FP64, or FP32 at reduced
    // precision), or the total and the component-0 share in 16 bits each.
    if (dims == 3) {
        if (storage == LBF_STORE_FP64) dispatch_coll<D3Q19, StoreF64>(collision, pull, out, a);
        else if (storage == LBF_STORE_FP16) dispatch_coll<D3Q19, ColorPacked<D3Q19, __half>>(collision, pull, out, a);
        else if (storage == LBF_STORE_BF16)
            dispatch_coll<D3Q19, ColorPacked<D3Q19, __nv_bfloat16>>(collision, pull, out, a);
        else dispatch_coll<D3Q19, StoreF32Full>(collision, pull, out, a);
    } else {
        if (storage == LBF_STORE_FP64) dispatch_coll<D2Q9, StoreF64>(collision, pull, out, a);
        else if (storage == LBF_STORE_FP16) dispatch_coll<D2Q9, ColorPacked<D2Q9, __half>>(collision, pull, out, a);
        else if (storage == LBF_STORE_BF16)
            dispatch_coll<D2Q9, ColorPacked<D2Q9, __nv_bfloat16>>(collision, pull, out, a);
        else dispatch_coll<D2Q9, StoreF32Full>(collision, pull, out, a);
    }
}

void launch_color_init(int dims, int storage, const Grid& g, const Force& F, const ColorParams& P,
                       const uint8_t* phase, void* f, cudaStream_t s)
{
    const unsigned threads = 256, blocks = blocks_for(g.nf, threads);
    if (blocks == 0) return;
    uint16_t* h = static_cast<uint16_t*>(f);
    if (dims == 3) {
        if (storage == LBF_STORE_FP64) color_init<D3Q19, StoreF64><<<blocks, threads, 0, s>>>(g, F, P, phase, (double*)f);
        else if (storage == LBF_STORE_FP16)
            color_init<D3Q19, ColorPacked<D3Q19, __half>><<<blocks, threads, 0, s>>>(g, F, P, phase, h);
        else if (storage == LBF_STORE_BF16)
            color_init<D3Q19, ColorPacked<D3Q19, __nv_bfloat16>><<<blocks, threads, 0, s>>>(g, F, P, phase, h);
        else color_init<D3Q19, StoreF32Full><<<blocks, threads, 0, s>>>(g, F, P, phase, (float*)f);
    } else {
        if (storage == LBF_STORE_FP64) color_init<D2Q9, StoreF64><<<blocks, threads, 0, s>>>(g, F, P, phase, (double*)f);
        else if (storage == LBF_STORE_FP16)
            color_init<D2Q9, ColorPacked<D2Q9, __half>><<<blocks, threads, 0, s>>>(g, F, P, phase, h);
        else if (storage == LBF_STORE_BF16)
            color_init<D2Q9, ColorPacked<D2Q9, __nv_bfloat16>><<<blocks, threads, 0, s>>>(g, F, P, phase, h);
        else color_init<D2Q9, StoreF32Full><<<blocks, threads, 0, s>>>(g, F, P, phase, (float*)f);
    }
}

}  // namespace lbf
