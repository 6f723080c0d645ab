// Template instantiation and dispatch of the single-phase kernels.
#include "internal.h"
#include "../../include/lbflow.h"

namespace lbf {

namespace {
template <class L, class S>
void dispatch(bool mrt, bool pull, int out, const ScspLaunch& a)
{
    using T = typename S::T;
    const T* fin = static_cast<const T*>(a.fin);
    T* fout = static_cast<T*>(a.fout);
    const unsigned threads = 128, blocks = blocks_for(a.g.nf, threads);
    if (blocks == 0) return;
    (void)mrt;   // the collision rates (SRT or MRT) are in a.P.rate
    if (pull)
        scsp_step<L, S, true><<<blocks, threads, 0, a.stream>>>(a.g, a.F, a.P, fin, fout, a.mo, out, a.err, a.ein, a.eout);
    else
        scsp_step<L, S, false><<<blocks, threads, 0, a.stream>>>(a.g, a.F, a.P, fin, fout, a.mo, out, a.err, a.ein, a.eout);
}

template <class L>
void dispatch_storage(int storage, bool mrt, bool pull, int out, const ScspLaunch& a)
{
    switch (storage) {
    case LBF_STORE_FP64: dispatch<L, StoreF64>(mrt, pull, out, a); break;
    case LBF_STORE_FP16: dispatch<L, StoreF16<L>>(mrt, pull, out, a); break;
    case LBF_STORE_BF16: dispatch<L, StoreBF16<L>>(mrt, pull, out, a); break;
    case LBF_STORE_BFP16: dispatch<L, StoreBFP16<L>>(mrt, pull, out, a); break;
    default: dispatch<L, StoreF32<L>>(mrt, pull, out, a); break;
    }
}

template <class L, class S>
void zou_he(const ScspLaunch& a, const ZouHe& z)
{
    using T = typename S::T;
    const unsigned threads = 128, blocks = blocks_for(z.n, threads);
    if (blocks == 0) return;
    scsp_zou_he<L, S><<<blocks, threads, 0, a.stream>>>(a.g, a.P, z, static_cast<const T*>(a.fin),
                                                         static_cast<T*>(a.fout), a.mo, a.out, a.err,
                                                         a.ein, a.eout);
}

template <class L>
void zou_he_storage(int storage, const ScspLaunch& a, const ZouHe& z)
{
    switch (storage) {
    case LBF_STORE_FP64: zou_he<L, StoreF64>(a, z); break;
    case LBF_STORE_FP16: zou_he<L, StoreF16<L>>(a, z); break;
    case LBF_STORE_BF16: zou_he<L, StoreBF16<L>>(a, z); break;
    case LBF_STORE_BFP16: zou_he<L, StoreBFP16<L>>(a, z); break;
    default: zou_he<L, StoreF32<L>>(a, z); break;
    }
}

template <class L>
void init_storage(int storage, const Grid& g, const Force& F, double rho0, void* f, int8_t* e, cudaStream_t s)
{
    const unsigned threads = 256, blocks = blocks_for(g.nf, threads);
    if (blocks == 0) return;
    switch (storage) {
    case LBF_STORE_FP64: scsp_init<L, StoreF64><<<blocks, threads, 0, s>>>(g, F, rho0, (double*)f, e); break;
    case LBF_STORE_FP16: scsp_init<L, StoreF16<L>><<<blocks, threads, 0, s>>>(g, F, rho0, (__half*)f, e); break;
    case LBF_STORE_BF16: scsp_init<L, StoreBF16<L>><<<blocks, threads, 0, s>>>(g, F, rho0, (__nv_bfloat16*)f, e); break;
    case LBF_STORE_BFP16: scsp_init<L, StoreBFP16<L>><<<blocks, threads, 0, s>>>(g, F, rho0, (int16_t*)f, e); break;
    default: scsp_init<L, StoreF32<L>><<<blocks, threads, 0, s>>>(g, F, rho0, (float*)f, e); break;
    }
}
template <class L>
void init_eq_storage(int storage, const Grid& g, const Force& F, double rho0, const float* fields, uint32_t ld,
                     void* f, int8_t* e, cudaStream_t s)
{
    const unsigned threads = 256, blocks = blocks_for(g.nf, threads);
    if (blocks == 0) return;
    switch (storage) {
    case LBF_STORE_FP64: scsp_init_eq<L, StoreF64><<<blocks, threads, 0, s>>>(g, F, rho0, fields, ld, (double*)f, e); break;
    case LBF_STORE_FP16: scsp_init_eq<L, StoreF16<L>><<<blocks, threads, 0, s>>>(g, F, rho0, fields, ld, (__half*)f, e); break;
    case LBF_STORE_BF16: scsp_init_eq<L, StoreBF16<L>><<<blocks, threads, 0, s>>>(g, F, rho0, fields, ld, (__nv_bfloat16*)f, e); break;
    case LBF_STORE_BFP16: scsp_init_eq<L, StoreBFP16<L>><<<blocks, threads, 0, s>>>(g, F, rho0, fields, ld, (int16_t*)f, e); break;
    default: scsp_init_eq<L, StoreF32<L>><<<blocks, threads, 0, s>>>(g, F, rho0, fields, ld, (float*)f, e); break;
    }
}
template <class L>
void add_density_storage(int storage, const Grid& g, const float* drho, void* f, int8_t* e, double rho0,
                         cudaStream_t s)
{
    const unsigned threads = 256, blocks = blocks_for(g.nf, threads);
    if (blocks == 0) return;
    switch (storage) {
    case LBF_STORE_FP64: scsp_add_density<L, StoreF64><<<blocks, threads, 0, s>>>(g, drho, (double*)f, e, rho0); break;
    case LBF_STORE_FP16: scsp_add_density<L, StoreF16<L>><<<blocks, threads, 0, s>>>(g, drho, (__half*)f, e, rho0); break;
    case LBF_STORE_BF16: scsp_add_density<L, StoreBF16<L>><<<blocks, threads, 0, s>>>(g, drho, (__nv_bfloat16*)f, e, rho0); break;
    case LBF_STORE_BFP16: scsp_add_density<L, StoreBFP16<L>><<<blocks, threads, 0, s>>>(g, drho, (int16_t*)f, e, rho0); break;
    default: scsp_add_density<L, StoreF32<L>><<<blocks, threads, 0, s>>>(g, drho, (float*)f, e, rho0); break;
    }
}
}  // namespace

void launch_scsp_add_density(int dims, int storage, const Grid& g, const float* drho, void* f, int8_t* e,
                             double rho0, cudaStream_t s)
{
    if (dims == 3) add_density_storage<D3Q19>(storage, g, drho, f, e, rho0, s);
    else add_density_storage<D2Q9>(storage, g, drho, f, e, rho0, s);
}

void launch_scsp_init_eq(int dims, int storage, const Grid& g, const Force& F, double rho0, const float* fields,
                         uint32_t ld, void* f, int8_t* e, cudaStream_t s)
{
    if (dims == 3) init_eq_storage<D3Q19>(storage, g, F, rho0, fields, ld, f, e, s);
    else init_eq_storage<D2Q9>(storage, g, F, rho0, fields, ld, f, e, s);
}

void launch_scsp(int dims, int storage, bool mrt, bool pull, int out, const ScspLaunch& a)
{
    if (dims == 3) dispatch_storage<D3Q19>(storage, mrt, pull, out, a);
    else dispatch_storage<D2Q9>(storage, mrt, pull, out, a);
}

void launch_scsp_zou_he(int dims, int storage, const ScspLaunch& a, const ZouHe& z)
{
    if (dims == 3) zou_he_storage<D3Q19>(storage, a, z);
    else zou_he_storage<D2Q9>(storage, a, z);
}

void launch_scsp_init(int dims, int storage, const Grid& g, const Force& F, double rho0,
                      void* f, int8_t* e, cudaStream_t s)
{
    if (dims == 3) init_storage<D3Q19>(storage, g, F, rho0, f, e, s);
    else init_storage<D2Q9>(storage, g, F, rho0, f, e, s);
}

}  // namespace lbf
