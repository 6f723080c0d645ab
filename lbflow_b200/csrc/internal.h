// Internal interfaces between the engine's translation units.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <string>
#include "kernels.cuh"
#include "color.cuh"

namespace lbf {

struct ScspLaunch {
    Grid g;
    Force F;
    ScspParams P;
    const void* fin;
    void* fout;
    Macros mo;
    uint32_t* err;
    cudaStream_t stream;
    const int8_t* ein;   // block exponents of fin (block-scaled storage only)
    int8_t* eout;
    int out;             // kOutMacros / kOutAdjacent of this step (boundary pass)
};

struct ColorLaunch {
    Grid g;
    Force F;
    ColorParams P;
    ColorWall W;
    const void* fin;   // [2][Q][nfp]
    void* fout;
    double2* dens;     // [nfp] component densities (rho0, rho1) of this step (written by pass 1)
    double* phid;      // [N] phase field (rho0 - rho1)/rho per voxel (solid voxels: kSolidPhi)
    Macros mo;
    uint32_t* err;
    cudaStream_t stream;
    ZouHe zh;          // PB/VB boundary nodes (n = 0: none)
    Film film;         // half-permeable film bitmaps (nullptr: none)
};

// storage: LBF_STORE_* value; dims: 2 or 3.
void launch_scsp(int dims, int storage, bool mrt, bool pull, int out, const ScspLaunch& a);
void launch_scsp_init(int dims, int storage, const Grid& g, const Force& F, double rho0,
                      void* f, int8_t* eout, cudaStream_t s);
// Zou-He PB/VB boundary pass of one pull step (after launch_scsp, same buffers).
void launch_scsp_zou_he(int dims, int storage, const ScspLaunch& a, const ZouHe& z);
void launch_scsp_add_density(int dims, int storage, const Grid& g, const float* drho, void* f, int8_t* eio,
                             double rho0, cudaStream_t s);
void launch_scsp_init_eq(int dims, int storage, const Grid& g, const Force& F, double rho0, const float* fields,
                         uint32_t ld, void* f, int8_t* eout, cudaStream_t s);
void launch_color(int dims, int storage, int collision, bool pull, int out, const ColorLaunch& a);
void launch_color_init(int dims, int storage, const Grid& g, const Force& F, const ColorParams& P,
                       const uint8_t* phase, void* f, cudaStream_t s);

// The library's stream-ordered device memory pool of a device (created on
// first use; keeps freed memory reserved for reuse up to a fixed amount), so
// that work repeated inside a run allocates without driver calls.
cudaError_t device_pool(int device, cudaMemPool_t* pool);

// Message returned by lbf_last_error(NULL) (calls without an engine).
void set_global_error(const std::string& msg);

inline unsigned blocks_for(uint32_t n, unsigned threads) { return (n + threads - 1) / threads; }

}  // namespace lbf
