// Lattice descriptors for the two velocity sets LBFlow simulates.
//
// Directions keep the reference's q ordering (solver/src/grid/gridspace.cpp:
// 82-97 for D2Q9, 106-144 for D3Q19) because that ordering is the block order
// of the population checkpoint.  Components are stored here as (x, y, z),
// whereas the reference stores them {y,x} / {z,y,x}; the values are the same.
//
// The reference's MRT transform (solver/src/lbm/simulator.cpp:162-197) is not
// needed on the device: with its legacy rates the collision is a two-rate
// update of opposite-direction pairs (kernels.cuh, collide_trt), so the
// descriptor carries the pairing instead.
#pragma once
#include <cstdint>

namespace lbf {

struct D2Q9 {
    static constexpr int D = 2, Q = 9, NPAIR = 4;
    __host__ __device__ static constexpr int ex(int i)
    { constexpr int t[9] = {0, 1, 0, -1, 0, 1, -1, -1, 1}; return t[i]; }
    __host__ __device__ static constexpr int ey(int i)
    { constexpr int t[9] = {0, 0, 1, 0, -1, 1, 1, -1, -1}; return t[i]; }
    __host__ __device__ static constexpr int ez(int i)
    { constexpr int t[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}; return t[i]; }
    __host__ __device__ static constexpr int op(int i)
    { constexpr int t[9] = {0, 3, 4, 1, 2, 7, 8, 5, 6}; return t[i]; }
    __host__ __device__ static constexpr int w36(int i)
    { constexpr int t[9] = {16, 4, 4, 4, 4, 1, 1, 1, 1}; return t[i]; }
    __host__ __device__ static constexpr int w36f(int q) { return q == 0 ? 16 : (q < 5 ? 4 : 1); }
    // One representative of each opposite pair.
    __host__ __device__ static constexpr int pair(int i)
    { constexpr int t[4] = {1, 2, 5, 6}; return t[i]; }
    // Color-gradient and perturbation weights (colorfluid.cpp:1152-1168).
    __host__ __device__ static constexpr double B(int i)
    { constexpr double t[9] = {-4.0/27, 2.0/27, 2.0/27, 2.0/27, 2.0/27,
                                     5.0/108, 5.0/108, 5.0/108, 5.0/108}; return t[i]; }
    // QrelD (gridspace.cpp:93): per reference axis (y, x), the gradient directions.
    static constexpr int NRELD = 6;
    __host__ __device__ static constexpr int reld(int i, int j)
    { constexpr int t[2][6] = {{2, 5, 6, 4, 7, 8}, {1, 5, 8, 3, 6, 7}}; return t[i][j]; }
};

struct D3Q19 {
    static constexpr int D = 3, Q = 19, NPAIR = 9;
    __host__ __device__ static constexpr int ex(int i)
    { constexpr int t[19] = {0, 1,-1, 0, 0, 0, 0, 1,-1, 1,-1, 1,-1, 1,-1, 0, 0, 0, 0}; return t[i]; }
    __host__ __device__ static constexpr int ey(int i)
    { constexpr int t[19] = {0, 0, 0, 1,-1, 0, 0, 1, 1,-1,-1, 0, 0, 0, 0, 1,-1, 1,-1}; return t[i]; }
    __host__ __device__ static constexpr int ez(int i)
    { constexpr int t[19] = {0, 0, 0, 0, 0, 1,-1, 0, 0, 0, 0, 1, 1,-1,-1, 1, 1,-1,-1}; return t[i]; }
    __host__ __device__ static constexpr int op(int i)
    { constexpr int t[19] = {0, 2, 1, 4, 3, 6, 5, 10, 9, 8, 7, 14, 13, 12, 11, 18, 17, 16, 15}; return t[i]; }
    __host__ __device__ static constexpr int w36(int i)
    { constexpr int t[19] = {12, 2, 2, 2, 2, 2, 2, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1}; return t[i]; }
    __host__ __device__ static constexpr int w36f(int q) { return q == 0 ? 12 : (q < 7 ? 2 : 1); }
    __host__ __device__ static constexpr int pair(int i)
    { constexpr int t[9] = {1, 3, 5, 7, 8, 11, 12, 15, 16}; return t[i]; }
    __host__ __device__ static constexpr double B(int i)
    { constexpr double t[19] = {
        -(2.0 + 2.0*2) / (3.0*2 + 12.0),
        2.0 / (6.0*2 + 24.0), 2.0 / (6.0*2 + 24.0), 2.0 / (6.0*2 + 24.0),
        2.0 / (6.0*2 + 24.0), 2.0 / (6.0*2 + 24.0), 2.0 / (6.0*2 + 24.0),
        1.0 / (6.0*2 + 24.0), 1.0 / (6.0*2 + 24.0), 1.0 / (6.0*2 + 24.0),
        1.0 / (6.0*2 + 24.0), 1.0 / (6.0*2 + 24.0), 1.0 / (6.0*2 + 24.0),
        1.0 / (6.0*2 + 24.0), 1.0 / (6.0*2 + 24.0), 1.0 / (6.0*2 + 24.0),
        1.0 / (6.0*2 + 24.0), 1.0 / (6.0*2 + 24.0), 1.0 / (6.0*2 + 24.0)}; return t[i]; }
    // QrelD (gridspace.cpp:132-134): per reference axis (z, y, x).
    static constexpr int NRELD = 10;
    __host__ __device__ static constexpr int reld(int i, int j)
    { constexpr int t[3][10] = {{5, 11, 12, 15, 16, 6, 13, 14, 17, 18},
                                        {3, 8, 7, 15, 17, 4, 9, 10, 16, 18},
                                        {1, 7, 9, 11, 13, 2, 8, 10, 12, 14}}; return t[i][j]; }
};

// ---- compile-time moment tables ------------------------------------------
template <class L> __host__ __device__ constexpr int comp(int q, int a)
{ return a == 0 ? L::ex(q) : (a == 1 ? L::ey(q) : L::ez(q)); }

template <class L> __host__ __device__ constexpr double w(int q) { return L::w36f(q) / 36.0; }
template <class L> __host__ __device__ constexpr bool axis_dir(int q)
{ return (L::ex(q) != 0) + (L::ey(q) != 0) + (L::ez(q) != 0) == 1; }

}  // namespace lbf
