/*
 * lbflow_operator.h - tensor-core 3D convolution kernels of the learned warm
 * start (a neural operator that predicts the steady velocity and density of
 * a periodic porous medium, used to initialise the populations).
 *
 * LBFlow has no counterpart: its solver always starts from rest
 * (SCSP::initialize, solver/src/lbm/scsp.cpp:116-134).  These entry points
 * are the device half of the warm start; the engine side is
 * lbf_initialize_equilibrium in lbflow.h.
 *
 * Conventions
 *  - Tensors are channels-last (batch, z, y, x, channel) bf16 in device
 *    memory; every gathered channel count is a multiple of 8.
 *  - A gathered operand reads source voxel  stride * row + tap - pad  on each
 *    axis, wrapped periodically, for taps 0 .. ksize-1 (ksize^3 taps, z
 *    slowest); the reduction index is k = tap * channels + channel.
 *  - Calls are asynchronous on `stream` (a cudaStream_t, NULL = legacy
 *    default stream).  They return LBF_OK or LBF_EINVAL/LBF_ECUDA; a tensor
 *    core wait that timed out sets LBF_ERR_MMA_TIMEOUT in *err.
 */
#ifndef LBFLOW_OPERATOR_H
#define LBFLOW_OPERATOR_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { LBF_ERR_MMA_TIMEOUT = 1u << 8 };

enum {
    LBF_OUT_BF16 = 0,          /* out[row][n] as bf16, row stride out_ld        */
    LBF_OUT_F32 = 1,           /* out[row][n] as fp32, row stride out_ld        */
    LBF_OUT_SCATTER2_BF16 = 2  /* n = tap*out_ld + c (8 taps of a 2x2x2 cell):
                                  out[fine voxel 2*row + tap][c] as bf16        */
};

typedef struct {
    const void *src0, *src1;   /* channels [0,c0) from src0, [c0,c0+c1) from src1 */
    uint32_t c0, c1;
    uint32_t batch;
    uint32_t in_d, in_h, in_w; /* source grid */
    uint32_t out_d, out_h, out_w; /* grid of the GEMM rows */
    uint32_t ksize, stride;    /* ksize in 1..3, stride 1 or 2 */
    int32_t pad;
} lbf_gather;

/* out[row][n] = act(sum_k A[row][k] * weight[n][k] + bias)
 *  weight: bf16 [n_pad][k_pad], zero beyond the real n and k;
 *          n_pad in {16, 32, 64} or a multiple of 128; k_pad a multiple of 64
 *          and >= ksize^3 * (c0 + c1)
 *  n:      real output columns (<= n_pad)
 *  bias:   fp32 per destination channel, or NULL
 *  act:    0 none, 1 leaky ReLU with the given slope */
typedef struct {
    lbf_gather a;
    const void *weight;
    uint32_t n, n_pad, k_pad;
    const float *bias;
    void *out;
    uint32_t out_mode, out_ld;
    uint32_t act;
    float slope;
    uint32_t *err;
} lbf_igemm;

int lbf_igemm_run(const lbf_igemm *g, void *stream);

/* Weight gradient: out[i][j] = sum_row A[row][i] * b[row][j]  (fp32)
 *  i = tap * (c0 + c1) + channel over the gathered operand a,
 *  j over the cb channels of b (bf16 [rows][cb], cb a multiple of 8).
 *  The reduction over rows is split across CTAs; partial sums go to
 *  `workspace` (lbf_wgrad_workspace bytes) and are summed in a fixed order,
 *  so the result is deterministic. */
typedef struct {
    lbf_gather a;
    const void *b;
    uint32_t cb;
    float *out;
    void *workspace;
    size_t workspace_bytes;
    uint32_t *err;
} lbf_wgrad;

size_t lbf_wgrad_workspace(const lbf_wgrad *w);
int lbf_wgrad_run(const lbf_wgrad *w, void *stream);

/* Compile-time facts of the kernels: tile rows, K per stage, stages. */
void lbf_operator_info(uint32_t out[4]);

#ifdef __cplusplus
}
#endif
#endif
