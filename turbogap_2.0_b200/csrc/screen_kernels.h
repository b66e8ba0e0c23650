// Learned screen of the Monte Carlo driver (screen.cu).
#pragma once

#include <cuda_bf16.h>

#include "tgap_internal.h"

namespace tgap {

constexpr int kScreenThreads = 512;
constexpr int kScreenRows = 4;  // rows per CTA (one float4 of activations per input index)
constexpr int kScreenMaxPca = 256;
constexpr int kScreenMaxHidden = 512;

// Device view of the screen weights, stored transposed (input index major); bf16 weights,
// FP32 biases and mean.
struct ScreenDev {
    int dim, n_pca, n_hidden;
    const float *mean;            // [dim]
    const __nv_bfloat16 *pca;     // [dim][n_pca]
    const __nv_bfloat16 *w1;      // [n_pca][n_hidden]
    const float *b1;              // [n_hidden]
    const __nv_bfloat16 *w2;      // [n_hidden][n_hidden] (input major)
    const float *b2;              // [n_hidden]
    const __nv_bfloat16 *w3;      // [n_hidden]
    float b3;
};

// Shared memory of one screen CTA (weights, biases, kScreenRows rows of activations and the
// split-reduction partials).
size_t screen_smem_bytes(int dim, int n_pca, int n_hidden);

// Screen energies of n_rows descriptor rows (rows >= *d_count skipped when d_count is set).
int screen_rows(tgap_context *ctx, const ScreenDev &s, const float *d_q, int q_ld, int n_rows, const int *d_count,
                float *d_e);

}  // namespace tgap
