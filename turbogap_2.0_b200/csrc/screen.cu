// Learned screen of the Monte Carlo driver: per-atom energy surrogate
//   e(q) = w3 . silu(W2 silu(W1 P (q - mu) + b1) + b2) + b3
// on the normalised descriptor q (FP32), P the PCA projection. Weights are stored in bf16 and
// every product accumulates in FP32. One CTA per descriptor row.
#include <cuda_bf16.h>

#include "screen_kernels.h"

namespace tgap {

__device__ __forceinline__ float silu(float x) { return x / (1.0f + __expf(-x)); }

// rows: descriptor rows q[r * q_ld + d], d < dim; rows with r >= *d_count (when d_count is set)
// are skipped. Writes e_out[r].
__global__ void __launch_bounds__(kScreenThreads) k_screen(ScreenDev s, const float *__restrict__ q, int q_ld,
                                                           int n_rows, const int *__restrict__ d_count,
                                                           float *__restrict__ e_out)
{
    extern __shared__ float sh[];
    float *qs = sh;              // [dim]
    float *z = qs + s.dim;       // [n_pca]
    float *h1 = z + s.n_pca;     // [n_hidden]
    float *h2 = h1 + s.n_hidden; // [n_hidden]
    __shared__ float red[kScreenThreads / 32];
    const int r = blockIdx.x, t = threadIdx.x;
    if (r >= n_rows || (d_count && r >= *d_count)) return;
    for (int d = t; d < s.dim; d += blockDim.x) qs[d] = q[(size_t)r * q_ld + d] - s.mean[d];
    __syncthreads();
    for (int k = t; k < s.n_pca; k += blockDim.x) {
        const __nv_bfloat16 *row = s.pca + (size_t)k * s.dim;
        float acc = 0.0f;
        for (int d = 0; d < s.dim; ++d) acc = fmaf(__bfloat162float(row[d]), qs[d], acc);
        z[k] = acc;
    }
    __syncthreads();
    for (int k = t; k < s.n_hidden; k += blockDim.x) {
        const __nv_bfloat16 *row = s.w1 + (size_t)k * s.n_pca;
        float acc = s.b1[k];
        for (int i = 0; i < s.n_pca; ++i) acc = fmaf(__bfloat162float(row[i]), z[i], acc);
        h1[k] = silu(acc);
    }
    __syncthreads();
    float part = 0.0f;
    for (int k = t; k < s.n_hidden; k += blockDim.x) {
        const __nv_bfloat16 *row = s.w2 + (size_t)k * s.n_hidden;
        float acc = s.b2[k];
        for (int i = 0; i < s.n_hidden; ++i) acc = fmaf(__bfloat162float(row[i]), h1[i], acc);
        h2[k] = silu(acc);
        part = fmaf(__bfloat162float(s.w3[k]), h2[k], part);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
    if ((t & 31) == 0) red[t >> 5] = part;
    __syncthreads();
    if (t == 0) {
        float e = s.b3;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) e += red[w];
        e_out[r] = e;
    }
}

int screen_rows(tgap_context *ctx, const ScreenDev &s, const float *d_q, int q_ld, int n_rows, const int *d_count,
                float *d_e)
{
    if (n_rows <= 0) return TGAP_OK;
    const size_t sm = sizeof(float) * ((size_t)s.dim + s.n_pca + 2 * (size_t)s.n_hidden);
    StageScope sc(ctx, "mc_screen");
    k_screen<<<n_rows, kScreenThreads, sm, ctx->stream>>>(s, d_q, q_ld, n_rows, d_count, d_e);
    TGAP_LAUNCH_CHECK(ctx);
    return TGAP_OK;
}

}  // namespace tgap
