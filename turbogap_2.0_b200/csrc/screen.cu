// Learned screen of the Monte Carlo driver: per-atom energy surrogate
//   e(q) = w3 . silu(W2 silu(W1 P (q - mu) + b1) + b2) + b3
// on the normalised descriptor q (FP32), P the PCA projection. Weights are stored in bf16
// (transposed: input index major) and every product accumulates in FP32.
//
// One CTA evaluates kScreenRows rows, so a Monte Carlo trial (a few dozen rows) spreads over
// several SMs. The CTA stages the weights in shared memory with 16-byte loads (one L2 round
// trip), keeps the activations input-index major with the rows innermost (one float4 broadcast
// per input index feeds all rows), and splits each layer's reduction over S slices of the input
// index so that all threads work even when the layer has few outputs.
#include <cuda_bf16.h>

#include <algorithm>

#include "screen_kernels.h"

namespace tgap {

namespace {

constexpr int RB = kScreenRows;
static_assert(RB == 4, "activations are read as one float4 per input index");

__device__ __forceinline__ float silu(float x) { return x / (1.0f + __expf(-x)); }

__host__ __device__ inline size_t weight_bytes(int D, int K, int H)
{
    return ((2 * ((size_t)D * K + (size_t)K * H + (size_t)H * H)) + 15) / 16 * 16;
}

__device__ __forceinline__ int slices(int n_out) { return max(1, kScreenThreads / n_out); }

// part[s][o] (float4 over rows) = sum over the s-th slice of k of W[k][o] * act[k]
__device__ __forceinline__ void layer_partials(const float4 *__restrict__ act, int n_in,
                                               const __nv_bfloat16 *__restrict__ W, int n_out,
                                               float4 *__restrict__ part)
{
    const int S = slices(n_out);
    for (int w = threadIdx.x; w < n_out * S; w += blockDim.x) {
        const int o = w % n_out, s = w / n_out;
        const int k0 = s * n_in / S, k1 = (s + 1) * n_in / S;
        float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll 4
        for (int k = k0; k < k1; ++k) {
            const float wk = __bfloat162float(W[(size_t)k * n_out + o]);
            const float4 a = act[k];
            acc.x = fmaf(wk, a.x, acc.x);
            acc.y = fmaf(wk, a.y, acc.y);
            acc.z = fmaf(wk, a.z, acc.z);
            acc.w = fmaf(wk, a.w, acc.w);
        }
        part[(size_t)s * n_out + o] = acc;
    }
}

__device__ __forceinline__ float4 sum_slices(const float4 *__restrict__ part, int n_out, int o)
{
    const int S = slices(n_out);
    float4 v = part[o];
    for (int s = 1; s < S; ++s) {
        const float4 p = part[(size_t)s * n_out + o];
        v.x += p.x;
        v.y += p.y;
        v.z += p.z;
        v.w += p.w;
    }
    return v;
}

__device__ __forceinline__ float4 silu4(float4 v, float b)
{
    return make_float4(silu(v.x + b), silu(v.y + b), silu(v.z + b), silu(v.w + b));
}

}  // namespace

size_t screen_smem_bytes(int dim, int n_pca, int n_hidden)
{
    const size_t f = 3 * (size_t)n_hidden;                                        // b1, b2, w3
    const size_t a = (size_t)RB * ((size_t)dim + n_pca + (size_t)n_hidden);      // activations
    const size_t p = (size_t)RB * std::max<size_t>((size_t)kScreenThreads, (size_t)n_hidden);  // partials
    return weight_bytes(dim, n_pca, n_hidden) + 4 * (f + ((a + 3) / 4 * 4) + p) + 16;
}

// rows: descriptor rows q[r * q_ld + d], d < dim; rows r >= count (count = *d_count when set,
// else n_rows) are skipped. Writes e_out[r]. CTA b takes rows [b RB, (b+1) RB).
__global__ void __launch_bounds__(kScreenThreads) k_screen(ScreenDev s, const float *__restrict__ q, int q_ld,
                                                           int n_rows, const int *__restrict__ d_count,
                                                           float *__restrict__ e_out)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int count = d_count ? min(*d_count, n_rows) : n_rows;
    const int r0 = blockIdx.x * RB;
    const int nr = min(RB, count - r0);
    if (nr <= 0) return;
    const int D = s.dim, K = s.n_pca, H = s.n_hidden, t = threadIdx.x, T = blockDim.x;
    __nv_bfloat16 *Pt = reinterpret_cast<__nv_bfloat16 *>(smem_raw);  // [D][K]
    __nv_bfloat16 *W1t = Pt + (size_t)D * K;                           // [K][H]
    __nv_bfloat16 *W2t = W1t + (size_t)K * H;                          // [H][H]
    float4 *X = reinterpret_cast<float4 *>(smem_raw + weight_bytes(D, K, H));  // [D] rows of q - mean
    float4 *Z = X + D;                                                         // [K]
    float4 *H1 = Z + K;                                                        // [H]
    float4 *PT = H1 + H;                                                       // partials
    float *b1 = reinterpret_cast<float *>(PT + max(kScreenThreads, H));
    float *b2 = b1 + H, *w3 = b2 + H;
    {
        // 16-byte copies where the matrix splits evenly (8 bf16), element copies otherwise
        auto stage = [&](__nv_bfloat16 *dst, const __nv_bfloat16 *src, size_t n) {
            const bool vec = n % 8 == 0 && (reinterpret_cast<uintptr_t>(dst) % 16 == 0) &&
                             (reinterpret_cast<uintptr_t>(src) % 16 == 0);
            if (vec) {
                for (size_t i = t; i < n / 8; i += T)
                    reinterpret_cast<uint4 *>(dst)[i] = reinterpret_cast<const uint4 *>(src)[i];
            } else {
                for (size_t i = t; i < n; i += T) dst[i] = src[i];
            }
        };
        stage(Pt, s.pca, (size_t)D * K);
        stage(W1t, s.w1, (size_t)K * H);
        stage(W2t, s.w2, (size_t)H * H);
    }
    for (int i = t; i < H; i += T) {
        w3[i] = __bfloat162float(s.w3[i]);
        b1[i] = s.b1[i];
        b2[i] = s.b2[i];
    }
    // rows of q - mean, input index major (rows past nr are zero and never written out)
    for (int d = t; d < D; d += T) {
        const float mu = s.mean[d];
        float v[RB];
#pragma unroll
        for (int r = 0; r < RB; ++r) v[r] = r < nr ? q[(size_t)(r0 + r) * q_ld + d] - mu : 0.0f;
        X[d] = make_float4(v[0], v[1], v[2], v[3]);
    }
    __syncthreads();
    // z = P (q - mean)
    layer_partials(X, D, Pt, K, PT);
    __syncthreads();
    for (int o = t; o < K; o += T) Z[o] = sum_slices(PT, K, o);
    __syncthreads();
    // h1 = silu(W1 z + b1)
    layer_partials(Z, K, W1t, H, PT);
    __syncthreads();
    for (int o = t; o < H; o += T) H1[o] = silu4(sum_slices(PT, H, o), b1[o]);
    __syncthreads();
    // w3 (.) silu(W2 h1 + b2), summed over the hidden index per row
    layer_partials(H1, H, W2t, H, PT);
    __syncthreads();
    float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int o = t; o < H; o += T) {
        const float4 h2 = silu4(sum_slices(PT, H, o), b2[o]);
        acc.x = fmaf(w3[o], h2.x, acc.x);
        acc.y = fmaf(w3[o], h2.y, acc.y);
        acc.z = fmaf(w3[o], h2.z, acc.z);
        acc.w = fmaf(w3[o], h2.w, acc.w);
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        acc.x += __shfl_xor_sync(0xffffffffu, acc.x, off);
        acc.y += __shfl_xor_sync(0xffffffffu, acc.y, off);
        acc.z += __shfl_xor_sync(0xffffffffu, acc.z, off);
        acc.w += __shfl_xor_sync(0xffffffffu, acc.w, off);
    }
    __syncthreads();  // PT is reused for the per-warp sums
    const int warp = t >> 5, nw = T >> 5;
    if ((t & 31) == 0) PT[warp] = acc;
    __syncthreads();
    if (t < nr) {
        float e = s.b3;
        for (int w = 0; w < nw; ++w) {
            const float4 p = PT[w];
            e += t == 0 ? p.x : t == 1 ? p.y : t == 2 ? p.z : p.w;
        }
        e_out[r0 + t] = e;
    }
}

int screen_rows(tgap_context *ctx, const ScreenDev &s, const float *d_q, int q_ld, int n_rows, const int *d_count,
                float *d_e)
{
    if (n_rows <= 0) return TGAP_OK;
    const size_t sm = screen_smem_bytes(s.dim, s.n_pca, s.n_hidden);
    TGAP_CUDA(ctx, cudaFuncSetAttribute(k_screen, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    StageScope sc(ctx, "mc_screen");
    k_screen<<<(n_rows + RB - 1) / RB, kScreenThreads, sm, ctx->stream>>>(s, d_q, q_ld, n_rows, d_count, d_e);
    TGAP_LAUNCH_CHECK(ctx);
    return TGAP_OK;
}

}  // namespace tgap
