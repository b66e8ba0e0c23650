// Training and evaluation of the Monte Carlo screen network on the device.
//
// Network (per atom, on standardised PCA coordinates z of the SOAP vector):
//   a1 = W1 z + b1, h1 = silu(a1), a2 = W2 h1 + b2, h2 = silu(a2), out = w3 . h2 + b3
// Loss of a batch of B rows: (1/B) sum_r (out_r - t_r)^2. Adam (beta 0.9 / 0.999, eps 1e-8,
// bias-corrected) on FP32 master weights.
//
// One training step is two kernels:
//   k_train_fb: one CTA per kTrainRows (16) rows of the batch (gathered through the epoch's
//     row order) stages W1, W2 and the row activations in shared memory, runs the forward pass,
//     back-propagates, and writes its rows' partial gradients (and squared-error sum) as one
//     row of a [CTA][parameter] table;
//   k_train_reduce_adam: one thread per parameter sums the table's column in CTA order (a
//     deterministic reduction) and applies the Adam update.
// The matrices are small (64 x 128, 128 x 128), so the products run on the FP32 pipes from
// shared memory with odd row pitches (conflict-free column reads); this is a one-off fit, not
// the Monte Carlo hot path.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "screen_kernels.h"
#include "tgap_internal.h"

namespace tgap {

namespace {

constexpr int kTrainThreads = 256;
constexpr int kTrainRows = 16;  // rows per CTA
constexpr int kScreenGradMaxRows = 16384;  // one partial-gradient row per 16 rows

__host__ __device__ inline int odd_pitch(int n) { return n | 1; }

__device__ __forceinline__ float sigm(float a) { return 1.0f / (1.0f + __expf(-a)); }

struct TrainShape {
    int K, H;
    __host__ __device__ int n_params() const { return H * K + H * H + 3 * H + 1; }
    // parameter vector: [W1 (H x K) | b1 (H) | W2 (H x H) | b2 (H) | w3 (H) | b3]
    __host__ __device__ int o_b1() const { return H * K; }
    __host__ __device__ int o_w2() const { return H * K + H; }
    __host__ __device__ int o_b2() const { return H * K + H + H * H; }
    __host__ __device__ int o_w3() const { return H * K + 2 * H + H * H; }
    __host__ __device__ int o_b3() const { return H * K + 3 * H + H * H; }
    // partial-gradient row: the parameters, then the squared-error sum
    __host__ __device__ int row() const { return n_params() + 1; }
};

size_t train_smem_bytes(int K, int H)
{
    const size_t R = kTrainRows;
    const size_t w = (size_t)H * odd_pitch(K) + (size_t)H * odd_pitch(H) + 3 * (size_t)H;
    const size_t a = R * K + 7 * R * (size_t)H + R;  // X, A1, H1, A2, H2, GA2, GH1, GA1 (GH1/GA1 share), gout
    return 4 * (w + a + 1);
}

// rows of this step: order[s0 + i], i < n_rows; params: FP32 master vector; part: [CTA][row()]
__global__ void __launch_bounds__(kTrainThreads) k_train_fb(TrainShape S, const float *__restrict__ Z,
                                                            const float *__restrict__ T,
                                                            const int *__restrict__ order, int n_rows,
                                                            const float *__restrict__ params,
                                                            float *__restrict__ part)
{
    extern __shared__ __align__(16) float sm[];
    const int K = S.K, H = S.H, pK = odd_pitch(K), pH = odd_pitch(H), R = kTrainRows;
    const int t = threadIdx.x, NT = blockDim.x;
    const int r0 = blockIdx.x * R;
    float *W1 = sm;                  // [H][pK]
    float *W2 = W1 + H * pK;         // [H][pH]
    float *b1 = W2 + H * pH, *b2 = b1 + H, *w3 = b2 + H;
    float *X = w3 + H;               // [R][K]
    float *A1 = X + R * K;           // [R][H] each below
    float *H1 = A1 + R * H;
    float *A2 = H1 + R * H;
    float *H2 = A2 + R * H;
    float *GA2 = H2 + R * H;
    float *GA1 = GA2 + R * H;        // back-propagated h1 gradient, then the a1 gradient in place
    float *gout = GA1 + R * H;       // [R]
    float *red = gout + R;           // [1] squared-error sum
    for (int i = t; i < H * K; i += NT) W1[(i / K) * pK + i % K] = params[i];
    for (int i = t; i < H * H; i += NT) W2[(i / H) * pH + i % H] = params[S.o_w2() + i];
    for (int i = t; i < H; i += NT) {
        b1[i] = params[S.o_b1() + i];
        b2[i] = params[S.o_b2() + i];
        w3[i] = params[S.o_w3() + i];
    }
    const int nr = min(R, n_rows - r0);
    for (int i = t; i < R * K; i += NT) {
        const int r = i / K, k = i % K;
        X[i] = r < nr ? Z[(size_t)order[r0 + r] * K + k] : 0.0f;
    }
    if (t == 0) red[0] = 0.0f;
    __syncthreads();
    // forward
    for (int i = t; i < R * H; i += NT) {
        const int r = i / H, h = i % H;
        float a = b1[h];
        for (int k = 0; k < K; ++k) a = fmaf(X[r * K + k], W1[h * pK + k], a);
        A1[i] = a;
        H1[i] = a * sigm(a);
    }
    __syncthreads();
    for (int i = t; i < R * H; i += NT) {
        const int r = i / H, h = i % H;
        float a = b2[h];
        for (int k = 0; k < H; ++k) a = fmaf(H1[r * H + k], W2[h * pH + k], a);
        A2[i] = a;
        H2[i] = a * sigm(a);
    }
    __syncthreads();
    // output and dL/dout = (2/B)(out - t), one warp per row
    const float inv_b = 2.0f / (float)n_rows;
    for (int r = t >> 5; r < R; r += NT >> 5) {
        float o = 0.0f;
        for (int h = t & 31; h < H; h += 32) o = fmaf(H2[r * H + h], w3[h], o);
#pragma unroll
        for (int s = 16; s > 0; s >>= 1) o += __shfl_xor_sync(0xffffffffu, o, s);
        if ((t & 31) == 0) {
            const float e = r < nr ? o + params[S.o_b3()] - T[order[r0 + r]] : 0.0f;
            gout[r] = inv_b * e;
            atomicAdd(red, e * e);
        }
    }
    __syncthreads();
    // back-propagation: silu'(a) = s (1 + a (1 - s))
    for (int i = t; i < R * H; i += NT) {
        const int r = i / H, h = i % H;
        const float a = A2[i], s = sigm(a);
        GA2[i] = gout[r] * w3[h] * (s * (1.0f + a * (1.0f - s)));
    }
    __syncthreads();
    for (int i = t; i < R * H; i += NT) {
        const int r = i / H, k = i % H;
        float g = 0.0f;
        for (int h = 0; h < H; ++h) g = fmaf(GA2[r * H + h], W2[h * pH + k], g);
        const float a = A1[i], s = sigm(a);
        GA1[i] = g * (s * (1.0f + a * (1.0f - s)));
    }
    __syncthreads();
    // this CTA's partial gradients
    float *out = part + (size_t)blockIdx.x * S.row();
    for (int i = t; i < H * K; i += NT) {
        const int h = i / K, k = i % K;
        float g = 0.0f;
        for (int r = 0; r < R; ++r) g = fmaf(GA1[r * H + h], X[r * K + k], g);
        out[i] = g;
    }
    for (int i = t; i < H * H; i += NT) {
        const int h = i / H, k = i % H;
        float g = 0.0f;
        for (int r = 0; r < R; ++r) g = fmaf(GA2[r * H + h], H1[r * H + k], g);
        out[S.o_w2() + i] = g;
    }
    for (int h = t; h < H; h += NT) {
        float gb1 = 0.0f, gb2 = 0.0f, gw3 = 0.0f;
        for (int r = 0; r < R; ++r) {
            gb1 += GA1[r * H + h];
            gb2 += GA2[r * H + h];
            gw3 = fmaf(gout[r], H2[r * H + h], gw3);
        }
        out[S.o_b1() + h] = gb1;
        out[S.o_b2() + h] = gb2;
        out[S.o_w3() + h] = gw3;
    }
    if (t == 0) {
        float gb3 = 0.0f;
        for (int r = 0; r < R; ++r) gb3 += gout[r];
        out[S.o_b3()] = gb3;
        out[S.n_params()] = red[0];
    }
}

struct AdamStep {
    float lr, beta1, beta2, eps, bc1, bc2;  // bc = 1 - beta^step
    int update;                             // 0: gradients only
};

// grad (optional): summed gradients; loss (optional): += squared-error sum (double)
__global__ void k_train_reduce_adam(TrainShape S, const float *__restrict__ part, int n_cta, float *__restrict__ params,
                                    float *__restrict__ m, float *__restrict__ v, AdamStep a,
                                    float *__restrict__ grad, double *__restrict__ loss)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    const int np = S.n_params(), row = S.row();
    if (p > np) return;
    float g = 0.0f;
    for (int c = 0; c < n_cta; ++c) g += part[(size_t)c * row + p];
    if (p == np) {
        if (loss) *loss += (double)g;
        return;
    }
    if (grad) grad[p] = g;
    if (!a.update) return;
    const float mm = a.beta1 * m[p] + (1.0f - a.beta1) * g;
    const float vv = a.beta2 * v[p] + (1.0f - a.beta2) * g * g;
    m[p] = mm;
    v[p] = vv;
    params[p] -= a.lr * (mm / a.bc1) / (sqrtf(vv / a.bc2) + a.eps);
}

int h2d(tgap_context *ctx, DevBuf &b, const void *h, size_t bytes)
{
    if (b.ensure(bytes ? bytes : 4)) return set_error(ctx, TGAP_ERR_NOMEM, "screen training buffers");
    if (bytes) TGAP_CUDA(ctx, cudaMemcpyAsync(b.ptr, h, bytes, cudaMemcpyHostToDevice, ctx->stream));
    return TGAP_OK;
}

#define TRC(x)                \
    do {                      \
        int _rc = (x);        \
        if (_rc) return _rc;  \
    } while (0)

struct TrainBufs {
    DevBuf Z, T, order, params, m, v, part, grad, loss;
    ~TrainBufs()
    {
        for (DevBuf *b : {&Z, &T, &order, &params, &m, &v, &part, &grad, &loss}) b->release();
    }
};

int check_shape(tgap_context *ctx, int64_t n, int K, int H)
{
    if (n < 1 || n > (int64_t)1 << 30 || K < 1 || K > kScreenMaxPca || H < 1 || H > kScreenMaxHidden)
        return set_error(ctx, TGAP_ERR_ARGUMENT, "screen training: bad sizes");
    if (train_smem_bytes(K, H) > 227 * 1024)
        return set_error(ctx, TGAP_ERR_ARGUMENT, "screen training: n_pca %d x n_hidden %d exceed one CTA's shared memory",
                         K, H);
    return TGAP_OK;
}

int pack_params(const TrainShape &S, const float *w1, const float *b1, const float *w2, const float *b2,
                const float *w3, float b3, std::vector<float> &p)
{
    p.assign(S.n_params(), 0.0f);
    std::copy(w1, w1 + S.H * S.K, p.begin());
    std::copy(b1, b1 + S.H, p.begin() + S.o_b1());
    std::copy(w2, w2 + S.H * S.H, p.begin() + S.o_w2());
    std::copy(b2, b2 + S.H, p.begin() + S.o_b2());
    std::copy(w3, w3 + S.H, p.begin() + S.o_w3());
    p[S.o_b3()] = b3;
    return 0;
}

void unpack_params(const TrainShape &S, const std::vector<float> &p, float *w1, float *b1, float *w2, float *b2,
                   float *w3, float *b3)
{
    std::copy(p.begin(), p.begin() + S.H * S.K, w1);
    std::copy(p.begin() + S.o_b1(), p.begin() + S.o_b1() + S.H, b1);
    std::copy(p.begin() + S.o_w2(), p.begin() + S.o_w2() + S.H * S.H, w2);
    std::copy(p.begin() + S.o_b2(), p.begin() + S.o_b2() + S.H, b2);
    std::copy(p.begin() + S.o_w3(), p.begin() + S.o_w3() + S.H, w3);
    *b3 = p[S.o_b3()];
}

// One pass (forward + backward) over rows order[s0 .. s0 + n_rows), then the reduction (and the
// Adam update when a.update).
int train_step(tgap_context *ctx, const TrainShape &S, TrainBufs &B, int s0, int n_rows, const AdamStep &a,
               float *d_grad, double *d_loss)
{
    const int n_cta = (n_rows + kTrainRows - 1) / kTrainRows;
    const size_t sm = train_smem_bytes(S.K, S.H);
    {
        StageScope sc(ctx, "screen_train_fb");
        k_train_fb<<<n_cta, kTrainThreads, sm, ctx->stream>>>(S, B.Z.as<float>(), B.T.as<float>(),
                                                               B.order.as<int>() + s0, n_rows, B.params.as<float>(),
                                                               B.part.as<float>());
        TGAP_LAUNCH_CHECK(ctx);
    }
    StageScope sc(ctx, "screen_train_adam");
    const int np = S.n_params() + 1;
    k_train_reduce_adam<<<(np + 255) / 256, 256, 0, ctx->stream>>>(S, B.part.as<float>(), n_cta, B.params.as<float>(),
                                                                  B.m.as<float>(), B.v.as<float>(), a, d_grad, d_loss);
    TGAP_LAUNCH_CHECK(ctx);
    return TGAP_OK;
}

int setup(tgap_context *ctx, const TrainShape &S, TrainBufs &B, int64_t n, int max_rows, const float *z, const float *t,
          const std::vector<float> &p)
{
    TRC(h2d(ctx, B.Z, z, sizeof(float) * (size_t)n * S.K));
    TRC(h2d(ctx, B.T, t, sizeof(float) * (size_t)n));
    TRC(h2d(ctx, B.params, p.data(), sizeof(float) * p.size()));
    const int n_cta = (max_rows + kTrainRows - 1) / kTrainRows;
    if (B.order.ensure(sizeof(int) * (size_t)n) || B.m.ensure(sizeof(float) * p.size()) ||
        B.v.ensure(sizeof(float) * p.size()) || B.part.ensure(sizeof(float) * (size_t)n_cta * S.row()) ||
        B.loss.ensure(sizeof(double)))
        return set_error(ctx, TGAP_ERR_NOMEM, "screen training buffers");
    TGAP_CUDA(ctx, cudaMemsetAsync(B.m.ptr, 0, B.m.bytes, ctx->stream));
    TGAP_CUDA(ctx, cudaMemsetAsync(B.v.ptr, 0, B.v.bytes, ctx->stream));
    TGAP_CUDA(ctx, cudaMemsetAsync(B.loss.ptr, 0, sizeof(double), ctx->stream));
    TGAP_CUDA(ctx, cudaFuncSetAttribute(k_train_fb, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)train_smem_bytes(S.K, S.H)));
    return TGAP_OK;
}

}  // namespace

}  // namespace tgap

using namespace tgap;

extern "C" int tgap_screen_grad(tgap_context *ctx, int64_t n, int n_pca, int n_hidden, const float *z, const float *t,
                                const float *w1, const float *b1, const float *w2, const float *b2, const float *w3,
                                float b3, float *g_w1, float *g_b1, float *g_w2, float *g_b2, float *g_w3, float *g_b3,
                                double *loss)
{
    if (!ctx) return TGAP_ERR_ARGUMENT;
    if (!z || !t || !w1 || !b1 || !w2 || !b2 || !w3 || !g_w1 || !g_b1 || !g_w2 || !g_b2 || !g_w3 || !g_b3)
        return set_error(ctx, TGAP_ERR_ARGUMENT, "tgap_screen_grad: null pointer");
    TGAP_CUDA(ctx, cudaSetDevice(ctx->device));
    TRC(check_shape(ctx, n, n_pca, n_hidden));
    if (n > kScreenGradMaxRows)
        return set_error(ctx, TGAP_ERR_ARGUMENT, "tgap_screen_grad: at most %d rows per call", kScreenGradMaxRows);
    const TrainShape S{n_pca, n_hidden};
    std::vector<float> p;
    pack_params(S, w1, b1, w2, b2, w3, b3, p);
    TrainBufs B;
    TRC(setup(ctx, S, B, n, (int)n, z, t, p));
    std::vector<int> ord((size_t)n);
    for (int64_t i = 0; i < n; ++i) ord[i] = (int)i;
    TGAP_CUDA(ctx, cudaMemcpyAsync(B.order.ptr, ord.data(), sizeof(int) * ord.size(), cudaMemcpyHostToDevice,
                                   ctx->stream));
    if (B.grad.ensure(sizeof(float) * p.size())) return set_error(ctx, TGAP_ERR_NOMEM, "screen training buffers");
    const AdamStep a{0.f, 0.9f, 0.999f, 1e-8f, 1.f, 1.f, 0};
    TRC(train_step(ctx, S, B, 0, (int)n, a, B.grad.as<float>(), B.loss.as<double>()));
    std::vector<float> g(p.size());
    double l = 0.0;
    TGAP_CUDA(ctx, cudaMemcpyAsync(g.data(), B.grad.ptr, sizeof(float) * g.size(), cudaMemcpyDeviceToHost, ctx->stream));
    TGAP_CUDA(ctx, cudaMemcpyAsync(&l, B.loss.ptr, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    TGAP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    unpack_params(S, g, g_w1, g_b1, g_w2, g_b2, g_w3, g_b3);
    if (loss) *loss = l / (double)n;
    return read_device_check(ctx);
}

extern "C" int tgap_screen_train(tgap_context *ctx, int64_t n, int n_pca, int n_hidden, const float *z, const float *t,
                                 int epochs, int batch, float lr, const int *order, float *w1, float *b1, float *w2,
                                 float *b2, float *w3, float *b3, double *loss_log)
{
    if (!ctx) return TGAP_ERR_ARGUMENT;
    if (!z || !t || !order || !w1 || !b1 || !w2 || !b2 || !w3 || !b3 || epochs < 1 || batch < 1 || !(lr > 0.0f))
        return set_error(ctx, TGAP_ERR_ARGUMENT, "tgap_screen_train: bad arguments");
    TGAP_CUDA(ctx, cudaSetDevice(ctx->device));
    TRC(check_shape(ctx, n, n_pca, n_hidden));
    for (int64_t i = 0; i < (int64_t)epochs * n; ++i)
        if (order[i] < 0 || order[i] >= n) return set_error(ctx, TGAP_ERR_ARGUMENT, "tgap_screen_train: order[%lld]", (long long)i);
    const TrainShape S{n_pca, n_hidden};
    std::vector<float> p;
    pack_params(S, w1, b1, w2, b2, w3, *b3, p);
    TrainBufs B;
    const int bmax = (int)std::min<int64_t>(batch, n);
    TRC(setup(ctx, S, B, n, bmax, z, t, p));
    const double pi = 3.14159265358979323846;
    std::vector<double> losses((size_t)epochs, 0.0);
    int64_t step = 0;
    for (int ep = 0; ep < epochs; ++ep) {
        TGAP_CUDA(ctx, cudaMemcpyAsync(B.order.ptr, order + (size_t)ep * n, sizeof(int) * (size_t)n,
                                       cudaMemcpyHostToDevice, ctx->stream));
        TGAP_CUDA(ctx, cudaMemsetAsync(B.loss.ptr, 0, sizeof(double), ctx->stream));
        const float lr_ep = (float)(lr * 0.5 * (1.0 + std::cos(pi * ep / epochs)));
        for (int64_t s0 = 0; s0 < n; s0 += batch) {
            ++step;
            const int rows = (int)std::min<int64_t>(batch, n - s0);
            const AdamStep a{lr_ep, 0.9f, 0.999f, 1e-8f, (float)(1.0 - std::pow(0.9, (double)step)),
                             (float)(1.0 - std::pow(0.999, (double)step)), 1};
            TRC(train_step(ctx, S, B, (int)s0, rows, a, nullptr, B.loss.as<double>()));
        }
        TGAP_CUDA(ctx, cudaMemcpyAsync(&losses[ep], B.loss.ptr, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    }
    TGAP_CUDA(ctx, cudaMemcpyAsync(p.data(), B.params.ptr, sizeof(float) * p.size(), cudaMemcpyDeviceToHost,
                                   ctx->stream));
    TGAP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    unpack_params(S, p, w1, b1, w2, b2, w3, b3);
    if (loss_log)
        for (int ep = 0; ep < epochs; ++ep) loss_log[ep] = losses[ep] / (double)n;
    return read_device_check(ctx);
}

extern "C" int tgap_screen_eval(tgap_context *ctx, int64_t n, int dim, int n_pca, int n_hidden, const float *mean,
                                const float *pca, const float *w1, const float *b1, const float *w2, const float *b2,
                                const float *w3, float b3, const float *q, double *e)
{
    if (!ctx) return TGAP_ERR_ARGUMENT;
    if (!mean || !pca || !w1 || !b1 || !w2 || !b2 || !w3 || !q || !e || n < 0 || n > ((int64_t)1 << 30) || dim < 1 ||
        n_pca < 1 || n_pca > kScreenMaxPca || n_hidden < 1 || n_hidden > kScreenMaxHidden)
        return set_error(ctx, TGAP_ERR_ARGUMENT, "tgap_screen_eval: bad arguments");
    if (screen_smem_bytes(dim, n_pca, n_hidden) > 227 * 1024)
        return set_error(ctx, TGAP_ERR_ARGUMENT, "screen too large for one CTA's shared memory");
    if (n == 0) return TGAP_OK;
    TGAP_CUDA(ctx, cudaSetDevice(ctx->device));
    // bf16, transposed to input-index-major, as the Monte Carlo driver stores them
    auto to_bf16_t = [](const float *x, size_t rows, size_t cols) {
        std::vector<__nv_bfloat16> v(rows * cols);
        for (size_t r = 0; r < rows; ++r)
            for (size_t c = 0; c < cols; ++c) v[c * rows + r] = __float2bfloat16_rn(x[r * cols + c]);
        return v;
    };
    const auto vp = to_bf16_t(pca, n_pca, dim), v1 = to_bf16_t(w1, n_hidden, n_pca),
               v2 = to_bf16_t(w2, n_hidden, n_hidden), v3 = to_bf16_t(w3, n_hidden, 1);
    struct Bufs {
        DevBuf mean, pca, w1, b1, w2, b2, w3, q, e;
        ~Bufs()
        {
            for (DevBuf *b : {&mean, &pca, &w1, &b1, &w2, &b2, &w3, &q, &e}) b->release();
        }
    } B;
    TRC(h2d(ctx, B.mean, mean, 4 * (size_t)dim));
    TRC(h2d(ctx, B.pca, vp.data(), 2 * vp.size()));
    TRC(h2d(ctx, B.w1, v1.data(), 2 * v1.size()));
    TRC(h2d(ctx, B.b1, b1, 4 * (size_t)n_hidden));
    TRC(h2d(ctx, B.w2, v2.data(), 2 * v2.size()));
    TRC(h2d(ctx, B.b2, b2, 4 * (size_t)n_hidden));
    TRC(h2d(ctx, B.w3, v3.data(), 2 * v3.size()));
    TRC(h2d(ctx, B.q, q, 4 * (size_t)n * dim));
    if (B.e.ensure(4 * (size_t)n)) return set_error(ctx, TGAP_ERR_NOMEM, "screen evaluation buffers");
    const ScreenDev sd{dim, n_pca, n_hidden, B.mean.as<float>(), B.pca.as<__nv_bfloat16>(), B.w1.as<__nv_bfloat16>(),
                       B.b1.as<float>(), B.w2.as<__nv_bfloat16>(), B.b2.as<float>(), B.w3.as<__nv_bfloat16>(), b3};
    TRC(screen_rows(ctx, sd, B.q.as<float>(), dim, (int)n, nullptr, B.e.as<float>()));
    std::vector<float> ef((size_t)n);
    TGAP_CUDA(ctx, cudaMemcpyAsync(ef.data(), B.e.ptr, 4 * (size_t)n, cudaMemcpyDeviceToHost, ctx->stream));
    TGAP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    for (int64_t i = 0; i < n; ++i) e[i] = ef[i];
    return read_device_check(ctx);
}
