// GAP kernel contraction, FP64 ("plain") path, and the force kernels of the reference
// get_soap_energy_and_forces surface (src/gap/gap.f90:39-244).
//
//   K = q Qs^T                      (gap.f90:123, dgemm "t","n")
//   E_i = delta^2 sum_s alpha_s K_is^zeta + e0           (:128-135)
//   g_i = dE_i/dq_i = zeta delta^2 sum_s alpha_s K_is^(zeta-1) Qs_s = -Qss_i   (:153-171)
//
// The first GEMM's epilogue evaluates K^zeta, the energy row partials and the scaled
// derivative matrix G = zeta delta^2 alpha o K^(zeta-1), which is the A operand of the
// second GEMM g = G Qs. Both are "NT" products (row-major operands, K contiguous).
#include <cmath>
#include <mutex>

#include "gap_kernels.h"

namespace tgap {

constexpr int kBM = 64, kBN = 64, kBK = 16, kGemmThreads = 256;

struct EpiStore {
    double *C;
    int ldc;
    double alpha;
    __device__ void operator()(int m, int n, int M, int N, const double acc[4][4], int ty, int tx,
                               int tile_n) const
    {
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int r = m + ty + 16 * i;
            if (r >= M) continue;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int c = n + tx + 16 * j;
                if (c < N) C[(size_t)r * ldc + c] = alpha * acc[i][j];
            }
        }
    }
};

struct EpiGap {
    const double *alphas;
    double *G;       // [M][ldg] zeta delta^2 alpha_s K^(zeta-1), or null
    int ldg;
    double *e_part;  // [n_tiles][M] sum_s alpha_s K^zeta over the tile's columns
    double zeta, zd2;
    int zeta_int;    // >= 0: integer power
    __device__ static double powi(double x, int n)
    {
        double r = 1.0;
        for (int i = 0; i < n; ++i) r *= x;
        return r;
    }
    __device__ void operator()(int m, int n, int M, int N, const double acc[4][4], int ty, int tx,
                               int tile_n) const
    {
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int r = m + ty + 16 * i;
            double e = 0.0;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int c = n + tx + 16 * j;
                if (r < M && c < N) {
                    const double k = acc[i][j];
                    const double a = alphas[c];
                    double kz, kz1;
                    if (zeta_int >= 0) {
                        kz1 = zeta_int >= 1 ? powi(k, zeta_int - 1) : 0.0;
                        kz = zeta_int >= 1 ? kz1 * k : 1.0;
                    } else {
                        kz = pow(k, zeta);
                        kz1 = pow(k, zeta - 1.0);
                    }
                    e += kz * a;
                    if (G) G[(size_t)r * ldg + c] = zd2 * a * kz1;
                }
            }
            // reduce over the 16 threads of this row (tx = lane & 15)
#pragma unroll
            for (int o = 8; o > 0; o >>= 1) e += __shfl_xor_sync(0xffffffffu, e, o);
            if (tx == 0 && r < M) e_part[(size_t)tile_n * M + r] = e;
        }
    }
};

template <class Epi>
__global__ void __launch_bounds__(kGemmThreads) k_dgemm_nt(int M, int N, int K, const double *__restrict__ A,
                                                           int lda, const double *__restrict__ B,
                                                           int ldb, Epi epi)
{
    __shared__ double As[2][kBK][kBM + 1];
    __shared__ double Bs[2][kBK][kBN + 1];
    const int t = threadIdx.x, ty = t >> 4, tx = t & 15;
    const int m0 = blockIdx.y * kBM, n0 = blockIdx.x * kBN;
    // loader mapping: 64 rows x 16 k = 1024 elements, 4 per thread (one row, 4 consecutive k)
    const int lr = t >> 2, lk = (t & 3) * 4;
    double acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = 0.0;
    double ra[4], rb[4];
    auto load = [&](int k0) {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int kk = k0 + lk + q;
            const int ar = m0 + lr, br = n0 + lr;
            ra[q] = (ar < M && kk < K) ? A[(size_t)ar * lda + kk] : 0.0;
            rb[q] = (br < N && kk < K) ? B[(size_t)br * ldb + kk] : 0.0;
        }
    };
    auto store = [&](int buf) {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            As[buf][lk + q][lr] = ra[q];
            Bs[buf][lk + q][lr] = rb[q];
        }
    };
    const int nk = (K + kBK - 1) / kBK;
    load(0);
    store(0);
    __syncthreads();
    for (int kt = 0; kt < nk; ++kt) {
        const int buf = kt & 1;
        if (kt + 1 < nk) load((kt + 1) * kBK);
#pragma unroll
        for (int kk = 0; kk < kBK; ++kk) {
            double a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) a[i] = As[buf][kk][ty + 16 * i];
#pragma unroll
            for (int j = 0; j < 4; ++j) b[j] = Bs[buf][kk][tx + 16 * j];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
        }
        if (kt + 1 < nk) store(buf ^ 1);
        __syncthreads();
    }
    epi(m0, n0, M, N, acc, ty, tx, blockIdx.x);
}

int dgemm_nt(tgap_context *ctx, int M, int N, int K, const double *A, int lda, const double *B,
             int ldb, double *C, int ldc, double alpha)
{
    if (M <= 0 || N <= 0) return TGAP_OK;
    StageScope sc(ctx, "dgemm_f64");
    dim3 grid((N + kBN - 1) / kBN, (M + kBM - 1) / kBM);
    EpiStore e{C, ldc, alpha};
    k_dgemm_nt<EpiStore><<<grid, kGemmThreads, 0, ctx->stream>>>(M, N, K, A, lda, B, ldb, e);
    TGAP_LAUNCH_CHECK(ctx);
    return TGAP_OK;
}

// e_row = delta^2 sum_tiles e_part + e0, added into energies[sites[row]] (or written when
// overwrite != 0).
__global__ void k_energy_reduce(int M, int n_tiles, const double *__restrict__ e_part, double d2,
                                double e0, const int *__restrict__ sites, double *__restrict__ e_rows,
                                double *__restrict__ energies)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= M) return;
    double s = 0.0;
    for (int t = 0; t < n_tiles; ++t) s += e_part[(size_t)t * M + r];
    const double e = d2 * s + e0;
    if (e_rows) e_rows[r] = e;
    if (energies) energies[sites ? sites[r] : r] += e;
}

int gap_energy_grad_f64(tgap_context *ctx, const DeviceModel &m, const double *d_q, int q_ld,
                        int n_rows, double e0, int do_forces, GapWork *w, const int *d_sites,
                        double *d_e_rows, double *d_energies)
{
    if (n_rows <= 0) return TGAP_OK;
    const int M = n_rows, N = m.n_sparse, K = m.dim;
    const int n_tiles = (N + kBN - 1) / kBN;
    if (w->e_part.ensure(sizeof(double) * (size_t)n_tiles * M) ||
        (do_forces && (w->G.ensure(sizeof(double) * (size_t)M * N) ||
                       w->g.ensure(sizeof(double) * (size_t)M * K))))
        return set_error(ctx, TGAP_ERR_NOMEM, "GAP workspace");
    EpiGap e;
    e.alphas = m.alphas.as<double>();
    e.G = do_forces ? w->G.as<double>() : nullptr;
    e.ldg = N;
    e.e_part = w->e_part.as<double>();
    const double zr = m.zeta_nint ? std::nearbyint(m.zeta) : (double)(int)m.zeta;
    const bool zi = std::fabs(m.zeta - zr) < m.zeta_tol;  // gap.f90:99-105 (local properties: :76-77)
    e.zeta_int = zi ? (int)zr : -1;
    e.zeta = zi ? zr : m.zeta;
    e.zd2 = e.zeta * m.delta * m.delta;
    dim3 grid(n_tiles, (M + kBM - 1) / kBM);
    StageScope sc(ctx, "dgemm_gap_kernel_f64");
    k_dgemm_nt<EpiGap><<<grid, kGemmThreads, 0, ctx->stream>>>(M, N, K, d_q, q_ld, m.Qs.as<double>(),
                                                               m.dim, e);
    TGAP_LAUNCH_CHECK(ctx);
    k_energy_reduce<<<(M + 127) / 128, 128, 0, ctx->stream>>>(M, n_tiles, w->e_part.as<double>(),
                                                              m.delta * m.delta, e0, d_sites,
                                                              d_e_rows, d_energies);
    TGAP_LAUNCH_CHECK(ctx);
    if (do_forces) {
        // g = G Qs  (A = G [M][N], B = Qs^T [K][N])
        int rc = dgemm_nt(ctx, M, K, N, w->G.as<double>(), N, m.QsT.as<double>(), N,
                          w->g.as<double>(), K, 1.0);
        if (rc) return rc;
    }
    return TGAP_OK;
}

// local_properties.f90:117-122: every V >= 0.
__global__ void k_clip_nonneg(int n, double *__restrict__ v)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && v[i] < 0.0) v[i] = 0.0;
}

int clip_nonneg(tgap_context *ctx, int n, double *d_v)
{
    if (n <= 0) return TGAP_OK;
    k_clip_nonneg<<<(n + 255) / 256, 256, 0, ctx->stream>>>(n, d_v);
    TGAP_LAUNCH_CHECK(ctx);
    return TGAP_OK;
}

// local_properties.f90:124-142 over a materialised soap_cart_der: one warp per site, V_der(:, j)
// = g_i . der(:, :, j) for each of its pairs (lanes over the descriptor, fixed reduction order),
// zero when V_i was clipped to 0.
__global__ void k_local_property_pairs(int n_sites, const int64_t *__restrict__ start, const double *__restrict__ g,
                                       int D, const double *__restrict__ der, const double *__restrict__ V,
                                       double *__restrict__ V_der)
{
    const int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (i >= n_sites) return;
    const double *gi = g + (size_t)i * D;
    const bool zero = V[i] == 0.0;
    for (int64_t j = start[i]; j < start[i + 1]; ++j) {
        double a0 = 0.0, a1 = 0.0, a2 = 0.0;
        if (!zero) {
            const double *dj = der + (size_t)j * 3 * D;
            for (int d = lane; d < D; d += 32) {
                const double gd = gi[d];
                a0 += gd * dj[3 * d];
                a1 += gd * dj[3 * d + 1];
                a2 += gd * dj[3 * d + 2];
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                a0 += __shfl_xor_sync(0xffffffffu, a0, o);
                a1 += __shfl_xor_sync(0xffffffffu, a1, o);
                a2 += __shfl_xor_sync(0xffffffffu, a2, o);
            }
        }
        if (lane == 0) {
            V_der[3 * j] = a0;
            V_der[3 * j + 1] = a1;
            V_der[3 * j + 2] = a2;
        }
    }
}

int local_property_pairs(tgap_context *ctx, int n_sites, const int64_t *d_start, const double *d_g, int D,
                         const double *d_der, const double *d_V, double *d_V_der)
{
    if (n_sites <= 0) return TGAP_OK;
    k_local_property_pairs<<<(n_sites + 3) / 4, 128, 0, ctx->stream>>>(n_sites, d_start, d_g, D, d_der, d_V, d_V_der);
    TGAP_LAUNCH_CHECK(ctx);
    return TGAP_OK;
}

// Reference pair loop (gap.f90:187-209) over a materialised soap_der: one warp per pair.
// Qss = -g. forces: 3 x n_sites0 (fold modulus), virial column-major 3x3.
__global__ void k_pair_forces_from_der(int n_sites, const int64_t *__restrict__ start,
                                       const int *__restrict__ nl, int n_sites0,
                                       const double *__restrict__ g, int D,
                                       const double *__restrict__ der, const double *__restrict__ xyz,
                                       double *__restrict__ forces, double *__restrict__ virial)
{
    const int i = blockIdx.x;
    if (i >= n_sites) return;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const double *gi = g + (size_t)i * D;
    double v[6] = {0, 0, 0, 0, 0, 0};
    for (int64_t l = start[i] + wid; l < start[i + 1]; l += nw) {
        const double *dl = der + (size_t)l * D * 3;
        double f0 = 0, f1 = 0, f2 = 0;
        for (int d = lane; d < D; d += 32) {
            const double q = -gi[d];
            f0 += q * dl[3 * d];
            f1 += q * dl[3 * d + 1];
            f2 += q * dl[3 * d + 2];
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            f0 += __shfl_xor_sync(0xffffffffu, f0, o);
            f1 += __shfl_xor_sync(0xffffffffu, f1, o);
            f2 += __shfl_xor_sync(0xffffffffu, f2, o);
        }
        if (lane == 0) {
            const int j2 = (nl[l] - 1) % n_sites0;
            atomicAdd(forces + 3 * (size_t)j2, f0);
            atomicAdd(forces + 3 * (size_t)j2 + 1, f1);
            atomicAdd(forces + 3 * (size_t)j2 + 2, f2);
            const double x0 = xyz[3 * l], x1 = xyz[3 * l + 1], x2 = xyz[3 * l + 2];
            v[0] += f0 * x0;
            v[1] += f1 * x1;
            v[2] += f2 * x2;
            v[3] += 0.5 * (f0 * x1 + f1 * x0);
            v[4] += 0.5 * (f0 * x2 + f2 * x0);
            v[5] += 0.5 * (f1 * x2 + f2 * x1);
        }
    }
    if (lane == 0) {
        const int idx[6][2] = {{0, 0}, {1, 1}, {2, 2}, {0, 1}, {0, 2}, {1, 2}};
        for (int c = 0; c < 6; ++c) {
            if (v[c] == 0.0) continue;
            const int a = idx[c][0], b = idx[c][1];
            atomicAdd(virial + a + 3 * b, v[c]);
            if (a != b) atomicAdd(virial + b + 3 * a, v[c]);
        }
    }
}

int pair_forces_from_der(tgap_context *ctx, int n_sites, const int64_t *d_start, const int *d_nl,
                         int n_sites0, const double *d_g, int D, const double *d_der,
                         const double *d_xyz, double *d_forces, double *d_virial)
{
    if (n_sites <= 0) return TGAP_OK;
    StageScope sc(ctx, "pair_forces_from_der");
    k_pair_forces_from_der<<<n_sites, 256, 0, ctx->stream>>>(n_sites, d_start, d_nl, n_sites0, d_g, D,
                                                             d_der, d_xyz, d_forces, d_virial);
    TGAP_LAUNCH_CHECK(ctx);
    return TGAP_OK;
}

// ----------------------------------------------------------------------------- no-allocation entry

// Scratch of tgap_soap_energies_noalloc: the per-tile energy partials of the K = q Qs^T
// product, one double per (64-column tile of sparse points, site). 2^20 doubles (8 MiB) are
// reserved on every GPU that loads the library, for the lifetime of the process.
constexpr size_t kNoAllocPartials = (size_t)1 << 20;
static __device__ __align__(256) double g_noalloc_e_part[kNoAllocPartials];

// Device address of the scratch array, looked up once per device (the symbol name is only a
// host-side handle; kernels must be given the address cudaGetSymbolAddress returns).
static int noalloc_scratch(double **out)
{
    static std::mutex mu;
    static double *addr[64] = {nullptr};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return TGAP_ERR_CUDA;
    std::lock_guard<std::mutex> lock(mu);
    if (!addr[dev]) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_e_part) != cudaSuccess || !p) return TGAP_ERR_CUDA;
        addr[dev] = static_cast<double *>(p);
    }
    *out = addr[dev];
    return TGAP_OK;
}

}  // namespace tgap

// Energies of get_soap_energy_and_forces with do_forces = .false. for device-resident inputs,
// with no device allocation (declaration and contract in include/tgap.h).
extern "C" int tgap_soap_energies_noalloc(void *stream, int n_soap, int n_sites, int n_sparse,
                                          const double *d_soap, const double *d_alphas, double delta,
                                          double zeta0, double e0, const double *d_Qs,
                                          double *d_energies)
{
    using namespace tgap;
    if (n_soap <= 0 || n_sites <= 0 || n_sparse <= 0 || !d_soap || !d_alphas || !d_Qs || !d_energies)
        return TGAP_ERR_ARGUMENT;
    const int n_tiles = (n_sparse + kBN - 1) / kBN;
    if ((size_t)n_tiles * (size_t)n_sites > kNoAllocPartials) return TGAP_ERR_CAPACITY;
    double *e_part = nullptr;
    int rc = noalloc_scratch(&e_part);
    if (rc) return rc;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    EpiGap e;
    e.alphas = d_alphas;
    e.G = nullptr;
    e.ldg = n_sparse;
    e.e_part = e_part;  // every (tile, site) entry is written before it is read
    const bool zi = std::fabs(zeta0 - (double)(int)zeta0) < 1.0e-5;  // gap.f90:99-105
    e.zeta_int = zi ? (int)zeta0 : -1;
    e.zeta = zi ? (double)(int)zeta0 : zeta0;
    e.zd2 = e.zeta * delta * delta;
    dim3 grid(n_tiles, (n_sites + kBM - 1) / kBM);
    k_dgemm_nt<EpiGap><<<grid, kGemmThreads, 0, s>>>(n_sites, n_sparse, n_soap, d_soap, n_soap, d_Qs, n_soap, e);
    k_energy_reduce<<<(n_sites + 127) / 128, 128, 0, s>>>(n_sites, n_tiles, e_part, delta * delta, e0, nullptr,
                                                          d_energies, nullptr);
    return cudaGetLastError() == cudaSuccess ? TGAP_OK : TGAP_ERR_CUDA;
}

namespace tgap {

__global__ void k_transpose(int R, int Cc, const double *__restrict__ in, double *__restrict__ out)
{
    __shared__ double tile[32][33];
    const int bx = blockIdx.x * 32, by = blockIdx.y * 32;
    for (int y = threadIdx.y; y < 32; y += blockDim.y) {
        const int r = by + y, c = bx + threadIdx.x;
        if (r < R && c < Cc) tile[y][threadIdx.x] = in[(size_t)r * Cc + c];
    }
    __syncthreads();
    for (int y = threadIdx.y; y < 32; y += blockDim.y) {
        const int c = bx + y, r = by + threadIdx.x;
        if (r < R && c < Cc) out[(size_t)c * R + r] = tile[threadIdx.x][y];
    }
}

int transpose_f64(tgap_context *ctx, int R, int Cc, const double *in, double *out)
{
    dim3 grid((Cc + 31) / 32, (R + 31) / 32), block(32, 8);
    k_transpose<<<grid, block, 0, ctx->stream>>>(R, Cc, in, out);
    TGAP_LAUNCH_CHECK(ctx);
    return TGAP_OK;
}

}  // namespace tgap
