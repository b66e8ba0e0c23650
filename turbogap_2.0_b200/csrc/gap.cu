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

#include "gap_kernels.h"

namespace tgap {

// ---------------------------------------------------------------------------- FP64 GEMM
//
// C = A B^T for row-major A [M][K] and B [N][K] (K contiguous, the "NT" form of both GAP
// products), on the FP64 tensor-core path: mma.sync m16n8k4 .f64 (DMMA). A CTA of WM x WN warps
// owns a BM x BN tile; k-tiles of 16 doubles stream through a STAGES-deep cp.async ring in shared
// memory, each operand row (one tile row, 16 doubles) padded to a 20-double pitch so the fragment
// loads of a warp (rows g = lane / 4, column t = lane % 4) fall into distinct banks per half warp.
// Fragment layout of m16n8k4 .f64: a0 = A[g][t], a1 = A[g + 8][t], b0 = B[t][g] (B col-major =
// our B rows), c0/c1 = C[g][2t, 2t + 1], c2/c3 = C[g + 8][2t, 2t + 1]. Accumulation is FP64
// throughout, in a fixed order (k ascending), so every launch is bitwise reproducible.
constexpr int kDK = 16;       // doubles per k-tile (128 bytes per operand row)
constexpr int kDPitch = 20;   // shared-memory row pitch in doubles
constexpr int kDStages = 3;

template <int BM, int BN> struct DgemmSmem {
    static constexpr size_t stage = (size_t)(BM + BN) * kDPitch * 8;
    static constexpr size_t bytes = kDStages * stage;
};

__device__ __forceinline__ void cp_async16(uint32_t dst, const void *src, int src_bytes)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(src_bytes) : "memory");
}

__device__ __forceinline__ void cp_async8(uint32_t dst, const void *src, int src_bytes)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(dst), "l"(src), "r"(src_bytes) : "memory");
}

__device__ __forceinline__ void dmma_16x8x4(double c[4], double a0, double a1, double b0)
{
    asm volatile("mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};"
                 : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
                 : "d"(a0), "d"(a1), "d"(b0));
}

// Stores alpha * C (rows < M, columns < N).
struct EpiStore {
    double *C;
    int ldc;
    double alpha;
    static constexpr bool kRowSum = false;
    __device__ __forceinline__ double element(int r, int c, double v) const
    {
        C[(size_t)r * ldc + c] = alpha * v;
        return 0.0;
    }
    __device__ __forceinline__ void row_sum(int, int, double) const {}
};

// GEMM1 epilogue of the GAP contraction: per element k = K[row][s], G = zeta delta^2 alpha_s
// k^(zeta-1) (the A operand of g = G Qs, gap.f90:153-171) and the energy row partial
// sum_s alpha_s k^zeta over the tile's columns (gap.f90:128-135), one per (column tile, row).
struct EpiGap {
    const double *alphas;
    double *G;       // [M][ldg] zeta delta^2 alpha_s K^(zeta-1), or null
    int ldg;
    double *e_part;  // [n_tiles][M] sum_s alpha_s K^zeta over the tile's columns
    int M;
    double zeta, zd2;
    int zeta_int;    // >= 0: integer power
    static constexpr bool kRowSum = true;
    __device__ static double powi(double x, int n)
    {
        double r = 1.0;
        for (int i = 0; i < n; ++i) r *= x;
        return r;
    }
    __device__ __forceinline__ double element(int r, int c, double k) const
    {
        const double a = alphas[c];
        double kz, kz1;
        if (zeta_int >= 0) {
            kz1 = zeta_int >= 1 ? powi(k, zeta_int - 1) : 0.0;
            kz = zeta_int >= 1 ? kz1 * k : 1.0;
        } else {
            kz = pow(k, zeta);
            kz1 = pow(k, zeta - 1.0);
        }
        if (G) G[(size_t)r * ldg + c] = zd2 * a * kz1;
        return kz * a;
    }
    __device__ __forceinline__ void row_sum(int r, int tile_n, double e) const
    {
        e_part[(size_t)tile_n * M + r] = e;
    }
};

template <int BM, int BN, int WM, int WN, class Epi>
__global__ void __launch_bounds__(WM * WN * 32)
    k_dgemm_tc(int M, int N, int K, const double *__restrict__ A, int lda, const double *__restrict__ B, int ldb,
               int vec16, Epi epi)
{
    constexpr int T = WM * WN * 32;
    constexpr int TM = BM / WM, TN = BN / WN, MI = TM / 16, NI = TN / 8;
    static_assert(TM % 16 == 0 && TN % 8 == 0, "warp tile: 16 x 8 fragments");
    extern __shared__ __align__(16) double dsm[];
    const uint32_t sbase = (uint32_t)__cvta_generic_to_shared(dsm);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int wm = warp / WN, wn = warp % WN, g = lane >> 2, t = lane & 3;
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
    const int nk = (K + kDK - 1) / kDK;

    // one k-tile of A (BM rows) and B (BN rows) into stage s; rows and columns past the matrix
    // are zero-filled (the source address is clamped to row 0 and copies no bytes)
    auto load = [&](int kt, int s) {
        const int k0 = kt * kDK;
        const uint32_t st = sbase + (uint32_t)(s * DgemmSmem<BM, BN>::stage);
        if (vec16) {
            for (int i = tid; i < (BM + BN) * (kDK / 2); i += T) {
                const int row = i / (kDK / 2), ch = i % (kDK / 2);
                const bool isA = row < BM;
                const int rr = isA ? m0 + row : n0 + row - BM;
                const int lim = isA ? M : N;
                const int k = k0 + 2 * ch;
                const int nb = (rr < lim && k < K) ? (K - k >= 2 ? 16 : 8) : 0;
                const double *src = isA ? A + (size_t)(nb ? rr : 0) * lda + (nb ? k : 0)
                                        : B + (size_t)(nb ? rr : 0) * ldb + (nb ? k : 0);
                cp_async16(st + (uint32_t)((row * kDPitch + 2 * ch) * 8), src, nb);
            }
        } else {
            for (int i = tid; i < (BM + BN) * kDK; i += T) {
                const int row = i / kDK, kk = i % kDK;
                const bool isA = row < BM;
                const int rr = isA ? m0 + row : n0 + row - BM;
                const int lim = isA ? M : N;
                const int k = k0 + kk;
                const int nb = (rr < lim && k < K) ? 8 : 0;
                const double *src = isA ? A + (size_t)(nb ? rr : 0) * lda + (nb ? k : 0)
                                        : B + (size_t)(nb ? rr : 0) * ldb + (nb ? k : 0);
                cp_async8(st + (uint32_t)((row * kDPitch + kk) * 8), src, nb);
            }
        }
    };

    double acc[MI][NI][4];
#pragma unroll
    for (int i = 0; i < MI; ++i)
#pragma unroll
        for (int j = 0; j < NI; ++j)
#pragma unroll
            for (int e = 0; e < 4; ++e) acc[i][j][e] = 0.0;

#pragma unroll
    for (int s = 0; s < kDStages - 1; ++s) {
        if (s < nk) load(s, s);
        asm volatile("cp.async.commit_group;" ::: "memory");
    }
    for (int kt = 0; kt < nk; ++kt) {
        asm volatile("cp.async.wait_group %0;" ::"n"(kDStages - 2) : "memory");
        __syncthreads();  // stage kt landed for every thread; stage kt - 1 is free again
        if (kt + kDStages - 1 < nk) load(kt + kDStages - 1, (kt + kDStages - 1) % kDStages);
        asm volatile("cp.async.commit_group;" ::: "memory");
        const double *sA = dsm + (size_t)(kt % kDStages) * ((BM + BN) * kDPitch);
        const double *sB = sA + BM * kDPitch;
#pragma unroll
        for (int k4 = 0; k4 < kDK; k4 += 4) {
            double a[MI][2], b[NI];
#pragma unroll
            for (int i = 0; i < MI; ++i) {
                const int r = wm * TM + 16 * i + g;
                a[i][0] = sA[r * kDPitch + k4 + t];
                a[i][1] = sA[(r + 8) * kDPitch + k4 + t];
            }
#pragma unroll
            for (int j = 0; j < NI; ++j) b[j] = sB[(wn * TN + 8 * j + g) * kDPitch + k4 + t];
#pragma unroll
            for (int i = 0; i < MI; ++i)
#pragma unroll
                for (int j = 0; j < NI; ++j) dmma_16x8x4(acc[i][j], a[i][0], a[i][1], b[j]);
        }
    }
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    __syncthreads();  // the ring is free: the row reduction below reuses it

    double rs[MI][2];
#pragma unroll
    for (int i = 0; i < MI; ++i) {
        rs[i][0] = rs[i][1] = 0.0;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int r = m0 + wm * TM + 16 * i + 8 * h + g;
#pragma unroll
            for (int j = 0; j < NI; ++j) {
                const int c = n0 + wn * TN + 8 * j + 2 * t;
                if (r < M) {
                    if (c < N) rs[i][h] += epi.element(r, c, acc[i][j][2 * h]);
                    if (c + 1 < N) rs[i][h] += epi.element(r, c + 1, acc[i][j][2 * h + 1]);
                }
            }
        }
    }
    if constexpr (Epi::kRowSum) {
        // the four lanes of a row (t = 0..3), then the WN warps of a row band in warp order
        double *red = dsm;  // [WN][BM]
#pragma unroll
        for (int i = 0; i < MI; ++i)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                double v = rs[i][h];
                v += __shfl_xor_sync(0xffffffffu, v, 1);
                v += __shfl_xor_sync(0xffffffffu, v, 2);
                if (t == 0) red[wn * BM + wm * TM + 16 * i + 8 * h + g] = v;
            }
        __syncthreads();
        for (int r = tid; r < BM; r += T) {
            double s = 0.0;
#pragma unroll
            for (int w = 0; w < WN; ++w) s += red[w * BM + r];
            if (m0 + r < M) epi.row_sum(m0 + r, blockIdx.x, s);
        }
    }
}

// Tile shape by problem size: 128 x 64 tiles (8 warps of 32 x 32, two CTAs per SM) when there are
// enough of them to fill the GPU twice over (measured 30 % faster than 128 x 128 tiles with one
// CTA per SM on the 4096 x 2000 x 324 energy product), else 64 x 64 (4 warps of 32 x 32), which
// gives small products (Monte Carlo rows, narrow descriptor products) twice the CTAs.
static bool dgemm_big(int M, int N) { return (long)((M + 127) / 128) * ((N + 63) / 64) >= 592; }
static int dgemm_bn(int, int) { return 64; }

static int dgemm_vec16(const double *A, int lda, const double *B, int ldb)
{
    return ((uintptr_t)A % 16 == 0 && (uintptr_t)B % 16 == 0 && lda % 2 == 0 && ldb % 2 == 0) ? 1 : 0;
}

template <class Epi>
static cudaError_t dgemm_launch(int M, int N, int K, const double *A, int lda, const double *B, int ldb,
                                const Epi &epi, cudaStream_t stream)
{
    const int v16 = dgemm_vec16(A, lda, B, ldb);
    if (dgemm_big(M, N)) {
        auto kern = k_dgemm_tc<128, 64, 4, 2, Epi>;
        constexpr size_t smem = DgemmSmem<128, 64>::bytes;
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        dim3 grid((N + 63) / 64, (M + 127) / 128);
        void *args[] = {&M, &N, &K, &A, &lda, &B, &ldb, const_cast<int *>(&v16), const_cast<Epi *>(&epi)};
        return cudaLaunchKernel((const void *)kern, grid, dim3(256), args, smem, stream);
    }
    auto kern = k_dgemm_tc<64, 64, 2, 2, Epi>;
    constexpr size_t smem = DgemmSmem<64, 64>::bytes;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    dim3 grid((N + 63) / 64, (M + 63) / 64);
    void *args[] = {&M, &N, &K, &A, &lda, &B, &ldb, const_cast<int *>(&v16), const_cast<Epi *>(&epi)};
    return cudaLaunchKernel((const void *)kern, grid, dim3(128), args, smem, stream);
}

int dgemm_nt(tgap_context *ctx, int M, int N, int K, const double *A, int lda, const double *B,
             int ldb, double *C, int ldc, double alpha)
{
    if (M <= 0 || N <= 0) return TGAP_OK;
    StageScope sc(ctx, "dgemm_f64");
    EpiStore e{C, ldc, alpha};
    TGAP_CUDA(ctx, dgemm_launch(M, N, K, A, lda, B, ldb, e, ctx->stream));
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
    const int bn = dgemm_bn(M, N);
    const int n_tiles = (N + bn - 1) / bn;
    if (w->e_part.ensure(sizeof(double) * (size_t)n_tiles * M) ||
        (do_forces && (w->G.ensure(sizeof(double) * (size_t)M * N) ||
                       w->g.ensure(sizeof(double) * (size_t)M * K))))
        return set_error(ctx, TGAP_ERR_NOMEM, "GAP workspace");
    EpiGap e;
    e.alphas = m.alphas.as<double>();
    e.G = do_forces ? w->G.as<double>() : nullptr;
    e.ldg = N;
    e.e_part = w->e_part.as<double>();
    e.M = M;
    const double zr = m.zeta_nint ? std::nearbyint(m.zeta) : (double)(int)m.zeta;
    const bool zi = std::fabs(m.zeta - zr) < m.zeta_tol;  // gap.f90:99-105 (local properties: :76-77)
    e.zeta_int = zi ? (int)zr : -1;
    e.zeta = zi ? zr : m.zeta;
    e.zd2 = e.zeta * m.delta * m.delta;
    {
        StageScope sc(ctx, "dgemm_gap_kernel_f64");
        TGAP_CUDA(ctx, dgemm_launch(M, N, K, d_q, q_ld, m.Qs.as<double>(), m.dim, e, ctx->stream));
        TGAP_LAUNCH_CHECK(ctx);
    }
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
// product, one double per (column tile of sparse points, site); the FP64 GEMM's tiles are 64 or
// 128 sparse points wide, so n_sites * ceil(n_sparse / 64) partials always suffice. 2^20 doubles
// (8 MiB) are reserved on every GPU that loads the library, for the lifetime of the process.
constexpr size_t kNoAllocPartials = (size_t)1 << 20;
static __device__ __align__(256) double g_noalloc_e_part[kNoAllocPartials];

// Device address of the scratch array on the current device `dev` (the symbol name is only a
// host-side handle; kernels must be given the address cudaGetSymbolAddress returns). Looked up on
// every call: the lookup allocates nothing, and a cached address would outlive a cudaDeviceReset.
static int noalloc_scratch(int dev, double **out)
{
    if (dev < 0) return TGAP_ERR_CUDA;
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_e_part);
    if (e != cudaSuccess || !p) {
        if (e != cudaSuccess) cudaGetLastError();  // this call's own error, reported below
        return thread_error(TGAP_ERR_CUDA, "tgap_soap_energies_noalloc: cudaGetSymbolAddress: %s",
                            cudaGetErrorString(e));
    }
    *out = static_cast<double *>(p);
    return TGAP_OK;
}

}  // namespace tgap

// Energies of get_soap_energy_and_forces with do_forces = .false. for device-resident inputs,
// with no device allocation (declaration and contract in include/tgap.h). Errors carry a message
// for tgap_last_error(NULL). The status reflects this call's own launches only: they are issued
// with cudaLaunchKernel, whose return value belongs to that launch, so an error left pending by
// the caller's earlier work is neither reported as this call's failure nor cleared.
extern "C" int tgap_soap_energies_noalloc(void *stream, int n_soap, int n_sites, int n_sparse,
                                          const double *d_soap, const double *d_alphas, double delta,
                                          double zeta0, double e0, const double *d_Qs,
                                          double *d_energies)
{
    using namespace tgap;
    if (n_soap <= 0 || n_sites <= 0 || n_sparse <= 0 || !d_soap || !d_alphas || !d_Qs || !d_energies)
        return thread_error(TGAP_ERR_ARGUMENT, "tgap_soap_energies_noalloc: bad arguments");
    const size_t n_tiles64 = ((size_t)n_sparse + 63) / 64;
    if (n_tiles64 * (size_t)n_sites > kNoAllocPartials)
        return thread_error(TGAP_ERR_CAPACITY,
                            "tgap_soap_energies_noalloc: n_sites * ceil(n_sparse / 64) = %zu exceeds %zu",
                            n_tiles64 * (size_t)n_sites, kNoAllocPartials);
    int dev = 0;
    cudaError_t ce = cudaGetDevice(&dev);
    if (ce != cudaSuccess) {
        cudaGetLastError();
        return thread_error(TGAP_ERR_CUDA, "tgap_soap_energies_noalloc: cudaGetDevice: %s", cudaGetErrorString(ce));
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (s && s != cudaStreamLegacy && s != cudaStreamPerThread) {
        int sdev = -1;
        ce = cudaStreamGetDevice(s, &sdev);
        if (ce != cudaSuccess) {
            cudaGetLastError();
            return thread_error(TGAP_ERR_ARGUMENT, "tgap_soap_energies_noalloc: stream: %s", cudaGetErrorString(ce));
        }
        if (sdev != dev)
            return thread_error(TGAP_ERR_ARGUMENT,
                                "tgap_soap_energies_noalloc: the stream belongs to device %d, device %d is current",
                                sdev, dev);
    }
    double *e_part = nullptr;
    int rc = noalloc_scratch(dev, &e_part);
    if (rc) return rc;
    const int bn = dgemm_bn(n_sites, n_sparse);
    int n_tiles = (n_sparse + bn - 1) / bn;
    EpiGap e;
    e.alphas = d_alphas;
    e.G = nullptr;
    e.ldg = n_sparse;
    e.e_part = e_part;  // every (tile, site) entry is written before it is read
    e.M = n_sites;
    const bool zi = std::fabs(zeta0 - (double)(int)zeta0) < 1.0e-5;  // gap.f90:99-105
    e.zeta_int = zi ? (int)zeta0 : -1;
    e.zeta = zi ? (double)(int)zeta0 : zeta0;
    e.zd2 = e.zeta * delta * delta;
    ce = dgemm_launch(n_sites, n_sparse, n_soap, d_soap, n_soap, d_Qs, n_soap, e, s);
    if (ce == cudaSuccess) {
        double d2 = delta * delta;
        const int *no_sites = nullptr;
        double *no_energies = nullptr;
        void *args[] = {&n_sites, &n_tiles, &e_part, &d2, &e0, &no_sites, &d_energies, &no_energies};
        ce = cudaLaunchKernel((const void *)k_energy_reduce, dim3((n_sites + 127) / 128), dim3(128), args, 0, s);
    }
    if (ce != cudaSuccess) {
        cudaGetLastError();  // the error of this call's own launch
        return thread_error(TGAP_ERR_CUDA, "tgap_soap_energies_noalloc: kernel launch: %s", cudaGetErrorString(ce));
    }
    return TGAP_OK;
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
