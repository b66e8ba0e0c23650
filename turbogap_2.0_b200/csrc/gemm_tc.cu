// Mixed-precision GAP kernel contraction on the 5th-generation tensor cores (sm_100a).
//
// bf16x3 split products: every FP32 operand x is stored as x_hi = bf16(x) and
// x_lo = bf16(x - x_hi); a product is accumulated as a_hi b_hi + a_hi b_lo + a_lo b_hi in
// FP32 (the a_lo b_lo term is below the FP32 accumulation error). Two GEMMs per model:
//
//   GEMM1  K = q Qs^T       (rows x n_sparse, K-dim = descriptor)   epilogue: K^zeta energy
//          partials and G = zeta delta^2 alpha o K^(zeta-1), written back as a bf16 split
//   GEMM2  g = G Qs         (rows x descriptor, K-dim = n_sparse)   epilogue: FP32 store
//
// For descriptor widths up to 384 both are fused into k_gap_flash (G stays on the SM).
//
// Persistent kernel, one CTA per SM over 128 x BN tiles: one thread issues TMA loads (no
// multicast) into a STAGES-deep ring of 128B-swizzled shared-memory tiles, one thread issues
// tcgen05.mma (cta_group::1, kind::f16) into one of two TMEM accumulator buffers, and eight
// epilogue warps drain the other buffer with tcgen05.ld. Every mbarrier wait is bounded (1 s of
// globaltimer); on timeout the kernel raises the device error flag, waits (bounded) for its
// own copies and MMAs in flight, frees TMEM and returns.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>

#include "gap_kernels.h"

namespace tgap {

constexpr int kBM = 128;
constexpr int kBK = 64;  // bf16 elements per 128-byte swizzle row
constexpr uint64_t kWaitNs = 1000000000ull;

// ---------------------------------------------------------------------------- PTX helpers

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ uint64_t globaltimer()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait: false after kWaitNs or once *abort is set by another thread of the CTA. The timer
// and the abort flag are read only when the phase has not completed on the first tries (every 8th
// try after that), so a wait that succeeds at once costs one try_wait and no %globaltimer read.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, volatile int *abort)
{
    if (mbar_try(bar, parity)) return true;
    const uint64_t t0 = globaltimer();
    for (unsigned i = 0;; ++i) {
        if (mbar_try(bar, parity)) return true;
        if ((i & 7u) == 7u) {
            if (*abort) return false;
            if (globaltimer() - t0 > kWaitNs) return false;
        }
    }
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap *map, uint32_t bar, int x,
                                            int y)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];"
        ::"r"(dst), "l"((uint64_t)map), "r"(bar), "r"(x), "r"(y)
        : "memory");
}

// K-major operand tile, 128-byte swizzle, 8-row groups 1024 bytes apart (SM100 descriptor:
// start>>4 [0,14), LBO>>4 [16,30) = 1, SBO>>4 [32,46) = 64, version [46,48) = 1,
// layout [61,64) = 2 (SWIZZLE_128B)).
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr)
{
    return (uint64_t)((saddr & 0x3FFFF) >> 4) | ((uint64_t)1 << 16) | ((uint64_t)64 << 32) |
           ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

// K-major operand tile of 32-element (64-byte) rows, 64-byte swizzle: 8-row groups 512 bytes apart
// (SBO>>4 = 32), layout [61,64) = 4 (SWIZZLE_64B); the tile base is 512-byte aligned and a 16-wide
// k-step advances the start address by 32 bytes, as in the 128-byte layout.
__device__ __forceinline__ uint64_t umma_desc64(uint32_t saddr)
{
    return (uint64_t)((saddr & 0x3FFFF) >> 4) | ((uint64_t)1 << 16) | ((uint64_t)32 << 32) |
           ((uint64_t)1 << 46) | ((uint64_t)4 << 61);
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc,
                                          uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
        ::"r"(tmem_d), "l"(da), "l"(db), "r"(idesc), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ void umma_commit(uint32_t bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float v[16])
{
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tmem_ld16_nowait(uint32_t taddr, uint32_t r[16])
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
}

// ---------------------------------------------------------------------------- epilogues

// k^(zeta - 1) for a compile-time integer zeta (ZI >= 1), else powf with the runtime zeta.
template <int ZI> __device__ __forceinline__ float kpow_zm1(float k, float zeta)
{
    if constexpr (ZI == 1) return 1.0f;
    else if constexpr (ZI == 2) return k;
    else if constexpr (ZI == 3) return k * k;
    else if constexpr (ZI == 4) return k * k * k;
    else if constexpr (ZI == 5) { const float k2 = k * k; return k2 * k2; }
    else if constexpr (ZI == 6) { const float k2 = k * k; return k2 * k2 * k; }
    else return powf(k, zeta - 1.0f);
}

// GEMM1: per element k = K[row][s]: energy alpha_s k^zeta summed over the row's columns and
// added (scaled by delta^2) into the row's atom, and G = zd2 alpha_s k^(zeta-1) written as a
// bf16 hi/lo split.
struct EpiKernelGap {
    const float *alphas;         // [m_pad]
    __nv_bfloat16 *G_hi, *G_lo;  // [rows_pad][ldg]
    int ldg;
    int n_rows;                  // rows past n_rows are padding
    const int *sites;            // row -> atom (null: identity)
    double *energies;            // energies[atom] += delta^2 sum_s alpha_s k^zeta (+ e0 once)
    double *e_rows;              // optional per-row copy (zeroed by the caller)
    double d2, e0;
    float zd2, zeta;
    int zeta_int;                // 1..6, or -1 for a non-integer zeta

    template <int ZI>
    __device__ __forceinline__ void chunk_z(int row, int col, const float v[16], float &acc) const
    {
        uint32_t hi[8], lo[8];
        const float4 *a4 = reinterpret_cast<const float4 *>(alphas + col);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const float4 a = a4[q];
            const float av[4] = {a.x, a.y, a.z, a.w};
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int j = 4 * q + 2 * h;
                const float k0 = v[j], k1 = v[j + 1];
                const float ak0 = av[2 * h] * kpow_zm1<ZI>(k0, zeta);
                const float ak1 = av[2 * h + 1] * kpow_zm1<ZI>(k1, zeta);
                acc = fmaf(ak0, k0, acc);
                acc = fmaf(ak1, k1, acc);
                const float g0 = zd2 * ak0, g1 = zd2 * ak1;
                const __nv_bfloat162 h2 = __floats2bfloat162_rn(g0, g1);
                const float2 hf = __bfloat1622float2(h2);
                const __nv_bfloat162 l2 = __floats2bfloat162_rn(g0 - hf.x, g1 - hf.y);
                hi[j / 2] = *reinterpret_cast<const uint32_t *>(&h2);
                lo[j / 2] = *reinterpret_cast<const uint32_t *>(&l2);
            }
        }
        uint4 *dh = reinterpret_cast<uint4 *>(G_hi + (size_t)row * ldg + col);
        uint4 *dl = reinterpret_cast<uint4 *>(G_lo + (size_t)row * ldg + col);
        dh[0] = make_uint4(hi[0], hi[1], hi[2], hi[3]);
        dh[1] = make_uint4(hi[4], hi[5], hi[6], hi[7]);
        dl[0] = make_uint4(lo[0], lo[1], lo[2], lo[3]);
        dl[1] = make_uint4(lo[4], lo[5], lo[6], lo[7]);
    }
    __device__ __forceinline__ void begin(float &acc) const { acc = 0.0f; }
    __device__ __forceinline__ void chunk(int row, int col, const float v[16], float &acc) const
    {
        switch (zeta_int) {
        case 1: chunk_z<1>(row, col, v, acc); break;
        case 2: chunk_z<2>(row, col, v, acc); break;
        case 3: chunk_z<3>(row, col, v, acc); break;
        case 4: chunk_z<4>(row, col, v, acc); break;
        case 5: chunk_z<5>(row, col, v, acc); break;
        case 6: chunk_z<6>(row, col, v, acc); break;
        default: chunk_z<-1>(row, col, v, acc); break;
        }
    }
    // part = 2 tile_n + half: each row receives one partial per tile column half
    __device__ __forceinline__ void end(int row, int part, float acc) const
    {
        if (row >= n_rows) return;
        double e = d2 * (double)acc;
        if (part == 0) e += e0;
        if (energies) atomicAdd(energies + (sites ? sites[row] : row), e);
        if (e_rows) atomicAdd(e_rows + row, e);
    }
};

struct EpiStoreF32 {
    float *C;
    int ldc;
    __device__ __forceinline__ void begin(float &) const {}
    __device__ __forceinline__ void chunk(int row, int col, const float v[16], float &) const
    {
        float4 *d = reinterpret_cast<float4 *>(C + (size_t)row * ldc + col);
#pragma unroll
        for (int i = 0; i < 4; ++i) d[i] = make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
    }
    __device__ __forceinline__ void end(int, int, float) const {}
};

// ---------------------------------------------------------------------------- kernel

// Persistent, warp-specialised: CTA c takes tiles c, c + gridDim.x, ... (tile = m_tile * n_tiles
// + n_tile). Warp 0 (one lane) streams A/B hi/lo k-blocks into the STAGES-deep ring, warp 1
// (one lane) issues the MMAs of a tile into one of two TMEM accumulator buffers (TmemPlan), warps 2..9 drain the other buffer through the epilogue, so a tile's epilogue overlaps
// the next tile's loads and MMAs. Epilogue warp w reads TMEM lanes 32 (w % 4) .. +31 (= tile
// rows) and one half of the tile's columns ((w - 2) / 4); its epilogue part index is
// 2 tile_n + half.
constexpr int kEpiWarps = 8;
constexpr int kTcWarps = 2 + kEpiWarps;
constexpr int kTcThreadsP = 32 * kTcWarps;
// Two TMEM accumulator buffers: BN <= 128 columns each in 256 allocated columns, or 256 each in 512.
template <int BN> struct TmemPlan {
    static constexpr uint32_t buf = BN <= 128 ? 128u : 256u;  // column stride of the buffers
    static constexpr uint32_t cols = 2 * buf;                  // allocation (power of two)
};

template <int BN, int STAGES, class Epi>
__global__ void __launch_bounds__(kTcThreadsP, 1)
    k_gemm_bf16x3(const __grid_constant__ CUtensorMap tmA_hi, const __grid_constant__ CUtensorMap tmA_lo,
                  const __grid_constant__ CUtensorMap tmB_hi, const __grid_constant__ CUtensorMap tmB_lo,
                  int n_tiles_n, int n_tiles, int num_kb, Epi epi, int *err_flag)
{
    static_assert(BN % 32 == 0 && BN >= 32 && BN <= 256, "BN: multiple of 32 in 32..256");
    constexpr uint32_t kTmemCols = TmemPlan<BN>::cols, kBuf = TmemPlan<BN>::buf;
    constexpr uint32_t A_BYTES = kBM * kBK * 2;
    constexpr uint32_t B_BYTES = BN * kBK * 2;
    constexpr uint32_t STAGE_BYTES = 2 * A_BYTES + 2 * B_BYTES;
    // instruction descriptor: D f32 [4,6)=1, A bf16 [7,10)=1, B bf16 [10,13)=1, K-major A/B,
    // N>>3 at [17,23), M>>4 at [24,29)
    constexpr uint32_t IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) |
                               ((uint32_t)(kBM >> 4) << 24);

    extern __shared__ __align__(1024) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t bar_full[STAGES], bar_empty[STAGES];
    __shared__ __align__(8) uint64_t bar_tfull[2], bar_tempty[2], bar_drain;
    __shared__ uint32_t tmem_base_slot;
    __shared__ volatile int abort_flag;
    __shared__ int issued, consumed;

    const uint32_t raw = smem_u32(smem_raw);
    const uint32_t base = (raw + 1023u) & ~1023u;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(smem_u32(&bar_full[s]), 1);
            mbar_init(smem_u32(&bar_empty[s]), 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(smem_u32(&bar_tfull[b]), 1);
            mbar_init(smem_u32(&bar_tempty[b]), 32 * kEpiWarps);
        }
        mbar_init(smem_u32(&bar_drain), 1);
        abort_flag = 0;
        issued = 0;
        consumed = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"((uint64_t)&tmA_hi) : "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"((uint64_t)&tmA_lo) : "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"((uint64_t)&tmB_hi) : "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"((uint64_t)&tmB_lo) : "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(&tmem_base_slot)),
                     "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_base_slot;

    if (warp == 0) {
        if (lane == 0) {
            // TMA producer
            int it = 0;
            for (int t = blockIdx.x; t < n_tiles && !abort_flag; t += gridDim.x) {
                const int m0 = (t / n_tiles_n) * kBM, n0 = (t % n_tiles_n) * BN;
                for (int kb = 0; kb < num_kb; ++kb, ++it) {
                    const int s = it % STAGES;
                    const uint32_t ph = (uint32_t)(it / STAGES) & 1u;
                    if (it >= STAGES && !mbar_wait(smem_u32(&bar_empty[s]), ph ^ 1u, &abort_flag)) {
                        abort_flag = 1;
                        break;
                    }
                    const uint32_t st = base + s * STAGE_BYTES;
                    const uint32_t fb = smem_u32(&bar_full[s]);
                    mbar_expect_tx(fb, STAGE_BYTES);
                    tma_load_2d(st, &tmA_hi, fb, kb * kBK, m0);
                    tma_load_2d(st + A_BYTES, &tmA_lo, fb, kb * kBK, m0);
                    tma_load_2d(st + 2 * A_BYTES, &tmB_hi, fb, kb * kBK, n0);
                    tma_load_2d(st + 2 * A_BYTES + B_BYTES, &tmB_lo, fb, kb * kBK, n0);
                    issued = it + 1;
                }
            }
            // tail: wait until the MMAs have released the last STAGES stages, so no asynchronous
            // arrive on a stage barrier is pending when the CTA exits (bounded)
            for (int i = (issued > STAGES ? issued - STAGES : 0); i < issued && !abort_flag; ++i)
                if (!mbar_wait(smem_u32(&bar_empty[i % STAGES]), (uint32_t)(i / STAGES) & 1u, &abort_flag))
                    abort_flag = 1;
        }
    } else if (warp == 1) {
        if (lane == 0) {
            // MMA issuer
            int it = 0, tc = 0;
            for (int t = blockIdx.x; t < n_tiles && !abort_flag; t += gridDim.x, ++tc) {
                const int b = tc & 1, use = tc >> 1;
                if (use > 0 && !mbar_wait(smem_u32(&bar_tempty[b]), (uint32_t)(use - 1) & 1u, &abort_flag)) {
                    abort_flag = 1;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t acc = tmem + (uint32_t)b * kBuf;
                for (int kb = 0; kb < num_kb; ++kb, ++it) {
                    const int s = it % STAGES;
                    const uint32_t ph = (uint32_t)(it / STAGES) & 1u;
                    if (!mbar_wait(smem_u32(&bar_full[s]), ph, &abort_flag)) {
                        abort_flag = 1;
                        break;
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    const uint32_t st = base + s * STAGE_BYTES;
#pragma unroll
                    for (int k = 0; k < kBK / 16; ++k) {
                        const uint64_t ahi = umma_desc(st + 32 * k);
                        const uint64_t alo = umma_desc(st + A_BYTES + 32 * k);
                        const uint64_t bhi = umma_desc(st + 2 * A_BYTES + 32 * k);
                        const uint64_t blo = umma_desc(st + 2 * A_BYTES + B_BYTES + 32 * k);
                        umma_bf16(acc, ahi, bhi, IDESC, (kb > 0 || k > 0) ? 1u : 0u);
                        umma_bf16(acc, ahi, blo, IDESC, 1u);
                        umma_bf16(acc, alo, bhi, IDESC, 1u);
                    }
                    umma_commit(smem_u32(&bar_empty[s]));
                    consumed = it + 1;
                }
                if (abort_flag) break;
                umma_commit(smem_u32(&bar_tfull[b]));
            }
            // every MMA issued so far has completed once bar_drain fires (bounded)
            umma_commit(smem_u32(&bar_drain));
            volatile int never = 0;
            mbar_wait(smem_u32(&bar_drain), 0, &never);
        }
    } else {
        // epilogue: rows 32 (warp % 4) + lane of the tile, columns [half BN/2, (half + 1) BN/2)
        const int quarter = warp & 3, half = (warp - 2) >> 2;
        const int r_local = quarter * 32 + lane;
        constexpr int HB = BN / 2;
        int tc = 0;
        for (int t = blockIdx.x; t < n_tiles; t += gridDim.x, ++tc) {
            const int b = tc & 1, use = tc >> 1;
            const bool ok = mbar_wait(smem_u32(&bar_tfull[b]), (uint32_t)use & 1u, &abort_flag);
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            __syncwarp();
            if (!ok || abort_flag) {
                abort_flag = 1;
                break;
            }
            const int row = (t / n_tiles_n) * kBM + r_local;
            const int tile_n = t % n_tiles_n, c0 = tile_n * BN + half * HB;
            const uint32_t taddr =
                tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)b * kBuf + (uint32_t)(half * HB);
            float acc;
            epi.begin(acc);
#pragma unroll 1
            for (int c = 0; c < HB; c += 16) {
                float v[16];
                tmem_ld16(taddr + (uint32_t)c, v);
                epi.chunk(row, c0 + c, v, acc);
            }
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            mbar_arrive(smem_u32(&bar_tempty[b]));
            epi.end(row, 2 * tile_n + half, acc);
        }
    }
    __syncwarp();
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (abort_flag) {
        if (threadIdx.x == 0) {
            atomicExch(err_flag, 1);
            // drain this CTA's own copies still in flight (bounded)
            volatile int dummy = 0;
            for (int i = consumed; i < issued; ++i)
                mbar_wait(smem_u32(&bar_full[i % STAGES]), (uint32_t)(i / STAGES) & 1u, &dummy);
        }
        __syncthreads();
    }
    if (warp == 1) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols)
                     : "memory");
    }
}

// ---------------------------------------------------------------------------- fused GAP kernel

// Energies and dE/dq of a 128-row tile against a chunk of T sparse tiles of BS points, without
// writing G (flash-style): per sparse tile j
//   S = q Q_j^T                          (tcgen05 bf16x3, TMEM columns [0, BS))
//   W = zeta delta^2 alpha o S^(zeta-1)   (epilogue warps: registers -> bf16 hi/lo in shared memory,
//                                          in the 128B-swizzled K-major layout the MMA reads)
//   g += W Q_j                           (tcgen05 bf16x3, N = DP in two halves, TMEM [BS, BS+DP))
// energies += delta^2 sum alpha S^zeta. MMA order S_{j+1} before g_j lets the epilogue of tile
// j+1 overlap the tensor work of tile j. At the end the tile's g partial is added to global g with
// vector atomics (g zeroed by the caller), energies with FP64 atomics.
// Warps: 0 TMA producer, 1 MMA issuer (+ TMEM owner), 2..9 epilogue (rows 32 (w % 4) + lane,
// columns half = (w - 2) / 4 of the tile). Shared memory: a STAGES-deep ring of equal slots (one
// k-block of q and Q_j, or one half of a Q_j^T k-block) and W.
constexpr int kFlashEpiWarps = 8;
constexpr int kFlashMaxChunkTiles = 16;  // sparse tiles per CTA (the chunk) at most
constexpr int kFlashThreads = 32 * (2 + kFlashEpiWarps);

// Ring slots hold kHK-element slices of the k dimension: for S the q rows and the sparse tile's rows
// over kHK descriptor components, for g one half of the tile's Q_j^T rows over kHK sparse points. The
// S product stops at the last 16-wide k-step holding descriptor components and the g halves cover
// the components only (the operands are zero past dim), which saves the padding's MMAs.
#ifndef TGAP_FLASH_HK
#define TGAP_FLASH_HK 64
#endif
// k elements per ring slot: 64 (128-byte swizzle, two 64 KB slots; the default) or 32 (64-byte
// swizzle, five 32 KB slots: measured 15 % slower on the MD workload, the kernel being bound by the
// L2 bandwidth all CTAs share rather than by one CTA's copies in flight)
constexpr int kHK = TGAP_FLASH_HK;
static_assert(kHK == 64 || kHK == 32, "ring slot width");
// operand descriptor of a ring slot
__device__ __forceinline__ uint64_t ring_desc(uint32_t saddr)
{
    if constexpr (kHK == 64) return umma_desc(saddr);
    else return umma_desc64(saddr);
}
template <int DP, int BS> struct FlashShape {
    static constexpr uint32_t TILE_A = kBM * kBK * 2;                 // W k-block of 64 (hi or lo), 128B swizzle
    static constexpr uint32_t HA = kBM * kHK * 2;                     // q slice (hi or lo)
    static constexpr uint32_t HB = BS * kHK * 2;                      // Q_j slice (hi or lo)
    static constexpr uint32_t HG = (DP / 2) * kHK * 2;                // Q_j^T half slice (hi or lo), largest
    static constexpr uint32_t SLOT_S = 2 * HA + 2 * HB;
    static constexpr uint32_t SLOT = SLOT_S > 2 * HG ? SLOT_S : 2 * HG;
    static constexpr uint32_t W = 2 * (BS / kBK) * TILE_A;            // hi + lo, BS/64 k-blocks each
    // 227 KB per CTA less the static part (barriers, the chunk's alphas)
    static constexpr int FIT = (int)((227u * 1024u - 2048u - 4u * kFlashMaxChunkTiles * BS - W) / SLOT);
    static constexpr int STAGES = FIT > 8 ? 8 : FIT;
    static constexpr size_t SMEM = (size_t)STAGES * SLOT + W + 1024;
};

struct FlashGap {
    const float *alphas;  // [m_pad]
    int n_rows;
    const int *sites;     // row -> atom (null: identity)
    double *energies;     // += delta^2 sum alpha k^zeta (+ e0 once per row)
    double *e_rows;       // optional per-row copy (zeroed by the caller)
    double d2, e0;
    float zd2, zeta;
    int zeta_int;
    float *g;             // dE/dq [rows_pad][ldg], accumulated (zeroed by the caller); null: energies only
    int ldg;
    const int *skip;      // optional device flag: when set, the launch does nothing
    const int *skip_tiles;  // optional per-row-tile flags: a CTA of a flagged tile does nothing
    // the descriptor's real width dim (<= DP): S takes n_kh 32-wide slices, the last with ks_last
    // 16-wide k-steps; g takes two halves of nh columns (nh a multiple of 16, 2 nh >= dim)
    int n_kh, ks_last, nh;
};

template <int ZI>
__device__ __forceinline__ void flash_w16(const float v[16], const float *__restrict__ alpha16, float zd2, float zeta,
                                          float &eacc, uint32_t hi[8], uint32_t lo[8])
{
    const float4 *a4 = reinterpret_cast<const float4 *>(alpha16);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const float4 a = a4[q];
        const float av[4] = {a.x, a.y, a.z, a.w};
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int j = 4 * q + 2 * h;
            const float ak0 = av[2 * h] * kpow_zm1<ZI>(v[j], zeta);
            const float ak1 = av[2 * h + 1] * kpow_zm1<ZI>(v[j + 1], zeta);
            eacc = fmaf(ak0, v[j], eacc);
            eacc = fmaf(ak1, v[j + 1], eacc);
            const float g0 = zd2 * ak0, g1 = zd2 * ak1;
            const __nv_bfloat162 h2 = __floats2bfloat162_rn(g0, g1);
            const float2 hf = __bfloat1622float2(h2);
            const __nv_bfloat162 l2 = __floats2bfloat162_rn(g0 - hf.x, g1 - hf.y);
            hi[j / 2] = *reinterpret_cast<const uint32_t *>(&h2);
            lo[j / 2] = *reinterpret_cast<const uint32_t *>(&l2);
        }
    }
}

__device__ __forceinline__ void st_shared_v4(uint32_t addr, uint32_t a, uint32_t b, uint32_t c, uint32_t d)
{
    asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(addr), "r"(a), "r"(b), "r"(c), "r"(d) : "memory");
}

template <int DP, int BS>
__global__ void __launch_bounds__(kFlashThreads, 1)
    k_gap_flash(const __grid_constant__ CUtensorMap tm_q_hi, const __grid_constant__ CUtensorMap tm_q_lo,
                const __grid_constant__ CUtensorMap tm_Q_hi, const __grid_constant__ CUtensorMap tm_Q_lo,
                const __grid_constant__ CUtensorMap tm_QT_hi, const __grid_constant__ CUtensorMap tm_QT_lo,
                int n_chunks, int tiles_per_chunk, FlashGap p, int *err_flag)
{
    using Sh = FlashShape<DP, BS>;
    static_assert(DP % 128 == 0 && DP + BS <= 512 && DP / 2 <= 256, "descriptor padding vs TMEM");
    static_assert(BS % 64 == 0 && BS <= 128, "sparse tile: 64 or 128");
    constexpr int STAGES = Sh::STAGES;
    static_assert(STAGES >= 2, "ring of at least two slots");
    constexpr int KG = BS / kBK;     // W k-blocks (64 wide) per sparse tile
    constexpr int HC = BS / 2;       // S columns per epilogue half
    constexpr uint32_t TILE_A = Sh::TILE_A, HA = Sh::HA, HB = Sh::HB, HG = Sh::HG, SLOT = Sh::SLOT;
    constexpr uint32_t IDESC_S = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BS >> 3) << 17) |
                                 ((uint32_t)(kBM >> 4) << 24);
    const int NH = p.nh;             // N of each g half
    const uint32_t IDESC_G = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(NH >> 3) << 17) |
                             ((uint32_t)(kBM >> 4) << 24);
    constexpr uint32_t kCols = 512;
    const bool forces = p.g != nullptr;
    pdl_enter();  // q, the cleared dE/dq rows and the skip flag come from earlier kernels
    if (p.skip && *p.skip) return;  // uniform over the grid, before any TMEM or barrier set-up
    if (p.skip_tiles && p.skip_tiles[blockIdx.x / n_chunks]) return;  // uniform over the CTA

    extern __shared__ __align__(1024) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t bar_full[STAGES], bar_empty[STAGES];
    __shared__ __align__(8) uint64_t bar_sfull, bar_sfree, bar_wfull, bar_wempty, bar_drain;
    // the alphas of the CTA's sparse tiles, read by the epilogue at shared-memory latency (a global
    // load per 16 columns put an L2 round trip between each S tile and its release)
    __shared__ __align__(16) float s_alpha[kFlashMaxChunkTiles * BS];
    __shared__ uint32_t tmem_base_slot;
    __shared__ volatile int abort_flag;
    __shared__ int issued, consumed;

    const uint32_t base = (smem_u32(smem_raw) + 1023u) & ~1023u;
    const uint32_t wbase = base + STAGES * SLOT;  // W: hi k-blocks, then lo k-blocks (TILE_A each)
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int unit = blockIdx.x, rt = unit / n_chunks, ch = unit - rt * n_chunks;
    const int T = tiles_per_chunk, j0 = ch * T, m0 = rt * kBM;
    for (int i = threadIdx.x; i < T * BS; i += blockDim.x) s_alpha[i] = p.alphas[j0 * BS + i];

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(smem_u32(&bar_full[s]), 1);
            mbar_init(smem_u32(&bar_empty[s]), 1);
        }
        mbar_init(smem_u32(&bar_sfull), 1);
        mbar_init(smem_u32(&bar_sfree), 32 * kFlashEpiWarps);
        mbar_init(smem_u32(&bar_wfull), 32 * kFlashEpiWarps);
        mbar_init(smem_u32(&bar_wempty), 1);
        mbar_init(smem_u32(&bar_drain), 1);
        abort_flag = 0;
        issued = 0;
        consumed = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        const CUtensorMap *maps[6] = {&tm_q_hi, &tm_q_lo, &tm_Q_hi, &tm_Q_lo, &tm_QT_hi, &tm_QT_lo};
        for (int i = 0; i < 6; ++i) asm volatile("prefetch.tensormap [%0];" ::"l"((uint64_t)maps[i]) : "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(&tmem_base_slot)),
                     "r"(kCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_base_slot;
    const uint32_t tS = tmem, tG = tmem + BS;

    if (warp == 0) {
        if (lane == 0) {
            // TMA producer: S_0 blocks, then per tile t: S_{t+1} blocks, g_t blocks (the MMA order)
            int it = 0;
            auto acquire = [&](uint32_t &slot, uint32_t &fb) -> bool {
                const int s = it % STAGES;
                const uint32_t ph = (uint32_t)(it / STAGES) & 1u;
                if (it >= STAGES && !mbar_wait(smem_u32(&bar_empty[s]), ph ^ 1u, &abort_flag)) return false;
                slot = base + s * SLOT;
                fb = smem_u32(&bar_full[s]);
                return true;
            };
            auto load_s = [&](int j) -> bool {
                for (int kh = 0; kh < p.n_kh; ++kh) {
                    uint32_t slot, fb;
                    if (!acquire(slot, fb)) return false;
                    mbar_expect_tx(fb, 2 * HA + 2 * HB);
                    tma_load_2d(slot, &tm_q_hi, fb, kh * kHK, m0);
                    tma_load_2d(slot + HA, &tm_q_lo, fb, kh * kHK, m0);
                    tma_load_2d(slot + 2 * HA, &tm_Q_hi, fb, kh * kHK, j * BS);
                    tma_load_2d(slot + 2 * HA + HB, &tm_Q_lo, fb, kh * kHK, j * BS);
                    issued = ++it;
                }
                return true;
            };
            const uint32_t g_bytes = 2u * (uint32_t)NH * (uint32_t)(kHK * 2);
            auto load_g = [&](int j) -> bool {
                for (int kh = 0; kh < BS / kHK; ++kh)
                    for (int h = 0; h < 2; ++h) {
                        uint32_t slot, fb;
                        if (!acquire(slot, fb)) return false;
                        mbar_expect_tx(fb, g_bytes);
                        tma_load_2d(slot, &tm_QT_hi, fb, j * BS + kh * kHK, h * NH);
                        tma_load_2d(slot + HG, &tm_QT_lo, fb, j * BS + kh * kHK, h * NH);
                        issued = ++it;
                    }
                return true;
            };
            bool ok = load_s(j0);
            for (int t = 0; t < T && ok; ++t) {
                if (t + 1 < T) ok = load_s(j0 + t + 1);
                if (ok && forces) ok = load_g(j0 + t);
            }
            if (!ok) abort_flag = 1;
            // tail: the last slots' releases land before the CTA exits (bounded)
            for (int i = (it > STAGES ? it - STAGES : 0); i < it && !abort_flag; ++i)
                if (!mbar_wait(smem_u32(&bar_empty[i % STAGES]), (uint32_t)(i / STAGES) & 1u, &abort_flag))
                    abort_flag = 1;
        }
    } else if (warp == 1) {
        if (lane == 0) {
            int it = 0;
            auto take = [&](uint32_t &slot) -> bool {
                const int s = it % STAGES;
                if (!mbar_wait(smem_u32(&bar_full[s]), (uint32_t)(it / STAGES) & 1u, &abort_flag)) return false;
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                slot = base + s * SLOT;
                return true;
            };
            auto release = [&]() {
                umma_commit(smem_u32(&bar_empty[it % STAGES]));
                consumed = ++it;
            };
            auto mma_s = [&]() -> bool {
                for (int kh = 0; kh < p.n_kh; ++kh) {
                    uint32_t slot;
                    if (!take(slot)) return false;
                    const int ks = kh == p.n_kh - 1 ? p.ks_last : kHK / 16;  // past dim the slice is zero
                    for (int k = 0; k < ks; ++k) {
                        const uint64_t ahi = ring_desc(slot + 32 * k), alo = ring_desc(slot + HA + 32 * k);
                        const uint64_t bhi = ring_desc(slot + 2 * HA + 32 * k);
                        const uint64_t blo = ring_desc(slot + 2 * HA + HB + 32 * k);
                        umma_bf16(tS, ahi, bhi, IDESC_S, (kh > 0 || k > 0) ? 1u : 0u);
                        umma_bf16(tS, ahi, blo, IDESC_S, 1u);
                        umma_bf16(tS, alo, bhi, IDESC_S, 1u);
                    }
                    release();
                }
                umma_commit(smem_u32(&bar_sfull));
                return true;
            };
            auto mma_g = [&](int t) -> bool {
                if (!mbar_wait(smem_u32(&bar_wfull), (uint32_t)t & 1u, &abort_flag)) return false;
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                for (int kh = 0; kh < BS / kHK; ++kh)
                    for (int h = 0; h < 2; ++h) {
                        uint32_t slot;
                        if (!take(slot)) return false;
#pragma unroll
                        for (int k = 0; k < kHK / 16; ++k) {
                            // W is K-major in 64-wide 128B-swizzled blocks: k-step kk of the tile
                            const int kk = kh * (kHK / 16) + k;
                            const uint32_t wo = (uint32_t)(kk / 4) * TILE_A + (uint32_t)(kk % 4) * 32;
                            const uint64_t ahi = umma_desc(wbase + wo), alo = umma_desc(wbase + KG * TILE_A + wo);
                            const uint64_t bhi = ring_desc(slot + 32 * k), blo = ring_desc(slot + HG + 32 * k);
                            const uint32_t d = tG + (uint32_t)(h * NH);
                            umma_bf16(d, ahi, bhi, IDESC_G, (t > 0 || kh > 0 || k > 0) ? 1u : 0u);
                            umma_bf16(d, ahi, blo, IDESC_G, 1u);
                            umma_bf16(d, alo, bhi, IDESC_G, 1u);
                        }
                        release();
                    }
                umma_commit(smem_u32(&bar_wempty));
                return true;
            };
            bool ok = mma_s();
            for (int t = 0; t < T && ok; ++t) {
                if (t + 1 < T) {
                    ok = mbar_wait(smem_u32(&bar_sfree), (uint32_t)t & 1u, &abort_flag);
                    if (ok) ok = mma_s();
                }
                if (ok && forces) ok = mma_g(t);
            }
            if (!ok) abort_flag = 1;
            // every MMA issued so far has completed once bar_drain fires (bounded)
            umma_commit(smem_u32(&bar_drain));
            volatile int never = 0;
            mbar_wait(smem_u32(&bar_drain), 0, &never);
        }
    } else {
        const int quarter = warp & 3, half = (warp - 2) >> 2;
        const int r = quarter * 32 + lane, row = m0 + r;
        const uint32_t lane_base = (uint32_t)(quarter * 32) << 16;
        float eacc = 0.0f;
        bool ok = true;
        for (int t = 0; t < T && ok; ++t) {
            const int j = j0 + t;
            ok = mbar_wait(smem_u32(&bar_sfull), (uint32_t)t & 1u, &abort_flag);
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            __syncwarp();
            if (!ok || abort_flag) break;
            // S leaves TMEM first (one wait for all loads), so the next tile's S product can start
            // while the W rows are computed
            uint32_t sraw[HC / 16][16];
#pragma unroll
            for (int c = 0; c < HC / 16; ++c) tmem_ld16_nowait(tS + lane_base + (uint32_t)(half * HC + c * 16), sraw[c]);
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            mbar_arrive(smem_u32(&bar_sfree));  // S may be overwritten
            uint32_t hi[HC / 16][8], lo[HC / 16][8];
#pragma unroll
            for (int c = 0; c < HC / 16; ++c) {
                float v[16];
#pragma unroll
                for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(sraw[c][i]);
                const float *a16 = s_alpha + (j - j0) * BS + half * HC + c * 16;
                switch (p.zeta_int) {
                case 1: flash_w16<1>(v, a16, p.zd2, p.zeta, eacc, hi[c], lo[c]); break;
                case 2: flash_w16<2>(v, a16, p.zd2, p.zeta, eacc, hi[c], lo[c]); break;
                case 3: flash_w16<3>(v, a16, p.zd2, p.zeta, eacc, hi[c], lo[c]); break;
                case 4: flash_w16<4>(v, a16, p.zd2, p.zeta, eacc, hi[c], lo[c]); break;
                case 5: flash_w16<5>(v, a16, p.zd2, p.zeta, eacc, hi[c], lo[c]); break;
                case 6: flash_w16<6>(v, a16, p.zd2, p.zeta, eacc, hi[c], lo[c]); break;
                default: flash_w16<-1>(v, a16, p.zd2, p.zeta, eacc, hi[c], lo[c]); break;
                }
            }
            if (!forces) continue;
            if (t > 0) {
                ok = mbar_wait(smem_u32(&bar_wempty), (uint32_t)(t - 1) & 1u, &abort_flag);
                if (!ok) break;
            }
            // W row r, sparse column col lies in k-block col / 64 of the K-major 128B-swizzled
            // tile, 16-byte chunk (col % 64) / 8 of the row, stored at chunk ^ (r % 8)
#pragma unroll
            for (int c = 0; c < HC / 16; ++c) {
#pragma unroll
                for (int u = 0; u < 2; ++u) {
                    const int col = half * HC + c * 16 + u * 8;
                    const uint32_t off = (uint32_t)(col / kBK) * TILE_A + r * 128 +
                                         (uint32_t)(((col % kBK) / 8) ^ (r & 7)) * 16;
                    st_shared_v4(wbase + off, hi[c][4 * u], hi[c][4 * u + 1], hi[c][4 * u + 2], hi[c][4 * u + 3]);
                    st_shared_v4(wbase + KG * TILE_A + off, lo[c][4 * u], lo[c][4 * u + 1], lo[c][4 * u + 2],
                                 lo[c][4 * u + 3]);
                }
            }
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            mbar_arrive(smem_u32(&bar_wfull));
        }
        if (ok && !abort_flag && row < p.n_rows) {
            double e = p.d2 * (double)eacc;
            if (ch == 0 && half == 0) e += p.e0;
            if (p.energies) atomicAdd(p.energies + (p.sites ? p.sites[row] : row), e);
            if (p.e_rows) atomicAdd(p.e_rows + row, e);
        }
        if (ok && !abort_flag && forces) {
            ok = mbar_wait(smem_u32(&bar_wempty), (uint32_t)(T - 1) & 1u, &abort_flag);
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            __syncwarp();
            if (ok && !abort_flag) {
#pragma unroll 1
                for (int c = 0; c < NH; c += 16) {
                    float v[16];
                    tmem_ld16(tG + lane_base + (uint32_t)(half * NH + c), v);
                    if (row < p.n_rows) {
                        float4 *dst = reinterpret_cast<float4 *>(p.g + (size_t)row * p.ldg + half * NH + c);
#pragma unroll
                        for (int i = 0; i < 4; ++i)
                            atomicAdd(dst + i, make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]));
                    }
                }
            }
        }
        if (!ok) abort_flag = 1;
    }
    __syncwarp();
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (abort_flag) {
        if (threadIdx.x == 0) {
            atomicExch(err_flag, 1);
            volatile int dummy = 0;
            for (int i = consumed; i < issued; ++i)
                mbar_wait(smem_u32(&bar_full[i % STAGES]), (uint32_t)(i / STAGES) & 1u, &dummy);
        }
        __syncthreads();
    }
    if (warp == 1) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kCols) : "memory");
    }
}

// ---------------------------------------------------------------------------- fused GAP kernel, CTA pair

// The same contraction on a pair of CTAs (a 2-CTA cluster on neighboring SMs) that share each sparse
// tile: tcgen05 MMAs of cta_group::2 have M = 256 (CTA r holds rows 128 r .. 128 r + 127 of the pair's
// two row tiles in its shared memory and TMEM) and read the B operand split along N, half from each
// CTA. Each CTA therefore loads its own q rows but only half of every Q_j and Q_j^T slice, which cuts
// the operand stream from L2 per SM by about a third (the single-CTA kernel is bound by that stream).
// The leader (rank 0) issues the MMAs and waits on its barriers for both CTAs' copies (each CTA's
// copies complete on the leader's full barrier) and both CTAs' epilogues (remote arrivals); the
// leader's commits arrive on the barriers of both CTAs. Every wait is bounded; a pair whose waits
// give up raises the error flag, and both CTAs meet at the closing cluster barrier before releasing
// TMEM.
__device__ __forceinline__ uint32_t cluster_ctarank()
{
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}

// shared::cluster address of the same shared variable in CTA `rank` of the cluster
__device__ __forceinline__ uint32_t cluster_addr(uint32_t saddr, uint32_t rank)
{
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(saddr), "r"(rank));
    return r;
}

__device__ __forceinline__ void mbar_arrive_cluster(uint32_t cluster_bar)
{
    asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(cluster_bar) : "memory");
}

__device__ __forceinline__ void cluster_sync_all()
{
    asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory");
    asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory");
}

// copy into this CTA's shared memory, completing bytes on the barrier `cluster_bar` (the leader's)
__device__ __forceinline__ void tma_load_2d_pair(uint32_t dst, const CUtensorMap *map, uint32_t cluster_bar, int x,
                                                 int y)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], "
        "[%2];" ::"r"(dst),
        "l"((uint64_t)map), "r"(cluster_bar), "r"(x), "r"(y)
        : "memory");
}

__device__ __forceinline__ void umma_bf16_pair(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc,
                                               uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(da), "l"(db), "r"(idesc), "r"(accumulate)
        : "memory");
}

// arrives once on the barrier at this shared offset in every CTA of `mask` when the pair's MMAs
// issued so far have completed
__device__ __forceinline__ void umma_commit_pair(uint32_t bar, uint16_t mask)
{
    asm volatile("tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 [%0], %1;"
                 ::"r"(bar), "h"(mask)
                 : "memory");
}

template <int DP, int BS> struct FlashPairShape {
    static constexpr uint32_t TILE_A = kBM * kBK * 2;           // W k-block of 64 (hi or lo), own rows
    static constexpr uint32_t HA = kBM * kBK * 2;               // q slice (hi or lo), own rows
    static constexpr uint32_t HB = (BS / 2) * kBK * 2;          // this CTA's half of a Q_j slice
    static constexpr uint32_t HG = (DP / 4) * kBK * 2;          // this CTA's half of a Q_j^T half slice, largest
    static constexpr uint32_t SLOT_S = 2 * HA + 2 * HB;
    static constexpr uint32_t SLOT = SLOT_S > 2 * HG ? SLOT_S : 2 * HG;
    static constexpr uint32_t W = 2 * (BS / kBK) * TILE_A;
    static constexpr int FIT = (int)((227u * 1024u - 2048u - 4u * kFlashMaxChunkTiles * BS - W) / SLOT);
    static constexpr int STAGES = FIT > 8 ? 8 : FIT;
    static constexpr size_t SMEM = (size_t)STAGES * SLOT + W + 1024;
};

template <int DP, int BS>
__global__ void __launch_bounds__(kFlashThreads, 1)
    k_gap_flash_pair(const __grid_constant__ CUtensorMap tm_q_hi, const __grid_constant__ CUtensorMap tm_q_lo,
                     const __grid_constant__ CUtensorMap tm_Q_hi, const __grid_constant__ CUtensorMap tm_Q_lo,
                     const __grid_constant__ CUtensorMap tm_QT_hi, const __grid_constant__ CUtensorMap tm_QT_lo,
                     int n_chunks, int tiles_per_chunk, FlashGap p, int *err_flag)
{
    using Sh = FlashPairShape<DP, BS>;
    static_assert(DP % 128 == 0 && DP + BS <= 512 && DP / 2 <= 256, "descriptor padding vs TMEM");
    static_assert(BS == 128, "sparse tile of 128 points, 64 per CTA");
    constexpr int STAGES = Sh::STAGES;
    static_assert(STAGES >= 2, "ring of at least two slots");
    constexpr int KG = BS / kBK;
    constexpr int HC = BS / 2;
    constexpr uint32_t TILE_A = Sh::TILE_A, HA = Sh::HA, HB = Sh::HB, HG = Sh::HG, SLOT = Sh::SLOT;
    // M = 256 over the pair (bits [24, 29) hold M >> 4)
    constexpr uint32_t IDESC_S = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BS >> 3) << 17) |
                                 ((uint32_t)((2 * kBM) >> 4) << 24);
    const int NH = p.nh;
    const uint32_t IDESC_G = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(NH >> 3) << 17) |
                             ((uint32_t)((2 * kBM) >> 4) << 24);
    constexpr uint32_t kCols = 512;
    const bool forces = p.g != nullptr;
    pdl_enter();
    if (p.skip && *p.skip) return;  // uniform over the grid: both CTAs of every pair leave together

    extern __shared__ __align__(1024) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t bar_full[STAGES], bar_empty[STAGES];
    __shared__ __align__(8) uint64_t bar_sfull, bar_sfree, bar_wfull, bar_wempty, bar_drain;
    __shared__ __align__(16) float s_alpha[kFlashMaxChunkTiles * BS];
    __shared__ uint32_t tmem_base_slot;
    __shared__ volatile int abort_flag;
    __shared__ int issued, consumed;

    const uint32_t base = (smem_u32(smem_raw) + 1023u) & ~1023u;
    const uint32_t wbase = base + STAGES * SLOT;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t rank = cluster_ctarank();
    const int pair = blockIdx.x >> 1, rtp = pair / n_chunks, ch = pair - rtp * n_chunks;
    const int T = tiles_per_chunk, j0 = ch * T, m0 = (2 * rtp + (int)rank) * kBM;
    for (int i = threadIdx.x; i < T * BS; i += blockDim.x) s_alpha[i] = p.alphas[j0 * BS + i];

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(smem_u32(&bar_full[s]), 1);
            mbar_init(smem_u32(&bar_empty[s]), 1);
        }
        mbar_init(smem_u32(&bar_sfull), 1);
        mbar_init(smem_u32(&bar_sfree), 2 * kFlashEpiWarps);  // one arrival per epilogue warp of the pair
        mbar_init(smem_u32(&bar_wfull), 2 * kFlashEpiWarps);
        mbar_init(smem_u32(&bar_wempty), 1);
        mbar_init(smem_u32(&bar_drain), 1);
        abort_flag = 0;
        issued = 0;
        consumed = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        const CUtensorMap *maps[6] = {&tm_q_hi, &tm_q_lo, &tm_Q_hi, &tm_Q_lo, &tm_QT_hi, &tm_QT_lo};
        for (int i = 0; i < 6; ++i) asm volatile("prefetch.tensormap [%0];" ::"l"((uint64_t)maps[i]) : "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(&tmem_base_slot)),
                     "r"(kCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    // both CTAs' barriers exist and both hold their TMEM before any copy, MMA or remote arrival
    cluster_sync_all();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_base_slot;
    const uint32_t tS = tmem, tG = tmem + BS;
    const uint32_t lead_sfree = cluster_addr(smem_u32(&bar_sfree), 0);
    const uint32_t lead_wfull = cluster_addr(smem_u32(&bar_wfull), 0);

    if (warp == 0) {
        if (lane == 0) {
            // TMA producer of both CTAs, same slot order as the single-CTA kernel; the leader posts the
            // pair's byte count on its full barrier, on which both CTAs' copies complete
            int it = 0;
            auto acquire = [&](uint32_t &slot, uint32_t &fb_own, uint32_t &fb_lead) -> bool {
                const int s = it % STAGES;
                const uint32_t ph = (uint32_t)(it / STAGES) & 1u;
                if (it >= STAGES && !mbar_wait(smem_u32(&bar_empty[s]), ph ^ 1u, &abort_flag)) return false;
                slot = base + s * SLOT;
                fb_own = smem_u32(&bar_full[s]);
                fb_lead = cluster_addr(fb_own, 0);
                return true;
            };
            auto load_s = [&](int j) -> bool {
                for (int kh = 0; kh < p.n_kh; ++kh) {
                    uint32_t slot, fo, fl;
                    if (!acquire(slot, fo, fl)) return false;
                    if (rank == 0) mbar_expect_tx(fo, 2u * (2 * HA + 2 * HB));
                    const int qrow = j * BS + (int)rank * (BS / 2);
                    tma_load_2d_pair(slot, &tm_q_hi, fl, kh * kBK, m0);
                    tma_load_2d_pair(slot + HA, &tm_q_lo, fl, kh * kBK, m0);
                    tma_load_2d_pair(slot + 2 * HA, &tm_Q_hi, fl, kh * kBK, qrow);
                    tma_load_2d_pair(slot + 2 * HA + HB, &tm_Q_lo, fl, kh * kBK, qrow);
                    issued = ++it;
                }
                return true;
            };
            const uint32_t g_bytes = 2u * 2u * (uint32_t)(NH / 2) * (uint32_t)(kBK * 2);
            auto load_g = [&](int j) -> bool {
                for (int kh = 0; kh < BS / kBK; ++kh)
                    for (int h = 0; h < 2; ++h) {
                        uint32_t slot, fo, fl;
                        if (!acquire(slot, fo, fl)) return false;
                        if (rank == 0) mbar_expect_tx(fo, g_bytes);
                        const int grow = h * NH + (int)rank * (NH / 2);
                        tma_load_2d_pair(slot, &tm_QT_hi, fl, j * BS + kh * kBK, grow);
                        tma_load_2d_pair(slot + HG, &tm_QT_lo, fl, j * BS + kh * kBK, grow);
                        issued = ++it;
                    }
                return true;
            };
            bool ok = load_s(j0);
            for (int t = 0; t < T && ok; ++t) {
                if (t + 1 < T) ok = load_s(j0 + t + 1);
                if (ok && forces) ok = load_g(j0 + t);
            }
            if (!ok) abort_flag = 1;
            for (int i = (it > STAGES ? it - STAGES : 0); i < it && !abort_flag; ++i)
                if (!mbar_wait(smem_u32(&bar_empty[i % STAGES]), (uint32_t)(i / STAGES) & 1u, &abort_flag))
                    abort_flag = 1;
        }
    } else if (warp == 1) {
        if (lane == 0 && rank == 0) {
            int it = 0;
            auto take = [&](uint32_t &slot) -> bool {
                const int s = it % STAGES;
                if (!mbar_wait(smem_u32(&bar_full[s]), (uint32_t)(it / STAGES) & 1u, &abort_flag)) return false;
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                slot = base + s * SLOT;
                return true;
            };
            auto release = [&]() {
                umma_commit_pair(smem_u32(&bar_empty[it % STAGES]), 0x3);  // the slot of both CTAs
                consumed = ++it;
            };
            auto mma_s = [&]() -> bool {
                for (int kh = 0; kh < p.n_kh; ++kh) {
                    uint32_t slot;
                    if (!take(slot)) return false;
                    const int ks = kh == p.n_kh - 1 ? p.ks_last : kBK / 16;
                    for (int k = 0; k < ks; ++k) {
                        const uint64_t ahi = umma_desc(slot + 32 * k), alo = umma_desc(slot + HA + 32 * k);
                        const uint64_t bhi = umma_desc(slot + 2 * HA + 32 * k);
                        const uint64_t blo = umma_desc(slot + 2 * HA + HB + 32 * k);
                        umma_bf16_pair(tS, ahi, bhi, IDESC_S, (kh > 0 || k > 0) ? 1u : 0u);
                        umma_bf16_pair(tS, ahi, blo, IDESC_S, 1u);
                        umma_bf16_pair(tS, alo, bhi, IDESC_S, 1u);
                    }
                    release();
                }
                umma_commit_pair(smem_u32(&bar_sfull), 0x3);
                return true;
            };
            auto mma_g = [&](int t) -> bool {
                if (!mbar_wait(smem_u32(&bar_wfull), (uint32_t)t & 1u, &abort_flag)) return false;
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                for (int kh = 0; kh < BS / kBK; ++kh)
                    for (int h = 0; h < 2; ++h) {
                        uint32_t slot;
                        if (!take(slot)) return false;
#pragma unroll
                        for (int k = 0; k < kBK / 16; ++k) {
                            const uint32_t wo = (uint32_t)kh * TILE_A + (uint32_t)k * 32;
                            const uint64_t ahi = umma_desc(wbase + wo), alo = umma_desc(wbase + KG * TILE_A + wo);
                            const uint64_t bhi = umma_desc(slot + 32 * k), blo = umma_desc(slot + HG + 32 * k);
                            const uint32_t d = tG + (uint32_t)(h * NH);
                            umma_bf16_pair(d, ahi, bhi, IDESC_G, (t > 0 || kh > 0 || k > 0) ? 1u : 0u);
                            umma_bf16_pair(d, ahi, blo, IDESC_G, 1u);
                            umma_bf16_pair(d, alo, bhi, IDESC_G, 1u);
                        }
                        release();
                    }
                umma_commit_pair(smem_u32(&bar_wempty), 0x3);
                return true;
            };
            bool ok = mma_s();
            for (int t = 0; t < T && ok; ++t) {
                if (t + 1 < T) {
                    ok = mbar_wait(smem_u32(&bar_sfree), (uint32_t)t & 1u, &abort_flag);
                    if (ok) ok = mma_s();
                }
                if (ok && forces) ok = mma_g(t);
            }
            if (!ok) abort_flag = 1;
            umma_commit_pair(smem_u32(&bar_drain), 0x1);
            volatile int never = 0;
            mbar_wait(smem_u32(&bar_drain), 0, &never);
        }
    } else {
        const int quarter = warp & 3, half = (warp - 2) >> 2;
        const int r = quarter * 32 + lane, row = m0 + r;
        const uint32_t lane_base = (uint32_t)(quarter * 32) << 16;
        float eacc = 0.0f;
        bool ok = true;
        for (int t = 0; t < T && ok; ++t) {
            const int j = j0 + t;
            ok = mbar_wait(smem_u32(&bar_sfull), (uint32_t)t & 1u, &abort_flag);
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            __syncwarp();
            if (!ok || abort_flag) break;
            uint32_t sraw[HC / 16][16];
#pragma unroll
            for (int c = 0; c < HC / 16; ++c) tmem_ld16_nowait(tS + lane_base + (uint32_t)(half * HC + c * 16), sraw[c]);
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive_cluster(lead_sfree);  // this warp's share of S may be overwritten
            uint32_t hi[HC / 16][8], lo[HC / 16][8];
#pragma unroll
            for (int c = 0; c < HC / 16; ++c) {
                float v[16];
#pragma unroll
                for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(sraw[c][i]);
                const float *a16 = s_alpha + (j - j0) * BS + half * HC + c * 16;
                switch (p.zeta_int) {
                case 1: flash_w16<1>(v, a16, p.zd2, p.zeta, eacc, hi[c], lo[c]); break;
                case 2: flash_w16<2>(v, a16, p.zd2, p.zeta, eacc, hi[c], lo[c]); break;
                case 3: flash_w16<3>(v, a16, p.zd2, p.zeta, eacc, hi[c], lo[c]); break;
                case 4: flash_w16<4>(v, a16, p.zd2, p.zeta, eacc, hi[c], lo[c]); break;
                case 5: flash_w16<5>(v, a16, p.zd2, p.zeta, eacc, hi[c], lo[c]); break;
                case 6: flash_w16<6>(v, a16, p.zd2, p.zeta, eacc, hi[c], lo[c]); break;
                default: flash_w16<-1>(v, a16, p.zd2, p.zeta, eacc, hi[c], lo[c]); break;
                }
            }
            if (!forces) continue;
            if (t > 0) {
                ok = mbar_wait(smem_u32(&bar_wempty), (uint32_t)(t - 1) & 1u, &abort_flag);
                if (!ok) break;
            }
#pragma unroll
            for (int c = 0; c < HC / 16; ++c) {
#pragma unroll
                for (int u = 0; u < 2; ++u) {
                    const int col = half * HC + c * 16 + u * 8;
                    const uint32_t off = (uint32_t)(col / kBK) * TILE_A + r * 128 +
                                         (uint32_t)(((col % kBK) / 8) ^ (r & 7)) * 16;
                    st_shared_v4(wbase + off, hi[c][4 * u], hi[c][4 * u + 1], hi[c][4 * u + 2], hi[c][4 * u + 3]);
                    st_shared_v4(wbase + KG * TILE_A + off, lo[c][4 * u], lo[c][4 * u + 1], lo[c][4 * u + 2],
                                 lo[c][4 * u + 3]);
                }
            }
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive_cluster(lead_wfull);  // this warp's W rows are in place
        }
        if (ok && !abort_flag && row < p.n_rows) {
            double e = p.d2 * (double)eacc;
            if (ch == 0 && half == 0) e += p.e0;
            if (p.energies) atomicAdd(p.energies + (p.sites ? p.sites[row] : row), e);
            if (p.e_rows) atomicAdd(p.e_rows + row, e);
        }
        if (ok && !abort_flag && forces) {
            ok = mbar_wait(smem_u32(&bar_wempty), (uint32_t)(T - 1) & 1u, &abort_flag);
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            __syncwarp();
            if (ok && !abort_flag) {
#pragma unroll 1
                for (int c = 0; c < NH; c += 16) {
                    float v[16];
                    tmem_ld16(tG + lane_base + (uint32_t)(half * NH + c), v);
                    if (row < p.n_rows) {
                        float4 *dst = reinterpret_cast<float4 *>(p.g + (size_t)row * p.ldg + half * NH + c);
#pragma unroll
                        for (int i = 0; i < 4; ++i)
                            atomicAdd(dst + i, make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]));
                    }
                }
            }
        }
        if (!ok) abort_flag = 1;
    }
    __syncwarp();
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (abort_flag) {
        if (threadIdx.x == 0) {
            atomicExch(err_flag, 1);
            volatile int dummy = 0;
            if (rank == 0)
                for (int i = consumed; i < issued; ++i)
                    mbar_wait(smem_u32(&bar_full[i % STAGES]), (uint32_t)(i / STAGES) & 1u, &dummy);
        }
        __syncthreads();
    }
    // neither CTA releases TMEM while the pair's MMAs or the other CTA's reads may still use it
    cluster_sync_all();
    if (warp == 1) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kCols) : "memory");
    }
}

// ---------------------------------------------------------------------------- host

typedef CUresult (*PFN_encodeTiled)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                    const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                    CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static PFN_encodeTiled encode_fn()
{
    static PFN_encodeTiled fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (PFN_encodeTiled)p;
    }
    return fn;
}

// Row-major bf16 matrix [rows][cols] (cols contiguous), box box_cols x box_rows: 64 columns with
// the 128-byte swizzle, 32 columns with the 64-byte one.
static int make_map(tgap_context *ctx, CUtensorMap *map, const void *ptr, int rows, int cols, int box_rows,
                    int box_cols = kBK)
{
    PFN_encodeTiled enc = encode_fn();
    if (!enc) return set_error(ctx, TGAP_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
    if (((uintptr_t)ptr & 15) || (cols * 2) % 16 || (box_cols != kBK && box_cols != 32))
        return set_error(ctx, TGAP_ERR_ARGUMENT, "tensor map alignment");
    cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)cols * 2};
    cuuint32_t box[2] = {(cuuint32_t)box_cols, (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void *>(ptr), dims, strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE,
                     box_cols == kBK ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return set_error(ctx, TGAP_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return TGAP_OK;
}

static int sm_count(tgap_context *ctx)
{
    static int n = 0;
    if (!n && cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, ctx->device) != cudaSuccess) n = 148;
    return n;
}

template <int BN, int STAGES, class Epi>
static int launch_gemm(tgap_context *ctx, const char *stage, const void *a_hi, const void *a_lo, const void *b_hi,
                       const void *b_lo, int M, int N, int K, Epi epi)
{
    // M, N, K are padded: M % 128 == 0, N % BN == 0, K % 64 == 0 (checked by the caller)
    CUtensorMap ta_hi, ta_lo, tb_hi, tb_lo;
    int rc;
    if ((rc = make_map(ctx, &ta_hi, a_hi, M, K, kBM)) || (rc = make_map(ctx, &ta_lo, a_lo, M, K, kBM)) ||
        (rc = make_map(ctx, &tb_hi, b_hi, N, K, BN)) || (rc = make_map(ctx, &tb_lo, b_lo, N, K, BN)))
        return rc;
    constexpr size_t smem = (size_t)STAGES * (2 * kBM * kBK * 2 + 2 * BN * kBK * 2) + 1024;
    static_assert(smem <= 227 * 1024 - 256, "stage ring exceeds shared memory");
    auto kern = k_gemm_bf16x3<BN, STAGES, Epi>;
    TGAP_CUDA(ctx, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    if (!ctx->d_flag) {
        TGAP_CUDA(ctx, cudaMalloc(&ctx->d_flag, sizeof(int)));
        TGAP_CUDA(ctx, cudaMemset(ctx->d_flag, 0, sizeof(int)));
    }
    const int n_tiles_n = N / BN, n_tiles = (M / kBM) * n_tiles_n;
    const int grid = n_tiles < sm_count(ctx) ? n_tiles : sm_count(ctx);
    StageScope sc(ctx, stage);
    kern<<<grid, kTcThreadsP, smem, ctx->stream>>>(ta_hi, ta_lo, tb_hi, tb_lo, n_tiles_n, n_tiles, K / kBK, epi,
                                                   ctx->d_flag);
    TGAP_LAUNCH_CHECK(ctx);
    return TGAP_OK;
}

#ifndef TGAP_FLASH_BS
#define TGAP_FLASH_BS 128
#endif
constexpr int kFlashBS = TGAP_FLASH_BS;  // sparse points per tile of the fused kernel

// Chunks of the sparse tiles per row tile: the fewest waves of (row tiles x chunks) CTAs times
// the tiles each CTA runs; ties go to fewer chunks (fewer g atomics).
static int flash_chunks(int n_rt, int J, int sms)
{
    int best = 1;
    long best_cost = -1;
    for (int nc = 1; nc <= J; ++nc) {
        if (J % nc || J / nc > kFlashMaxChunkTiles) continue;
        const long waves = ((long)n_rt * nc + sms - 1) / sms;
        const long cost = waves * (J / nc);
        if (best_cost < 0 || cost < best_cost) {
            best = nc;
            best_cost = cost;
        }
    }
    return best;
}

template <int DP, int BS>
static int launch_flash(tgap_context *ctx, const DeviceModel &m, const __nv_bfloat16 *q_hi, const __nv_bfloat16 *q_lo,
                        int rows_pad, const FlashGap &p)
{
    using Sh = FlashShape<DP, BS>;
    // the real descriptor width: S stops at the last 16-wide k-step that holds components, g at the
    // two halves of NH columns that cover them (the operands are zero beyond dim)
    FlashGap q = p;
    q.n_kh = (m.dim + kHK - 1) / kHK;
    q.ks_last = (m.dim - (q.n_kh - 1) * kHK + 15) / 16;
    q.nh = ((m.dim + 1) / 2 + 15) / 16 * 16;
    if (q.nh > DP / 2 || q.n_kh > DP / kHK) return set_error(ctx, TGAP_ERR_ARGUMENT, "fused GAP shape");
    CUtensorMap tq_hi, tq_lo, tQ_hi, tQ_lo, tT_hi, tT_lo;
    int rc;
    if ((rc = make_map(ctx, &tq_hi, q_hi, rows_pad, DP, kBM, kHK)) ||
        (rc = make_map(ctx, &tq_lo, q_lo, rows_pad, DP, kBM, kHK)) ||
        (rc = make_map(ctx, &tQ_hi, m.Q_hi.ptr, m.m_pad, DP, BS, kHK)) ||
        (rc = make_map(ctx, &tQ_lo, m.Q_lo.ptr, m.m_pad, DP, BS, kHK)) ||
        (rc = make_map(ctx, &tT_hi, m.QT_hi.ptr, DP, m.m_pad, q.nh, kHK)) ||
        (rc = make_map(ctx, &tT_lo, m.QT_lo.ptr, DP, m.m_pad, q.nh, kHK)))
        return rc;
    auto kern = k_gap_flash<DP, BS>;
    TGAP_CUDA(ctx, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Sh::SMEM));
    if (!ctx->d_flag) {
        TGAP_CUDA(ctx, cudaMalloc(&ctx->d_flag, sizeof(int)));
        TGAP_CUDA(ctx, cudaMemset(ctx->d_flag, 0, sizeof(int)));
    }
    const int J = m.m_pad / BS, n_rt = rows_pad / kBM;
    std::vector<int> divisors;
    for (int d = 1; d <= J; ++d)
        if (J % d == 0 && J / d <= kFlashMaxChunkTiles) divisors.push_back(d);
    char key[96];
    std::snprintf(key, sizeof(key), "gap_fused/dp%d/bs%d/row_tiles%d/sparse_tiles%d", DP, BS, n_rt, J);
    const int nc = tuned(ctx, key, "gemm_bf16x3_fused", divisors, flash_chunks(n_rt, J, sm_count(ctx)));
    StageScope sc(ctx, "gemm_bf16x3_fused");
    TGAP_CUDA(ctx, launch_pdl(kern, dim3(n_rt * nc), dim3(kFlashThreads), Sh::SMEM, ctx->stream, tq_hi, tq_lo, tQ_hi,
                              tQ_lo, tT_hi, tT_lo, nc, J / nc, q, ctx->d_flag));
    TGAP_LAUNCH_CHECK(ctx);
    return TGAP_OK;
}

// The CTA-pair form (k_gap_flash_pair): row tiles in pairs, a 2-CTA cluster per (pair, sparse chunk).
template <int DP, int BS>
static int launch_flash_pair(tgap_context *ctx, const DeviceModel &m, const __nv_bfloat16 *q_hi,
                             const __nv_bfloat16 *q_lo, int rows_pad, const FlashGap &p)
{
    using Sh = FlashPairShape<DP, BS>;
    FlashGap q = p;
    q.n_kh = (m.dim + kBK - 1) / kBK;
    q.ks_last = (m.dim - (q.n_kh - 1) * kBK + 15) / 16;
    q.nh = ((m.dim + 1) / 2 + 15) / 16 * 16;  // halves split again between the two CTAs: nh / 2 rows each
    if (q.nh > DP / 2 || q.n_kh > DP / kBK) return set_error(ctx, TGAP_ERR_ARGUMENT, "fused GAP shape");
    CUtensorMap tq_hi, tq_lo, tQ_hi, tQ_lo, tT_hi, tT_lo;
    int rc;
    if ((rc = make_map(ctx, &tq_hi, q_hi, rows_pad, DP, kBM)) || (rc = make_map(ctx, &tq_lo, q_lo, rows_pad, DP, kBM)) ||
        (rc = make_map(ctx, &tQ_hi, m.Q_hi.ptr, m.m_pad, DP, BS / 2)) ||
        (rc = make_map(ctx, &tQ_lo, m.Q_lo.ptr, m.m_pad, DP, BS / 2)) ||
        (rc = make_map(ctx, &tT_hi, m.QT_hi.ptr, DP, m.m_pad, q.nh / 2)) ||
        (rc = make_map(ctx, &tT_lo, m.QT_lo.ptr, DP, m.m_pad, q.nh / 2)))
        return rc;
    auto kern = k_gap_flash_pair<DP, BS>;
    TGAP_CUDA(ctx, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Sh::SMEM));
    if (!ctx->d_flag) {
        TGAP_CUDA(ctx, cudaMalloc(&ctx->d_flag, sizeof(int)));
        TGAP_CUDA(ctx, cudaMemset(ctx->d_flag, 0, sizeof(int)));
    }
    const int J = m.m_pad / BS, n_rt = rows_pad / kBM, n_pairs = (n_rt + 1) / 2;
    std::vector<int> divisors;
    for (int d = 1; d <= J; ++d)
        if (J % d == 0 && J / d <= kFlashMaxChunkTiles) divisors.push_back(d);
    char key[96];
    std::snprintf(key, sizeof(key), "gap_fused_pair/dp%d/bs%d/row_tiles%d/sparse_tiles%d", DP, BS, n_rt, J);
    const int nc = tuned(ctx, key, "gemm_bf16x3_fused", divisors, flash_chunks(2 * n_pairs, J, sm_count(ctx)));
    StageScope sc(ctx, "gemm_bf16x3_fused");
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(2 * n_pairs * nc);
    cfg.blockDim = dim3(kFlashThreads);
    cfg.dynamicSmemBytes = Sh::SMEM;
    cfg.stream = ctx->stream;
    cudaLaunchAttribute at[2];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = 2;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    at[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[1].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 2;
    TGAP_CUDA(ctx, cudaLaunchKernelEx(&cfg, kern, tq_hi, tq_lo, tQ_hi, tQ_lo, tT_hi, tT_lo, nc, J / nc, q, ctx->d_flag));
    TGAP_LAUNCH_CHECK(ctx);
    return TGAP_OK;
}

// The pair form where it applies (forces, no per-launch skip, at least two row tiles) and chosen,
// else the single-CTA kernel: the autotuner times both ("gap_fused_pair/.../pair" 1 or 0); the
// single-CTA form is the default (the pair form halves the sparse operands each SM loads but measured
// no faster on the MD workload, 49.6 against 47.6 us).
template <int DP, int BS>
static int launch_flash_any(tgap_context *ctx, const DeviceModel &m, const __nv_bfloat16 *q_hi,
                            const __nv_bfloat16 *q_lo, int rows_pad, const FlashGap &p)
{
    const int n_rt = rows_pad / kBM, J = m.m_pad / BS;
    if (p.g && !p.skip && !p.skip_tiles && n_rt >= 2) {
        char key[96];
        std::snprintf(key, sizeof(key), "gap_fused_pair/dp%d/bs%d/row_tiles%d/sparse_tiles%d/pair", DP, BS, n_rt, J);
        if (tuned(ctx, key, "gemm_bf16x3_fused", {0, 1}, 0)) return launch_flash_pair<DP, BS>(ctx, m, q_hi, q_lo, rows_pad, p);
    }
    return launch_flash<DP, BS>(ctx, m, q_hi, q_lo, rows_pad, p);
}

// ---------------------------------------------------------------------------- GAP mixed path

__global__ void k_split_bf16(int R, int C, int ld_in, const double *__restrict__ in, int R_pad, int C_pad,
                             int transpose, __nv_bfloat16 *__restrict__ hi, __nv_bfloat16 *__restrict__ lo)
{
    // out is [R_pad][C_pad] (or [C_pad][R_pad] when transposed), zero padded
    const size_t total = (size_t)R_pad * C_pad;
    for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < total; idx += (size_t)gridDim.x * blockDim.x) {
        const int r = (int)(idx / C_pad), c = (int)(idx % C_pad);
        const float v = (r < R && c < C) ? (float)in[(size_t)r * ld_in + c] : 0.0f;
        const __nv_bfloat16 h = __float2bfloat16_rn(v);
        const __nv_bfloat16 l = __float2bfloat16_rn(v - __bfloat162float(h));
        const size_t o = transpose ? (size_t)c * R_pad + r : idx;
        hi[o] = h;
        lo[o] = l;
    }
}

__global__ void k_pad_alphas(int n, int n_pad, const double *__restrict__ a, float *__restrict__ out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n_pad) out[i] = i < n ? (float)a[i] : 0.0f;
}

int model_upload_mixed(tgap_context *ctx, DeviceModel *m)
{
    m->dim_pad = (m->dim + 127) / 128 * 128;
    m->m_pad = (m->n_sparse + 127) / 128 * 128;
    const size_t n = (size_t)m->dim_pad * m->m_pad;
    if (m->Q_hi.ensure(2 * n) || m->Q_lo.ensure(2 * n) || m->QT_hi.ensure(2 * n) || m->QT_lo.ensure(2 * n) ||
        m->alphas32.ensure(4 * (size_t)m->m_pad))
        return set_error(ctx, TGAP_ERR_NOMEM, "mixed model operands");
    k_split_bf16<<<592, 256, 0, ctx->stream>>>(m->n_sparse, m->dim, m->dim, m->Qs.as<double>(), m->m_pad,
                                               m->dim_pad, 0, m->Q_hi.as<__nv_bfloat16>(),
                                               m->Q_lo.as<__nv_bfloat16>());
    TGAP_LAUNCH_CHECK(ctx);
    k_split_bf16<<<592, 256, 0, ctx->stream>>>(m->n_sparse, m->dim, m->dim, m->Qs.as<double>(), m->m_pad,
                                               m->dim_pad, 1, m->QT_hi.as<__nv_bfloat16>(),
                                               m->QT_lo.as<__nv_bfloat16>());
    TGAP_LAUNCH_CHECK(ctx);
    k_pad_alphas<<<(m->m_pad + 255) / 256, 256, 0, ctx->stream>>>(m->n_sparse, m->m_pad, m->alphas.as<double>(),
                                                                 m->alphas32.as<float>());
    TGAP_LAUNCH_CHECK(ctx);
    return TGAP_OK;
}

int gap_energy_grad_mixed(tgap_context *ctx, const DeviceModel &m, const __nv_bfloat16 *q_hi,
                          const __nv_bfloat16 *q_lo, int n_rows, double e0, int do_forces, GapWork *w,
                          const int *d_sites, double *d_e_rows, double *d_energies, const int *d_skip,
                          bool g_cleared, const int *d_skip_tiles)
{
    if (n_rows <= 0) return TGAP_OK;
    constexpr int BN1 = 128;  // m_pad is a multiple of 128; 256-column tiles when it allows
    const int rows_pad = (n_rows + kBM - 1) / kBM * kBM;
    if (m.dim_pad % 128 || m.m_pad % BN1 || m.dim_pad % kBK || m.m_pad % kBK)
        return set_error(ctx, TGAP_ERR_ARGUMENT, "mixed GEMM padding");
    if (do_forces && w->g.ensure(4 * (size_t)rows_pad * m.dim_pad))
        return set_error(ctx, TGAP_ERR_NOMEM, "mixed GAP workspace");
    if (d_e_rows) TGAP_CUDA(ctx, cudaMemsetAsync(d_e_rows, 0, sizeof(double) * (size_t)n_rows, ctx->stream));
    const double zr = m.zeta_nint ? std::nearbyint(m.zeta) : (double)(int)m.zeta;
    const bool zi = std::fabs(m.zeta - zr) < m.zeta_tol;  // gap.f90:99-105 (local properties: :76-77)
    if (m.dim_pad <= 384 && m.m_pad % 128 == 0) {
        // fused: G never leaves the SM (k_gap_flash); dE/dq accumulates with atomics
        if (do_forces && !g_cleared)
            TGAP_CUDA(ctx, cudaMemsetAsync(w->g.ptr, 0, 4 * (size_t)rows_pad * m.dim_pad, ctx->stream));
        FlashGap p;
        p.alphas = m.alphas32.as<float>();
        p.n_rows = n_rows;
        p.sites = d_sites;
        p.energies = d_energies;
        p.e_rows = d_e_rows;
        p.d2 = m.delta * m.delta;
        p.e0 = e0;
        p.zeta_int = zi ? (int)zr : -1;
        p.zeta = (float)(zi ? zr : m.zeta);
        p.zd2 = (float)(p.zeta * m.delta * m.delta);
        p.g = do_forces ? w->g.as<float>() : nullptr;
        p.ldg = m.dim_pad;
        p.skip = d_skip;
        p.skip_tiles = d_skip_tiles;
        // 128-point sparse tiles (64-point ones allow a deeper ring but double the per-tile handoffs,
        // and measured slower)
        switch (m.dim_pad) {
        case 128: return launch_flash_any<128, kFlashBS>(ctx, m, q_hi, q_lo, rows_pad, p);
        case 256: return launch_flash_any<256, kFlashBS>(ctx, m, q_hi, q_lo, rows_pad, p);
        default: return launch_flash_any<384, kFlashBS>(ctx, m, q_hi, q_lo, rows_pad, p);
        }
    }
    if (d_skip) return set_error(ctx, TGAP_ERR_UNSUPPORTED, "skippable launch needs the fused GAP kernel");
    if (w->G_hi.ensure(2 * (size_t)rows_pad * m.m_pad) || w->G_lo.ensure(2 * (size_t)rows_pad * m.m_pad))
        return set_error(ctx, TGAP_ERR_NOMEM, "mixed GAP workspace");
    EpiKernelGap e1;
    e1.alphas = m.alphas32.as<float>();
    e1.G_hi = w->G_hi.as<__nv_bfloat16>();
    e1.G_lo = w->G_lo.as<__nv_bfloat16>();
    e1.ldg = m.m_pad;
    e1.n_rows = n_rows;
    e1.sites = d_sites;
    e1.energies = d_energies;
    e1.e_rows = d_e_rows;
    e1.d2 = m.delta * m.delta;
    e1.e0 = e0;
    e1.zeta_int = zi ? (int)zr : -1;
    e1.zeta = (float)(zi ? zr : m.zeta);
    e1.zd2 = (float)(e1.zeta * m.delta * m.delta);
    // 256-column tiles re-read the descriptor rows half as often as 128-column ones (the GEMM is
    // bound by L2 -> SM operand traffic); two 96 KB stages then fill the shared memory
    int rc = m.m_pad % 256 == 0
                 ? launch_gemm<256, 2, EpiKernelGap>(ctx, "gemm_bf16x3_kernel", q_hi, q_lo, m.Q_hi.ptr, m.Q_lo.ptr,
                                                     rows_pad, m.m_pad, m.dim_pad, e1)
                 : launch_gemm<BN1, 3, EpiKernelGap>(ctx, "gemm_bf16x3_kernel", q_hi, q_lo, m.Q_hi.ptr, m.Q_lo.ptr,
                                                     rows_pad, m.m_pad, m.dim_pad, e1);
    if (rc) return rc;
    if (!do_forces) return TGAP_OK;
    // dE/dq: N = dim_pad is small, so 96-column tiles (when they divide it) give more tiles to
    // spread over the SMs than 128-column ones
    EpiStoreF32 e2{w->g.as<float>(), m.dim_pad};
    if (m.dim_pad % 96 == 0)
        return launch_gemm<96, 4, EpiStoreF32>(ctx, "gemm_bf16x3_grad", w->G_hi.ptr, w->G_lo.ptr, m.QT_hi.ptr,
                                               m.QT_lo.ptr, rows_pad, m.dim_pad, m.m_pad, e2);
    return launch_gemm<128, 3, EpiStoreF32>(ctx, "gemm_bf16x3_grad", w->G_hi.ptr, w->G_lo.ptr, m.QT_hi.ptr,
                                            m.QT_lo.ptr, rows_pad, m.dim_pad, m.m_pad, e2);
}

}  // namespace tgap
