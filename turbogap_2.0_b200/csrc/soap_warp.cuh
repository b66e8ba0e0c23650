// Warp-per-site SOAP kernels: forward expansion + power spectrum, and the adjoint that turns
// dE/dq into forces and the virial. Instantiated by soap_fwd_*.cu / soap_bwd_*.cu.
//
// A warp owns one central site; its in-cutoff pairs are compacted with a ballot into groups of
// at most 32 and each lane evaluates one pair completely (radial values, Bessel ratios, every
// real harmonic) with l_max (L) and the radial block bound (AMB >= alpha_max of every species)
// fixed at compile time, so harmonic indices, per-l factors and radial arrays live in registers.
//
//  forward   c[s-block][n][lm] = sum_{pairs j of species s} R_n(r_j) f_l(r_j) Y_lm(u_j)
//            One pass per species: the group's radial rows (AMB wide) and angular rows go to
//            shared memory and every lane accumulates the product for its own harmonics
//            lm = lane + 32 i over all n in registers. Then the power spectrum
//            p[n n' l] = (sqrt 2 if n != n') sum_m c[n][lm] c[n'][lm] and q = p / |p|.
//  adjoint   h = (g - q (q.g)) / |p|, Gc = dE/dc = M_l c (M from h), stored per species block
//            harmonic-major and AMB wide (zero padded) so a lane reads its radial weights with
//            16-byte loads; per pair w = sum_lm [R'.G f Y u + R.G (df Y u + f (grad Y)_perp / r)],
//            force -w on the neighbor and +w on the site, virial sum of r (x) f.
//
// FP32 instantiations (mixed path) take the radial values from a cubic Hermite table of R_n
// and dR_n/dr over kTabIntervals uniform intervals of [0, rcut_hard] (built in FP64 from the
// quadrature); FP64 instantiations run the Gauss-Legendre quadrature itself.
#pragma once

#include <cuda_bf16.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <tuple>
#include <type_traits>

#include "neighbors_device.cuh"
#include "soap_device.cuh"
#include "soap_kernels.h"

namespace tgap {

constexpr int kWarpsPerCta = 4;  // sites (warps) per CTA, fewer when shared memory is short

__device__ __forceinline__ unsigned lanemask_lt()
{
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// f_l = i_l(k)/i_0(k), l = 0..L+1: upward recurrence when k > L+2, else the continued fraction
// started at l = L+33 (same rule as the reference restatement; L+13 in FP32, where the start error
// has decayed below the rounding).
template <class T, int L>
__device__ __forceinline__ void bessel_ratios_fixed(T k, T f[L + 2])
{
    if (k < (T)1.0e-12) {
#pragma unroll
        for (int l = 0; l <= L + 1; ++l) f[l] = (l == 0) ? (T)1 : (T)0;
        return;
    }
    if (k > (T)(L + 2)) {
        f[0] = 1;
        f[1] = t_tanh_inv<T>(k) - (T)1 / k;
        if (std::is_same<T, float>::value) {
            const T ik = (T)1 / k;
#pragma unroll
            for (int l = 1; l <= L; ++l) f[l + 1] = f[l - 1] - (T)(2 * l + 1) * ik * f[l];
        } else {
#pragma unroll
            for (int l = 1; l <= L; ++l) f[l + 1] = f[l - 1] - (T)(2 * l + 1) / k * f[l];
        }
    } else {
        T rho = 0;
        if constexpr (std::is_same<T, float>::value) {
            // each backward step scales the error of its start value by k^2 / (2l+1)^2 < 1/4 (k <= L+2,
            // l >= L+2), so 12 steps leave < 4^-12 < 6e-8 of it, below the FP32 rounding; the fast
            // division's own rounding in these steps is damped the same way
#pragma unroll
            for (int l = L + 1 + 12; l > L + 1; --l) rho = __fdividef(k, (T)(2 * l + 1) + k * rho);
        } else {
            for (int l = L + 1 + 32; l > L + 1; --l) rho = k / ((T)(2 * l + 1) + k * rho);
        }
        T ratio[L + 2];
#pragma unroll
        for (int l = L + 1; l >= 1; --l) {
            rho = k / ((T)(2 * l + 1) + k * rho);
            ratio[l] = rho;
        }
        f[0] = 1;
#pragma unroll
        for (int l = 1; l <= L + 1; ++l) f[l] = f[l - 1] * ratio[l];
    }
}

// Every real harmonic of the unit vector u for a fixed L: fn(k, l, Y, dY/dux, dY/duy, dY/duz)
// with k = l^2 + {0 | 2m-1 (cos) | 2m (sin)}; the gradient treats the components as independent.
template <class T, int L, bool GRAD, class F>
__device__ __forceinline__ void ylm_all(const YlmConst &Yc, T ux, T uy, T uz, F &&fn)
{
    T Cc = 1, Sc = 0, Cp = 0, Sp = 0;
#pragma unroll
    for (int m = 0; m <= L; ++m) {
        if (m > 0) {
            Cp = Cc;
            Sp = Sc;
            const T cn = ux * Cc - uy * Sc;
            const T sn = ux * Sc + uy * Cc;
            Cc = cn;
            Sc = sn;
        }
        T Q2 = 0, Q1 = 0, dQ2 = 0, dQ1 = 0;
        const T qmm = yc_dfact<T>(Yc, m);
#pragma unroll
        for (int l = m; l <= L; ++l) {
            T Q, dQ;
            if (l == m) {
                Q = qmm;
                dQ = 0;
            } else if (l == m + 1) {
                Q = (T)(2 * m + 1) * uz * qmm;
                dQ = (T)(2 * m + 1) * qmm;
            } else {
                const T inv = (T)(1.0 / (double)(l - m));
                Q = ((T)(2 * l - 1) * uz * Q1 - (T)(l + m - 1) * Q2) * inv;
                dQ = ((T)(2 * l - 1) * (Q1 + uz * dQ1) - (T)(l + m - 1) * dQ2) * inv;
            }
            Q2 = Q1;
            Q1 = Q;
            dQ2 = dQ1;
            dQ1 = dQ;
            const T N = yc_norm<T>(Yc, l * (l + 1) / 2 + m);
            if (m == 0) {
                fn(l * l, l, N * Q, (T)0, (T)0, GRAD ? N * dQ : (T)0);
            } else {
                const T NQ = N * Q;
                if (GRAD) {
                    const T NQm = NQ * (T)m;
                    fn(l * l + 2 * m - 1, l, NQ * Cc, NQm * Cp, -NQm * Sp, N * dQ * Cc);
                    fn(l * l + 2 * m, l, NQ * Sc, NQm * Sp, NQm * Cp, N * dQ * Sc);
                } else {
                    fn(l * l + 2 * m - 1, l, NQ * Cc, (T)0, (T)0, (T)0);
                    fn(l * l + 2 * m, l, NQ * Sc, (T)0, (T)0, (T)0);
                }
            }
        }
    }
}

// Geometry of a group of at most 32 accepted pairs, staged per warp by the compaction so that the
// lane evaluating pair p reads it from shared memory: |r_ij|, r_j - r_i, the list index and the
// neighbor's species channel (0-based).
struct GroupStage {
    double r[32], x[32], y[32], z[32];
    long long k[32];
    int s[32];
};

// Compacts the next (at most 32) accepted pairs of [scan, ke) into st with their geometry (accepted:
// species channel known, and equal to only_s when only_s >= 0, and 0 < r < rcut_hard(s)); returns
// the count and advances scan past the last pair taken. Every lane loads the geometry of its list
// entry together with its species, so the group costs one round trip to L2 per 32 entries scanned.
__device__ __forceinline__ int compact_stage(const SoapParams &P, int64_t &scan, int64_t ke,
                                             const double *__restrict__ rjs, const double *__restrict__ xyz,
                                             const int *__restrict__ nsp, int only_s, GroupStage *st, int lane)
{
    int cnt = 0;
    while (cnt < 32 && scan < ke) {
        const int64_t k = scan + lane;
        bool ok = false;
        double d = 0.0, x = 0.0, y = 0.0, z = 0.0;
        int s = -1;
        if (k < ke) {
            s = nsp[k] - 1;
            // L2-coherent: an MD step's forward may have written them this launch
            d = __ldcg(rjs + k);
            x = __ldcg(xyz + 3 * k);
            y = __ldcg(xyz + 3 * k + 1);
            z = __ldcg(xyz + 3 * k + 2);
            ok = s >= 0 && s < P.n_species && (only_s < 0 || s == only_s) && d > 0.0 && d < P.rcut_hard[s];
        }
        const unsigned mask = __ballot_sync(0xffffffffu, ok);
        const int nv = __popc(mask);
        const int room = 32 - cnt;
        const int rank = __popc(mask & lanemask_lt());
        if (ok && rank < room) {
            const int o = cnt + rank;
            st->r[o] = d;
            st->x[o] = x;
            st->y[o] = y;
            st->z[o] = z;
            st->k[o] = (long long)k;
            st->s[o] = s;
        }
        if (nv > room) {
            // resume at the first accepted pair that did not fit
            scan += __fns(mask, 0, room + 1);
            cnt = 32;
            break;
        }
        cnt += nv;
        scan += 32;
    }
    __syncwarp();
    return cnt;
}

// Radial values (and d/dr) from the cubic Hermite table: entry (s, i, n) holds the coefficients
// (a, b, c, d) of R_n on interval i in t = r/h - i; dR/dr = (b + 2ct + 3dt^2) / h.
template <int AMB, bool DERIV>
__device__ __forceinline__ void radial_tab(const SoapParams &P, int s, double r, const float4 *__restrict__ tab,
                                           float R[AMB], float dR[AMB])
{
    const int am = P.alpha_max[s];
    const double xr = r * P.tab_scale[s];
    int i = (int)xr;
    i = i < 0 ? 0 : (i > kTabIntervals - 1 ? kTabIntervals - 1 : i);
    const float t = (float)(xr - (double)i);
    const float ih = (float)P.tab_scale[s];
    const float4 *e = tab + ((size_t)s * kTabIntervals + i) * P.am_pad;
#pragma unroll
    for (int n = 0; n < AMB; ++n) {
        if (n < am) {
            const float4 c = __ldg(e + n);
            R[n] = c.x + t * (c.y + t * (c.z + t * c.w));
            dR[n] = DERIV ? (c.y + t * (2.0f * c.z + 3.0f * t * c.w)) * ih : 0.0f;
        } else {
            R[n] = 0.0f;
            dR[n] = 0.0f;
        }
    }
}

template <class T, int AMB, bool DERIV>
__device__ __forceinline__ void radial_values(const SoapParams &P, int s, double rd, const T *__restrict__ xq,
                                              const T *__restrict__ tq, const float4 *__restrict__ tab,
                                              T R[AMB], T dR[AMB])
{
    if constexpr (std::is_same<T, float>::value)
        radial_tab<AMB, DERIV>(P, s, rd, tab, R, dR);
    else
        radial_quad<T, AMB, DERIV>(P, s, (T)rd, xq, tq, R, dR);
}

// 16-byte loads of N consecutive values (N a multiple of 16 / sizeof(T), p 16-byte aligned).
template <class T, int N>
__device__ __forceinline__ void load_vec(const T *__restrict__ p, T v[N])
{
    if constexpr (std::is_same<T, float>::value) {
        static_assert(N % 4 == 0, "float rows are loaded 4 at a time");
#pragma unroll
        for (int i = 0; i < N / 4; ++i) {
            const float4 x = reinterpret_cast<const float4 *>(p)[i];
            v[4 * i] = x.x;
            v[4 * i + 1] = x.y;
            v[4 * i + 2] = x.z;
            v[4 * i + 3] = x.w;
        }
    } else {
        static_assert(N % 2 == 0, "double rows are loaded 2 at a time");
#pragma unroll
        for (int i = 0; i < N / 2; ++i) {
            const double2 x = reinterpret_cast<const double2 *>(p)[i];
            v[2 * i] = x.x;
            v[2 * i + 1] = x.y;
        }
    }
}

// 16-byte stores of N consecutive values (p 16-byte aligned).
template <class T, int N>
__device__ __forceinline__ void store_vec(T *p, const T v[N])
{
    if constexpr (std::is_same<T, float>::value) {
        static_assert(N % 4 == 0, "float rows are stored 4 at a time");
#pragma unroll
        for (int i = 0; i < N / 4; ++i)
            reinterpret_cast<float4 *>(p)[i] = make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
    } else {
        static_assert(N % 2 == 0, "double rows are stored 2 at a time");
#pragma unroll
        for (int i = 0; i < N / 2; ++i) reinterpret_cast<double2 *>(p)[i] = make_double2(v[2 * i], v[2 * i + 1]);
    }
}

// dst[o] = src[o] for o < n by the 32 lanes of a warp, 16 bytes at a time when n and both
// pointers allow it.
template <class T>
__device__ __forceinline__ void warp_copy_row(T *dst, const T *__restrict__ src, int n, int lane)
{
    constexpr int VW = 16 / (int)sizeof(T);
    using V = typename std::conditional<std::is_same<T, float>::value, float4, double2>::type;
    if (n % VW == 0 && ((reinterpret_cast<uintptr_t>(src) | reinterpret_cast<uintptr_t>(dst)) & 15) == 0) {
        const V *sv = reinterpret_cast<const V *>(src);
        V *dv = reinterpret_cast<V *>(dst);
        for (int o = lane; o < n / VW; o += 32) dv[o] = sv[o];
    } else {
        for (int o = lane; o < n; o += 32) dst[o] = src[o];
    }
}

// dst[o] = src[o] for o < n as warp_copy_row, with asynchronous 16-byte copies (cp.async, one
// commit group) where n and both pointers allow it, else a plain copy; dst may be read after
// cp_async_wait_all and a __syncwarp.
template <class T>
__device__ __forceinline__ void warp_copy_row_async(T *dst, const T *__restrict__ src, int n, int lane)
{
    constexpr int VW = 16 / (int)sizeof(T);
    if (n % VW == 0 && ((reinterpret_cast<uintptr_t>(src) | reinterpret_cast<uintptr_t>(dst)) & 15) == 0) {
        const uint32_t d0 = (uint32_t)__cvta_generic_to_shared(dst);
        for (int o = lane; o < n / VW; o += 32)
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d0 + 16u * (uint32_t)o), "l"(src + VW * o)
                         : "memory");
        asm volatile("cp.async.commit_group;" ::: "memory");
    } else {
        for (int o = lane; o < n; o += 32) dst[o] = src[o];
    }
}

__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Lane partial of q . g over n elements (FP32 rows of the same type four at a time when aligned;
// the caller reduces across the warp).
template <class T, class GT>
__device__ __forceinline__ T warp_dot_part(const T *__restrict__ q, const GT *__restrict__ g, int n, int lane)
{
    T acc = 0;
    if constexpr (std::is_same<T, float>::value && std::is_same<GT, float>::value) {
        if (n % 4 == 0 && ((reinterpret_cast<uintptr_t>(q) | reinterpret_cast<uintptr_t>(g)) & 15) == 0) {
            const float4 *q4 = reinterpret_cast<const float4 *>(q);
            const float4 *g4 = reinterpret_cast<const float4 *>(g);
            for (int o = lane; o < n / 4; o += 32) {
                const float4 a = q4[o], b = g4[o];
                acc += a.x * b.x;
                acc += a.y * b.y;
                acc += a.z * b.z;
                acc += a.w * b.w;
            }
            return acc;
        }
    }
    for (int d = lane; d < n; d += 32) acc += q[d] * (T)g[d];
    return acc;
}

// acc[n] += x[n] a for n < N. FP32 rows use the packed two-lane FMA of sm_100 (FFMA2: two
// independent FMAs per instruction, each rounded as a scalar fmaf, so results are unchanged).
template <class T, int N>
__device__ __forceinline__ void axpy_row(T acc[N], const T x[N], T a)
{
    if constexpr (std::is_same<T, float>::value && N % 2 == 0) {
        const float2 a2 = make_float2(a, a);
#pragma unroll
        for (int n = 0; n < N; n += 2) {
            const float2 r = __ffma2_rn(make_float2(x[n], x[n + 1]), a2, make_float2(acc[n], acc[n + 1]));
            acc[n] = r.x;
            acc[n + 1] = r.y;
        }
    } else {
#pragma unroll
        for (int n = 0; n < N; ++n) acc[n] += x[n] * a;
    }
}

// Even and odd partial sums of x . y (s0 over even indices, s1 over odd, each in index order);
// FP32 with the packed two-lane FMA.
template <class T, int N>
__device__ __forceinline__ void dot_even_odd(const T x[N], const T y[N], T &s0, T &s1)
{
    static_assert(N % 2 == 0, "even length");
    if constexpr (std::is_same<T, float>::value) {
        float2 acc = make_float2(0.0f, 0.0f);
#pragma unroll
        for (int e = 0; e < N; e += 2) acc = __ffma2_rn(make_float2(x[e], x[e + 1]), make_float2(y[e], y[e + 1]), acc);
        s0 = acc.x;
        s1 = acc.y;
    } else {
        T a0 = 0, a1 = 0;
#pragma unroll
        for (int e = 0; e < N; e += 2) {
            a0 += x[e] * y[e];
            a1 += x[e + 1] * y[e + 1];
        }
        s0 = a0;
        s1 = a1;
    }
}

// Adjoint of one pair's angular-radial product, summed over every real harmonic:
//   w = u (A1 - u.Gam) + Gam,  A1 = sum_lm Y_lm (f_l V_lm + df_l U_lm),
//   Gam = (1/r) sum_lm f_l U_lm dY_lm/du,   U_lm = Gc[lm].R, V_lm = Gc[lm].R'
// which equals sum_lm [u Y (f V + df U) + f U (grad Y - u (u.grad Y)) / r]. The order m is
// unrolled (compile time) and the degree l = m..L runs as a loop (in the instruction cache). The
// Legendre factor is carried fully normalised (Qb = N Q) by the three-term recurrence
// Qb_{l+1} = ra uz Qb_l - rb Qb_{l-1}, advanced at the end of each pass so the body has no
// branch; the Gc row, f_l / df_l (fl[l * 32] / dfl[l * 32]) and the recurrence
// coefficients are reached by running offsets. The cos and sin harmonics of one (l, m) share
// their Legendre factors and read their two adjacent Gc rows together.
template <class T, int L, int AMB>
__device__ __forceinline__ void pair_adjoint(const YlmConst &Yc, T ux, T uy, T uz, T ir, const T *fl, const T *dfl,
                                             const T *__restrict__ Gs, const T R[AMB], const T dR[AMB], T w[3])
{
    // the degree loop runs unrolled by 2 in FP32 (46 against 48 us for the 4096-atom adjoint: the
    // recurrence's rotation of Q, dQ needs no moves); in FP64 that costs registers and runs slower
    constexpr int kDegUnroll = std::is_same<T, float>::value ? 2 : 1;
    T A1 = 0, Gx = 0, Gy = 0, Gz = 0;
    // m = 0: Y = Qb, dY/du = (0, 0, dQb)
    {
        T Q = yc_qb0<T>(Yc, 0), dQ = 0, Qp = 0, dQp = 0;
        const T *row = Gs;
        int step = AMB;  // row (l+1)^2 - row l^2, in elements
        const T *f = fl, *df = dfl;
#pragma unroll(kDegUnroll)
        for (int l = 0; l <= L; ++l) {
            T g[AMB];
            load_vec<T, AMB>(row, g);
            T U0, U1, V0, V1;
            dot_even_odd<T, AMB>(g, R, U0, U1);
            dot_even_odd<T, AMB>(g, dR, V0, V1);
            const T U = U0 + U1, V = V0 + V1;
            const T fv = *f, dfv = *df;
            A1 += Q * (fv * V + dfv * U);
            Gz += dQ * (fv * U);
            const int ri = rec_off(0) + l;  // target degree l + 1
            const T ra = yc_ra<T>(Yc, ri), rb = yc_rb<T>(Yc, ri);
            const T Qn = ra * uz * Q - rb * Qp;
            const T dQn = ra * (Q + uz * dQ) - rb * dQp;
            Qp = Q;
            Q = Qn;
            dQp = dQ;
            dQ = dQn;
            row += step;
            step += 2 * AMB;
            f += 32;
            df += 32;
        }
    }
    T Cc = 1, Sc = 0;
#pragma unroll
    for (int m = 1; m <= L; ++m) {
        const T Cp = Cc, Sp = Sc;
        Cc = ux * Cp - uy * Sp;
        Sc = ux * Sp + uy * Cp;
        const T fm = (T)m;
        T Q = yc_qb0<T>(Yc, m), dQ = 0, Qp = 0, dQp = 0;
        // rows of the cos (l^2 + 2m - 1) and sin (l^2 + 2m) harmonics, adjacent in Gs
        const T *row = Gs + (m * m + 2 * m - 1) * AMB;
        int step = (2 * m + 1) * AMB;
        const T *f = fl + m * 32, *df = dfl + m * 32;
#pragma unroll(kDegUnroll)
        for (int l = m; l <= L; ++l) {
            T gc[AMB], gs[AMB];
            load_vec<T, AMB>(row, gc);
            load_vec<T, AMB>(row + AMB, gs);
            T Uc0, Uc1, Vc0, Vc1, Us0, Us1, Vs0, Vs1;
            dot_even_odd<T, AMB>(gc, R, Uc0, Uc1);
            dot_even_odd<T, AMB>(gc, dR, Vc0, Vc1);
            dot_even_odd<T, AMB>(gs, R, Us0, Us1);
            dot_even_odd<T, AMB>(gs, dR, Vs0, Vs1);
            const T Uc = Uc0 + Uc1, Vc = Vc0 + Vc1, Us = Us0 + Us1, Vs = Vs0 + Vs1;
            const T fv = *f, dfv = *df;
            const T ac = fv * Vc + dfv * Uc, as = fv * Vs + dfv * Us;
            const T bc = fv * Uc, bs = fv * Us;
            const T Qm = Q * fm;
            // cos: Y = Qb C, dY/du = (m Qb C', -m Qb S', dQb C); sin: Y = Qb S, (m Qb S', m Qb C', dQb S)
            A1 += Q * (ac * Cc + as * Sc);
            Gx += Qm * (bc * Cp + bs * Sp);
            Gy += Qm * (bs * Cp - bc * Sp);
            Gz += dQ * (bc * Cc + bs * Sc);
            const int ri = rec_off(m) + (l - m);  // target degree l + 1
            const T ra = yc_ra<T>(Yc, ri), rb = yc_rb<T>(Yc, ri);
            const T Qn = ra * uz * Q - rb * Qp;
            const T dQn = ra * (Q + uz * dQ) - rb * dQp;
            Qp = Q;
            Q = Qn;
            dQp = dQ;
            dQ = dQn;
            row += step;
            step += 2 * AMB;
            f += 32;
            df += 32;
        }
    }
    Gx *= ir;
    Gy *= ir;
    Gz *= ir;
    const T ug = ux * Gx + uy * Gy + uz * Gz;
    w[0] = ux * (A1 - ug) + Gx;
    w[1] = uy * (A1 - ug) + Gy;
    w[2] = uz * (A1 - ug) + Gz;
}

// Row stride of the angular rows in shared memory: odd, so the 32 lanes writing their own pair's
// row hit 32 different banks.
template <int NLM> struct AStride {
    static constexpr int value = (NLM % 2 == 0) ? NLM + 1 : NLM;
};

// ----------------------------------------------------------------------------- forward

// Values of the compression P in the kernel's precision: by rows (the forward) or by columns.
template <class T> __device__ __forceinline__ const T *cmp_vals(const SoapParams &P, bool by_rows)
{
    if constexpr (std::is_same<T, float>::value) return by_rows ? P.cmp_rval32 : P.cmp_cval32;
    else return by_rows ? P.cmp_rval : P.cmp_cval;
}

// Elements of the forward's middle area: the angular rows [32][astr], the power spectrum [dim] (and
// its compression P p [dim_c] after it, dim_c = 0 without compression) and the group stage,
// whichever is largest, rounded to 16 bytes.
template <class T> __host__ __device__ constexpr int fwd_area(int astr, int dim, int dim_c)
{
    const int a = 32 * astr > dim + dim_c ? 32 * astr : dim + dim_c;
    const int g = (int)((sizeof(GroupStage) + sizeof(T) - 1) / sizeof(T));
    const int m = a > g ? a : g;
    return (m + (int)(16 / sizeof(T)) - 1) / (int)(16 / sizeof(T)) * (int)(16 / sizeof(T));
}

// Shared memory of one warp: Rs [32][AMB], then an area holding the group's staged geometry
// (GroupStage, until the lanes have read it) and the angular rows [32][ASTR] during the passes and
// the power spectrum [dim] after them, then the expansion c [n_max][NLM].
// Minimum resident CTAs of 4 warps asked of the compiler for the forward: 4 in FP32 (at most 128
// registers, the count at which four CTAs' shared memory also fits), none in FP64 (128 spills).
template <class T, bool PERSIST> struct FwdMinCtas {
    static constexpr int value = std::is_same<T, float>::value ? 4 : 0;
};

template <class T, int L, int AMB, bool SPLIT, bool PERSIST, bool CMP>
__global__ void __launch_bounds__(32 * kWarpsPerCta, FwdMinCtas<T, PERSIST>::value) k_soap_fwd_warp(
    const __grid_constant__ SoapParams P, const __grid_constant__ YlmConst Yc, const T *__restrict__ xq,
    const T *__restrict__ tq, const float4 *__restrict__ rtab, const T *__restrict__ central,
    const int *__restrict__ sites, int n_rows, const int64_t *__restrict__ start,
    const double *__restrict__ rjs, const double *__restrict__ xyz, const int *__restrict__ nsp,
    T *__restrict__ c_out, T *__restrict__ q_out, int q_ld, T *__restrict__ norm_out,
    __nv_bfloat16 *__restrict__ q_hi, __nv_bfloat16 *__restrict__ q_lo, int warp_smem, int *check,
    const __grid_constant__ GeomSrc geo, float *__restrict__ g_clear, int *queue)
{
    constexpr int NLM = (L + 1) * (L + 1);
    constexpr int ASTR = AStride<NLM>::value;
    constexpr int KPL = (NLM + 31) / 32;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    pdl_enter();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    // one site: no CTA-wide synchronisation in this kernel
    auto site_body = [&](const int row) {
        unsigned char *wbase = smem_raw + (size_t)warp * warp_smem;
        const int nmax = P.n_max, dim = P.dim, nout = nmax * NLM;
        T *Rs = reinterpret_cast<T *>(wbase);
        T *As = Rs + 32 * AMB;
        GroupStage *stage = reinterpret_cast<GroupStage *>(As);
        T *cs = As + fwd_area<T>(ASTR, dim, CMP ? P.dim_out : 0);

        const int site = sites ? sites[row] : row;
        const int64_t kb = start[site], ke = start[site + 1];
        // the central atom's weights, loaded now and added to l = 0 of its own species block at the end
        // (a site with no list entries at all, which the list's capacity clamp can leave, has none)
        const int s_self = ke > kb ? nsp[kb] - 1 : -1;
        const bool has_central = s_self >= 0 && s_self < P.n_species && lane < P.alpha_max[s_self];
        const T cen = has_central ? central[P.n_off[s_self] + lane] : (T)0;
        if (geo.pos) {
            // this step's pair geometry from the primitive positions (what the neighbor module's
            // geometry pass would write), read back by the compaction through L2-coherent loads
            const StructDesc &S = static_cast<const StructDesc *>(geo.sd)[geo.site_struct[site]];
            double pi[3];
            sc_position(S, geo.pos, site - S.atom_off + 1, pi);
            for (int64_t k = kb + lane; k < ke; k += 32) {
                double dist[3] = {0.0, 0.0, 0.0}, d = 0.0;
                if (k > kb) {
                    double pj[3];
                    sc_position(S, geo.pos, geo.list[k], pj);
                    get_distance_dev(pi, pj, S, dist, &d);
                }
                geo.rjs_out[k] = d;
                geo.xyz_out[3 * k] = dist[0];
                geo.xyz_out[3 * k + 1] = dist[1];
                geo.xyz_out[3 * k + 2] = dist[2];
            }
            __threadfence_block();
            __syncwarp();
        }
        for (int s = 0; s < P.n_species; ++s) {
            T acc[KPL][AMB];
    #pragma unroll
            for (int j = 0; j < KPL; ++j)
    #pragma unroll
                for (int n = 0; n < AMB; ++n) acc[j][n] = 0;
            int64_t scan = kb + 1;
            while (scan < ke) {
                const int cnt = compact_stage(P, scan, ke, rjs, xyz, nsp, s, stage, lane);
                if (cnt == 0) break;
                double rd = 1.0, xd = 0.0, yd = 0.0, zd = 1.0;
                if (lane < cnt) {
                    rd = stage->r[lane];
                    xd = stage->x[lane];
                    yd = stage->y[lane];
                    zd = stage->z[lane];
                }
                __syncwarp();  // the angular rows below overwrite the stage
                if (lane < cnt) {
                    const T r = (T)rd, ir = (T)1 / r;
                    const T ux = (T)xd * ir, uy = (T)yd * ir, uz = (T)zd * ir;
                    T R[AMB], dR[AMB];
                    radial_values<T, AMB, false>(P, s, rd, xq, tq, rtab, R, dR);
                    T *Rrow = Rs + lane * AMB;
    #pragma unroll
                    for (int n = 0; n < AMB; ++n) Rrow[n] = R[n];
                    const T st = (T)P.sigma_t[s] + (T)P.sigma_t_scaling[s] * r;
                    T f[L + 2];
                    bessel_ratios_fixed<T, L>(r * r / (st * st), f);
                    T *Arow = As + lane * ASTR;
                    ylm_all<T, L, false>(Yc, ux, uy, uz, [&](int kk, int l, T y, T, T, T) { Arow[kk] = f[l] * y; });
                }
                __syncwarp();
                for (int p = 0; p < cnt; ++p) {
                    T rv[AMB];
                    load_vec<T, AMB>(Rs + p * AMB, rv);
    #pragma unroll
                    for (int j = 0; j < KPL; ++j) {
                        const int kk = lane + 32 * j;
                        if (kk < NLM) axpy_row<T, AMB>(acc[j], rv, As[p * ASTR + kk]);
                    }
                }
                __syncwarp();
            }
            const int off = P.n_off[s], am = P.alpha_max[s];
    #pragma unroll
            for (int j = 0; j < KPL; ++j) {
                const int kk = lane + 32 * j;
                if (kk < NLM) {
    #pragma unroll
                    for (int n = 0; n < AMB; ++n)
                        if (n < am) cs[(off + n) * NLM + kk] = acc[j][n];
                }
            }
        }
        __syncwarp();
        // central atom on l = 0 of its own species block
        if (has_central) cs[(P.n_off[s_self] + lane) * NLM] += cen;
        __syncwarp();
        warp_copy_row<T>(c_out + (size_t)row * nout, cs, nout, lane);
        // power spectrum into the (now free) angular area: lane owns the (n, n') pairs
        // pp = lane + 32 i (n-major, n <= n') and every l, component d = pp (L + 1) + l
        T *ps = As;
        T part = 0;
        const int npair = nmax * (nmax + 1) / 2;
        for (int pp = lane; pp < npair; pp += 32) {
            int n = 0, rem = pp;
            while (rem >= nmax - n) {
                rem -= nmax - n;
                ++n;
            }
            const int np = n + rem;
            const T *a = cs + n * NLM, *b = cs + np * NLM;
            const T sc = (n == np) ? (T)1 : (T)1.4142135623730951;
    #pragma unroll
            for (int l = 0; l <= L; ++l) {
                T acc = 0;
    #pragma unroll
                for (int kk = l * l; kk < (l + 1) * (l + 1); ++kk) acc += a[kk] * b[kk];
                const T v = acc * sc;
                ps[pp * (L + 1) + l] = v;
                part += v * v;
            }
        }
        // with compression the descriptor is P p / |P p|: P p in the area after the power spectrum,
        // each row summed in the order its entries were given
        const T *qsrc = ps;
        int dq = dim;
        if constexpr (CMP) {
            __syncwarp();
            T *pcs = ps + dim;
            const T *val = cmp_vals<T>(P, true);
            part = 0;
            for (int r = lane; r < P.dim_out; r += 32) {
                T acc = 0;
                for (int e = P.cmp_row[r]; e < P.cmp_row[r + 1]; ++e) acc += val[e] * ps[P.cmp_rcol[e]];
                pcs[r] = acc;
                part += acc * acc;
            }
            qsrc = pcs;
            dq = P.dim_out;
        }
    #pragma unroll
        for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
        const T nrm = t_sqrt<T>(part);
        const T inv = nrm > (T)0 ? (T)1 / nrm : (T)0;
        __syncwarp();
        // the row of the dE/dq accumulator the GAP kernel adds into (saves a separate clear)
        if constexpr (std::is_same<T, float>::value) {
            const bool vec = (q_ld & 3) == 0 && (reinterpret_cast<uintptr_t>(q_out) & 15) == 0 &&
                             (reinterpret_cast<uintptr_t>(g_clear) & 15) == 0 &&
                             (!SPLIT || ((reinterpret_cast<uintptr_t>(q_hi) | reinterpret_cast<uintptr_t>(q_lo)) & 7) == 0);
            // four consecutive components per lane: 16-byte q and dE/dq stores, 8-byte bf16 halves
            for (int d = 4 * lane; vec && d < q_ld; d += 128) {
                float v[4];
    #pragma unroll
                for (int e = 0; e < 4; ++e) v[e] = d + e < dq ? (float)(qsrc[d + e] * inv) : 0.0f;
                const size_t o = (size_t)row * q_ld + d;
                *reinterpret_cast<float4 *>(q_out + o) = make_float4(v[0], v[1], v[2], v[3]);
                if (g_clear) *reinterpret_cast<float4 *>(g_clear + o) = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                if (SPLIT) {
                    const __nv_bfloat162 h01 = __floats2bfloat162_rn(v[0], v[1]), h23 = __floats2bfloat162_rn(v[2], v[3]);
                    const float2 f01 = __bfloat1622float2(h01), f23 = __bfloat1622float2(h23);
                    const __nv_bfloat162 l01 = __floats2bfloat162_rn(v[0] - f01.x, v[1] - f01.y);
                    const __nv_bfloat162 l23 = __floats2bfloat162_rn(v[2] - f23.x, v[3] - f23.y);
                    *reinterpret_cast<uint2 *>(q_hi + o) = make_uint2(*reinterpret_cast<const unsigned *>(&h01),
                                                                      *reinterpret_cast<const unsigned *>(&h23));
                    *reinterpret_cast<uint2 *>(q_lo + o) = make_uint2(*reinterpret_cast<const unsigned *>(&l01),
                                                                      *reinterpret_cast<const unsigned *>(&l23));
                }
            }
            if (vec) {
                if (lane == 0) norm_out[row] = nrm;
                return;
            }
        }
        if (g_clear)
            for (int d = lane; d < q_ld; d += 32) g_clear[(size_t)row * q_ld + d] = 0.0f;
        for (int d = lane; d < q_ld; d += 32) {
            const T qv = d < dq ? qsrc[d] * inv : (T)0;
            q_out[(size_t)row * q_ld + d] = qv;
            if (SPLIT) {
                const float qf = (float)qv;
                const __nv_bfloat16 h = __float2bfloat16_rn(qf);
                q_hi[(size_t)row * q_ld + d] = h;
                q_lo[(size_t)row * q_ld + d] = __float2bfloat16_rn(qf - __bfloat162float(h));
            }
        }
        if (lane == 0) norm_out[row] = nrm;
    };
    if constexpr (!PERSIST) {
        const int row = blockIdx.x * nw + warp;
        if (row < n_rows) site_body(row);
    } else {
        // persistent form: the warp takes sites from the queue until it runs dry
        for (;;) {
            int r = 0;
            if (lane == 0) r = atomicAdd(queue, 1);
            const int row = __shfl_sync(0xffffffffu, r, 0);
            if (row >= n_rows) break;
            site_body(row);
            __syncwarp();
        }
    }
}

// ----------------------------------------------------------------------------- adjoint

// virial[st] += the symmetric tensor (xx yy zz xy xz yz) in v6 (column-major 3x3).
__device__ __forceinline__ void add_virial6(double *virial, int st, const double *v6)
{
    double *V = virial + 9 * (size_t)st;
    atomicAdd(V + 0, v6[0]);
    atomicAdd(V + 4, v6[1]);
    atomicAdd(V + 8, v6[2]);
    atomicAdd(V + 3, v6[3]);
    atomicAdd(V + 1, v6[3]);
    atomicAdd(V + 6, v6[4]);
    atomicAdd(V + 2, v6[4]);
    atomicAdd(V + 7, v6[5]);
    atomicAdd(V + 5, v6[5]);
}

// Elements of the c area of the adjoint: c [n_max][NLM] rounded up to 4, and at least the
// lanes' force/virial partials [32][9] (double) that reuse it after the prologue.
template <class T> __host__ __device__ constexpr int bwd_c_elems(int nout)
{
    return ((nout + 3) / 4 * 4) > (int)(32 * 9 * sizeof(double) / sizeof(T)) ? (nout + 3) / 4 * 4
                                                                               : (int)(32 * 9 * sizeof(double) / sizeof(T));
}

// Pitch (elements) of one M_l block of the adjoint: n_max rows of n_species * AMB columns, rounded
// to an odd number of 16-byte vectors, so lanes that read blocks of different l with 16-byte loads
// fall in different banks.
template <class T> __host__ __device__ constexpr int bwd_m_pitch(int nmax, int mp)
{
    return (((nmax * mp + (int)(16 / sizeof(T)) - 1) / (int)(16 / sizeof(T))) | 1) * (int)(16 / sizeof(T));
}

// Minimum resident CTAs of 4 warps asked of the compiler. The one-site adjoint asks for 1 (its
// natural register count; forcing 6 CTAs on the FP32 kernel spilled and ran slower). The site loop
// of the persistent form otherwise keeps loop-invariant values in registers (168 instead of 112 in
// FP32): it asks for 4 (at most 128 registers) in FP32 and 2 in FP64, where 128 spills.
template <class T, bool PERSIST> struct BwdMinCtas {
    static constexpr int value = PERSIST ? (std::is_same<T, float>::value ? 4 : 2) : 1;
};

// Shared memory of one warp: the group's staged geometry (GroupStage), c [n_max][NLM] (then the lanes'
// force/virial partials), M [L+1][MSP] with M_l[n][n'] = (2 if n == n' else sqrt 2) h[n n' l] in
// padded species columns (MSP = bwd_m_pitch), Gc [n_species][NLM][AMB] (dE/dc per species block,
// zero beyond alpha_max), f_l / df_l of each lane's pair [2][L+1][32]; h [dim] occupies the area
// of Gc and f_l / df_l (grown to dim when smaller) until M is formed. After the warps, the CTA's
// virial partials [kWarpsPerCta][6] and structure ids [kWarpsPerCta].
template <class T, class GT, int L, int AMB, bool PERSIST, bool CMP>
__global__ void __launch_bounds__(32 * kWarpsPerCta, BwdMinCtas<T, PERSIST>::value) k_soap_bwd_warp(
    const __grid_constant__ SoapParams P, const __grid_constant__ YlmConst Yc, const T *__restrict__ xq,
    const T *__restrict__ tq, const float4 *__restrict__ rtab, const int *__restrict__ sites, int n_rows,
    const int64_t *__restrict__ start, const double *__restrict__ rjs, const double *__restrict__ xyz,
    const int *__restrict__ nsp, const int *__restrict__ jatom, const int *__restrict__ site_struct,
    const T *__restrict__ c_in, const T *__restrict__ q_in, int q_ld, const T *__restrict__ norm_in,
    const GT *__restrict__ g_in, int g_ld, double *__restrict__ forces, double *__restrict__ virial,
    int warp_smem, int n_atoms, int *check, double *__restrict__ pair_der, const double *__restrict__ gate,
    int *queue)
{
    constexpr int NLM = (L + 1) * (L + 1);
    constexpr int KPL = (NLM + 31) / 32;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    pdl_enter();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    double *vpart = reinterpret_cast<double *>(smem_raw + (size_t)nw * warp_smem);
    int *vstruct = reinterpret_cast<int *>(vpart + 6 * kWarpsPerCta);
    if (lane == 0) {
        vstruct[warp] = -1;
#pragma unroll
        for (int c = 0; c < 6; ++c) vpart[6 * warp + c] = 0.0;
    }
    __syncwarp();
    auto site_body = [&](const int row) {
        // pair-derivative mode: a site whose gate is 0 writes nothing (its pairs stay zero)
        if (pair_der && gate && gate[sites ? sites[row] : row] == 0.0) return;
        unsigned char *wbase = smem_raw + (size_t)warp * warp_smem;
        const int nmax = P.n_max, dim = P.dim, nout = nmax * NLM;
        GroupStage *stage = reinterpret_cast<GroupStage *>(wbase);
        T *cs = reinterpret_cast<T *>(wbase + sizeof(GroupStage));
        const int MP = P.n_species * AMB, MSP = bwd_m_pitch<T>(nmax, MP);
        T *Ms = cs + bwd_c_elems<T>(nout);
        T *Gc = Ms + (L + 1) * MSP;
        T *fdf = Gc + P.n_species * NLM * AMB;  // [2][L+1][32]: f_l, df_l of each lane's pair
        T *hb = Gc;                             // h [dim] until M is formed

        const int site = sites ? sites[row] : row;
        const int my_struct = site_struct ? site_struct[site] : 0;
        const int64_t kb = start[site], ke = start[site + 1];
        // c arrives asynchronously (it is first read when Gc is formed)
        warp_copy_row_async<T>(cs, c_in + (size_t)row * nout, nout, lane);
        const T nrm = norm_in[row];
        const T *qrow = q_in + (size_t)row * q_ld;
        const GT *grow = g_in + (size_t)row * g_ld;
        // h = dE/dp = (g - q (q.g)) / |p| into shared memory: independent coalesced loads (the rows
        // were just read for q.g), so the M entries below are formed at shared-memory latency. With
        // compression q and g have dim_out entries and this is dE/d(P p), placed after h, and h = P^T
        // of it, each column summed in the order its entries were given
        if constexpr (!CMP) {
            T qg = warp_dot_part<T, GT>(qrow, grow, dim, lane);
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) qg += __shfl_xor_sync(0xffffffffu, qg, o);
            const T inv = nrm > (T)0 ? (T)1 / nrm : (T)0;
            for (int d = lane; d < dim; d += 32) hb[d] = ((T)grow[d] - qrow[d] * qg) * inv;
        } else {
            const int dq = P.dim_out;
            T qg = warp_dot_part<T, GT>(qrow, grow, dq, lane);
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) qg += __shfl_xor_sync(0xffffffffu, qg, o);
            const T inv = nrm > (T)0 ? (T)1 / nrm : (T)0;
            T *hc = hb + dim;
            for (int d = lane; d < dq; d += 32) hc[d] = ((T)grow[d] - qrow[d] * qg) * inv;
            __syncwarp();
            const T *val = cmp_vals<T>(P, false);
            for (int j = lane; j < dim; j += 32) {
                T acc = 0;
                for (int e = P.cmp_col[j]; e < P.cmp_col[j + 1]; ++e) acc += val[e] * hc[P.cmp_crow[e]];
                hb[j] = acc;
            }
        }
        __syncwarp();
        // M_l[n][n'] = (2 if n == n' else sqrt 2) h[n n' l], h = dE/dp = (g - q (q.g)) / |p|, stored
        // as rows n' of n_species blocks of AMB columns (radial index n_off[s] + a in column
        // s AMB + a; columns beyond alpha_max stay zero). M_l is symmetric, so the slice of row n'
        // in block s holds M_l[n_off[s] + a][n'] for every a.
        if (nmax != MP) {
            for (int o = lane; o < (L + 1) * MSP; o += 32) Ms[o] = (T)0;
            __syncwarp();
        }
        {
            // lane -> (sub, l); it visits the pairs pp = sub + PPW t (n-major, n <= n'), component
            // d = pp (L + 1) + l, with (n, n') advanced incrementally
            constexpr int PPW = 32 / (L + 1);
            const int sub = lane / (L + 1), l = lane - sub * (L + 1);
            const int npair = nmax * (nmax + 1) / 2;
            int n = 0, rem = sub;
            while (n < nmax && rem >= nmax - n) {
                rem -= nmax - n;
                ++n;
            }
            for (int pp = sub; sub < PPW && pp < npair; pp += PPW) {
                const int np = n + rem, d = pp * (L + 1) + l;
                const T hv = hb[d];
                const T mv = (n == np) ? (T)2 * hv : (T)1.4142135623730951 * hv;
                int sn = 0, snp = 0;  // species blocks of n and n'
                for (int s = 1; s < P.n_species; ++s) {
                    if (n >= P.n_off[s]) sn = s;
                    if (np >= P.n_off[s]) snp = s;
                }
                const int cn = sn * AMB + n - P.n_off[sn], cnp = snp * AMB + np - P.n_off[snp];
                Ms[l * MSP + np * MP + cn] = mv;
                Ms[l * MSP + n * MP + cnp] = mv;
                rem += PPW;
                while (n < nmax && rem >= nmax - n) {
                    rem -= nmax - n;
                    ++n;
                }
            }
        }
        cp_async_wait_all();
        __syncwarp();
        // Gc[s][lm][a] = sum_n' M_l[n_off[s] + a][n'] c[n'][lm]: one c value and one padded M row
        // slice per n', accumulated with row FMAs
#pragma unroll
        for (int j = 0; j < KPL; ++j) {
            const int kk = lane + 32 * j;
            if (kk < NLM) {
                const int l = (int)sqrtf((float)kk);
                const T *Ml = Ms + l * MSP;
                for (int s = 0; s < P.n_species; ++s) {
                    T acc[AMB];
#pragma unroll
                    for (int a = 0; a < AMB; ++a) acc[a] = (T)0;
                    const T *mcol = Ml + s * AMB;
                    for (int np = 0; np < nmax; ++np) {
                        T mr[AMB];
                        load_vec<T, AMB>(mcol + np * MP, mr);
                        axpy_row<T, AMB>(acc, mr, cs[np * NLM + kk]);
                    }
                    store_vec<T, AMB>(Gc + (s * NLM + kk) * AMB, acc);
                }
            }
        }
        __syncwarp();
        // per-lane force/virial partials, kept out of registers during the pair loop; they reuse
        // the area of c, which is dead once Gc is formed
        double *vl = reinterpret_cast<double *>(cs) + lane * 9;
#pragma unroll
        for (int i = 0; i < 9; ++i) vl[i] = 0.0;

        int64_t scan = kb + 1;
        while (scan < ke) {
            const int cnt = compact_stage(P, scan, ke, rjs, xyz, nsp, -1, stage, lane);
            if (cnt == 0) break;
            if (lane < cnt) {
                const int64_t k = stage->k[lane];
                const int s = stage->s[lane];
                const double xd0 = stage->x[lane], xd1 = stage->y[lane], xd2 = stage->z[lane];
                const double rd = stage->r[lane];
                const T r = (T)rd;
                const T ir = (T)1 / r;
                const T u0 = (T)xd0 * ir, u1 = (T)xd1 * ir, u2 = (T)xd2 * ir;
                T R[AMB], dR[AMB];
                radial_values<T, AMB, true>(P, s, rd, xq, tq, rtab, R, dR);
                const T sts = (T)P.sigma_t_scaling[s];
                const T st = (T)P.sigma_t[s] + sts * r;
                const T kap = r * r / (st * st);
                const T dkap = (T)2 * r / (st * st) - (T)2 * r * r * sts / (st * st * st);
                {
                    T f[L + 2];
                    bessel_ratios_fixed<T, L>(kap, f);
                    const T ikap = kap > (T)0 ? (T)1 / kap : (T)0;
#pragma unroll
                    for (int l = 0; l <= L; ++l) {
                        fdf[l * 32 + lane] = f[l];
                        fdf[(L + 1 + l) * 32 + lane] = (f[l + 1] + (T)l * ikap * f[l] - f[l] * f[1]) * dkap;
                    }
                }
                T w[3];
                pair_adjoint<T, L, AMB>(Yc, u0, u1, u2, ir, fdf + lane, fdf + (L + 1) * 32 + lane, Gc + s * NLM * AMB,
                                        R, dR, w);
                const T w0 = w[0], w1 = w[1], w2 = w[2];
                // w = dE_i/dr_ij: force -w on the neighbor, +w on the site (its self slot)
                const double f0 = -(double)w0, f1 = -(double)w1, f2 = -(double)w2;
                if (pair_der) {
                    pair_der[3 * k] = (double)w0;
                    pair_der[3 * k + 1] = (double)w1;
                    pair_der[3 * k + 2] = (double)w2;
                } else {
                    const int j = jatom[k];
                    if (j >= 0 && j < n_atoms) {
                        atomicAdd(forces + 3 * (size_t)j, f0);
                        atomicAdd(forces + 3 * (size_t)j + 1, f1);
                        atomicAdd(forces + 3 * (size_t)j + 2, f2);
                    } else {
                        check_fail(check, kCheckBwdAtom, k, j);
                    }
                }
                vl[0] -= f0;
                vl[1] -= f1;
                vl[2] -= f2;
                vl[3] += f0 * xd0;
                vl[4] += f1 * xd1;
                vl[5] += f2 * xd2;
                vl[6] += 0.5 * (f0 * xd1 + f1 * xd0);
                vl[7] += 0.5 * (f0 * xd2 + f2 * xd0);
                vl[8] += 0.5 * (f1 * xd2 + f2 * xd1);
            }
            __syncwarp();
        }
        // component c < 9 of the site's sum: lane c adds column c of the 32 lanes' rows in lane
        // order (components 0-2: the self force; 3-8: the virial)
        __syncwarp();  // every lane's row is complete (also when the site had no pairs)
        double csum = 0.0;
        if (lane < 9) {
            const double *col = reinterpret_cast<const double *>(cs) + lane;
#pragma unroll 8
            for (int q = 0; q < 32; ++q) csum += col[9 * q];
        }
        if (lane < 3 && ke > kb) {  // the self entry (absent only in a list the capacity clamp cut)
            const double fv = csum;
            if (pair_der) {
                pair_der[3 * kb + lane] = -fv;  // dq_i/dr_i = -sum_j dq_i/dr_j
            } else {
                const int js = jatom[kb];
                if (js >= 0 && js < n_atoms)
                    atomicAdd(forces + 3 * (size_t)js + lane, fv);
                else if (lane == 0)
                    check_fail(check, kCheckSelfAtom, kb, js);
            }
        }
        // the site's virial into the warp's partial, flushed to its structure when the next site
        // belongs to another one
        if (!pair_der) {
            if (lane == 0) {
                const int cur = vstruct[warp];
                if (cur != my_struct) {
                    if (cur >= 0) add_virial6(virial, cur, vpart + 6 * warp);
                    vstruct[warp] = my_struct;
#pragma unroll
                    for (int c = 0; c < 6; ++c) vpart[6 * warp + c] = 0.0;
                }
            }
            __syncwarp();
            if (lane >= 3 && lane < 9) vpart[6 * warp + lane - 3] += csum;
        }
    };
    if constexpr (!PERSIST) {
        const int row = blockIdx.x * nw + warp;
        if (row < n_rows) site_body(row);
    } else {
        // persistent form: the warp takes sites from the queue until it runs dry
        for (;;) {
            int r = 0;
            if (lane == 0) r = atomicAdd(queue, 1);
            const int row = __shfl_sync(0xffffffffu, r, 0);
            if (row >= n_rows) break;
            site_body(row);
            __syncwarp();
        }
    }
    if (pair_der) return;  // uniform over the grid: no virial in pair-derivative mode
    // virial (xx yy zz xy xz yz -> column-major 3x3): one set of atomics per CTA when its warps'
    // last structures agree, else one per warp
    __syncthreads();
    if (warp == 0) {
        const int st0 = vstruct[0];
        bool same = true;
        for (int w = 1; w < nw; ++w)
            if (vstruct[w] >= 0 && vstruct[w] != st0) same = false;
        // component c of (xx yy zz xy xz yz) -> matrix indices (a, b)
        auto ia = [](int c) { return c < 3 ? c : (c == 5 ? 1 : 0); };
        auto ib = [](int c) { return c < 3 ? c : (c == 3 ? 1 : 2); };
        if (same) {
            if (lane < 6 && st0 >= 0) {
                double v = 0;
                for (int w = 0; w < nw; ++w) v += vpart[6 * w + lane];
                const int a = ia(lane), c = ib(lane);
                atomicAdd(virial + 9 * (size_t)st0 + a + 3 * c, v);
                if (a != c) atomicAdd(virial + 9 * (size_t)st0 + c + 3 * a, v);
            }
        } else if (lane < 6 * nw) {
            const int w = lane / 6, c6 = lane - 6 * w;
            const int st = vstruct[w];
            if (st >= 0) {
                const int a = ia(c6), c = ib(c6);
                atomicAdd(virial + 9 * (size_t)st + a + 3 * c, vpart[6 * w + c6]);
                if (a != c) atomicAdd(virial + 9 * (size_t)st + c + 3 * a, vpart[6 * w + c6]);
            }
        }
    }
}

// ----------------------------------------------------------------------------- launchers

inline size_t fwd_warp_bytes(const SoapParams &P, size_t tsz, int astr, int amb)
{
    const size_t nlm = (size_t)(P.l_max + 1) * (P.l_max + 1);
    const int dc = P.cmp_row ? P.dim_out : 0;
    const size_t area =
        tsz == 8 ? (size_t)fwd_area<double>(astr, P.dim, dc) : (size_t)fwd_area<float>(astr, P.dim, dc);
    return (tsz * (32 * (size_t)amb + area + (size_t)P.n_max * nlm) + 15) / 16 * 16;
}

template <class T> inline size_t bwd_warp_bytes(const SoapParams &P, int amb)
{
    const size_t nlm = (size_t)(P.l_max + 1) * (P.l_max + 1);
    const int nout = P.n_max * (int)nlm;
    const size_t ms = (size_t)(P.l_max + 1) * bwd_m_pitch<T>(P.n_max, P.n_species * amb);
    const size_t fdf = 2 * (size_t)(P.l_max + 1) * 32;
    // Gc + f/df, or h (and the compressed dE/dp after it)
    const size_t gf = std::max<size_t>((size_t)P.n_species * nlm * amb + fdf,
                                       (size_t)P.dim + (P.cmp_row ? (size_t)P.dim_out : 0));
    static_assert(sizeof(GroupStage) % 16 == 0, "the adjoint's arrays after the stage stay 16-byte aligned");
    return sizeof(GroupStage) + (sizeof(T) * ((size_t)bwd_c_elems<T>(nout) + ms + gf) + 15) / 16 * 16;
}

constexpr size_t kMaxDynSmem = 227 * 1024;

// Autotuner key of a descriptor launch (sites per CTA): kernel, precision, l_max, radial block,
// bf16 split, and the row count rounded up to a power of two.
inline std::string warps_key(const char *kind, bool f64, int L, int amb, bool split, int n_rows, bool cmp)
{
    int b = 1;
    while (b < n_rows) b <<= 1;
    char k[96];
    std::snprintf(k, sizeof(k), "soap_%s/%s/l%d/a%d/s%d/rows%d%s", kind, f64 ? "f64" : "f32", L, amb, (int)split, b,
                  cmp ? "/cmp" : "");
    return k;
}

inline std::vector<int> warp_candidates(int nw_max)
{
    std::vector<int> c;
    for (int v = 1; v <= nw_max; v *= 2) c.push_back(v);
    if (c.back() != nw_max) c.push_back(nw_max);
    return c;
}

// CTAs of a descriptor launch: one per nw rows, or in the persistent form no more than can be
// resident on the device at once (the warps loop over the queue). The persistent form is the
// default in FP32 (as fast as one site per warp on a uniform system, and it balances uneven
// batches); FP64 defaults to one site per warp (its site loop needs 182 registers: 198 against
// 170 us for the 4096-atom adjoint).
inline int site_grid(const void *kern, int nw, size_t smem, int n_rows, bool persistent)
{
    const int g = (n_rows + nw - 1) / nw;
    if (!persistent) return g;
    static std::mutex mu;
    static std::map<std::tuple<const void *, int, size_t, int>, int> cache;
    int dev = 0;
    cudaGetDevice(&dev);
    const auto key = std::make_tuple(kern, nw, smem, dev);
    int cap;
    {
        std::lock_guard<std::mutex> lock(mu);
        auto it = cache.find(key);
        if (it == cache.end()) {
            int nb = 0, sms = 0;
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, 32 * nw, smem);
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
            it = cache.emplace(key, std::max(1, nb * sms)).first;
        }
        cap = it->second;
    }
    return std::min(g, cap);
}

template <class T> inline const T *soap_tab(const DevBuf &d64, const DevBuf &d32)
{
    return std::is_same<T, double>::value ? (const T *)d64.ptr : (const T *)d32.ptr;
}

template <class T, bool SPLIT, bool CMP, int L, int AMB>
int launch_fwd_l(tgap_context *ctx, const DeviceSoap &ds, const PairView &pv, const int *d_sites, int n_rows,
                 SoapOut &o)
{
    constexpr int NLM = (L + 1) * (L + 1);
    const size_t wb = fwd_warp_bytes(ds.p, sizeof(T), AStride<NLM>::value, AMB);
    const int nw_max = (int)std::min<size_t>(kWarpsPerCta, kMaxDynSmem / wb);
    if (nw_max < 1) return set_error(ctx, TGAP_ERR_HYPERS, "descriptor forward needs %zu bytes of shared memory", wb);
    const bool f64 = std::is_same<T, double>::value;
    const std::string key = warps_key("fwd", f64, L, AMB, SPLIT, n_rows, CMP);
    const int nw = tuned(ctx, key, f64 ? "soap_forward_f64" : "soap_forward_f32", warp_candidates(nw_max), nw_max);
    const bool persist =
        pv.queue && tuned(ctx, key + "/persist",
                          f64 ? "soap_forward_f64" : "soap_forward_f32", {0, 1}, f64 ? 0 : 1);
    const size_t sm = wb * nw;
    auto kern = persist ? k_soap_fwd_warp<T, L, AMB, SPLIT, true, CMP> : k_soap_fwd_warp<T, L, AMB, SPLIT, false, CMP>;
    TGAP_CUDA(ctx, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    const int grid = site_grid((const void *)kern, nw, sm, n_rows, persist);
    TGAP_CUDA(ctx, launch_pdl(kern, dim3(grid), dim3(32 * nw), sm, ctx->stream, ds.p, ylm_host_constants(),
                              soap_tab<T>(ds.xq, ds.xq32), soap_tab<T>(ds.tq, ds.tq32), ds.rtab.as<float4>(),
                              soap_tab<T>(ds.central, ds.central32), d_sites, n_rows, pv.start, pv.rjs, pv.xyz,
                              pv.species, (T *)o.c, (T *)o.q, o.q_ld, (T *)o.norm, o.q_hi, o.q_lo, (int)wb, pv.check,
                              pv.geo, o.g_clear, persist ? pv.queue : nullptr));
    TGAP_LAUNCH_CHECK(ctx);
    return TGAP_OK;
}

template <class T, class GT, bool CMP, int L, int AMB>
int launch_bwd_l(tgap_context *ctx, const DeviceSoap &ds, const PairView &pv, const int *d_sites, int n_rows,
                 const SoapOut &o, const void *d_g, int g_ld, const int *site_struct, double *d_forces,
                 double *d_virial)
{
    const size_t wb = bwd_warp_bytes<T>(ds.p, AMB);
    const size_t tail = kWarpsPerCta * (6 * sizeof(double) + sizeof(int));
    const int nw_max = (int)std::min<size_t>(kWarpsPerCta, (kMaxDynSmem - tail) / wb);
    if (nw_max < 1) return set_error(ctx, TGAP_ERR_HYPERS, "descriptor adjoint needs %zu bytes of shared memory", wb);
    const bool f64 = std::is_same<T, double>::value;
    const std::string key = warps_key("bwd", f64, L, AMB, false, n_rows, CMP);
    const int nw = tuned(ctx, key, f64 ? "soap_backward_f64" : "soap_backward_f32", warp_candidates(nw_max), nw_max);
    const bool persist =
        pv.queue && tuned(ctx, key + "/persist",
                          f64 ? "soap_backward_f64" : "soap_backward_f32", {0, 1}, f64 ? 0 : 1);
    const size_t sm = wb * nw + tail;
    auto kern = persist ? k_soap_bwd_warp<T, GT, L, AMB, true, CMP> : k_soap_bwd_warp<T, GT, L, AMB, false, CMP>;
    TGAP_CUDA(ctx, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    const int grid = site_grid((const void *)kern, nw, sm, n_rows, persist);
    TGAP_CUDA(ctx, launch_pdl(kern, dim3(grid), dim3(32 * nw), sm, ctx->stream, ds.p, ylm_host_constants(),
                              soap_tab<T>(ds.xq, ds.xq32), soap_tab<T>(ds.tq, ds.tq32), ds.rtab.as<float4>(), d_sites,
                              n_rows, pv.start, pv.rjs, pv.xyz, pv.species, pv.jatom, site_struct, (const T *)o.c,
                              (const T *)o.q, o.q_ld, (const T *)o.norm, (const GT *)d_g, g_ld, d_forces, d_virial,
                              (int)wb, pv.n_atoms, pv.check, pv.pair_der, pv.gate, persist ? pv.queue : nullptr));
    TGAP_LAUNCH_CHECK(ctx);
    return TGAP_OK;
}

#define TGAP_FOR_EACH_L(X) X(0) X(1) X(2) X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10)
static_assert(kMaxL == 10, "TGAP_FOR_EACH_L lists l_max = 0..10");
static_assert(kMaxAlpha <= 16, "radial blocks are instantiated for alpha_max <= 8 and <= 16");

template <class T, bool SPLIT, bool CMP, int AMB>
int launch_fwd_amb(tgap_context *ctx, const DeviceSoap &ds, const PairView &pv, const int *d_sites, int n_rows,
                   SoapOut &o)
{
    switch (ds.p.l_max) {
#define TGAP_CASE(l) \
    case l: return launch_fwd_l<T, SPLIT, CMP, l, AMB>(ctx, ds, pv, d_sites, n_rows, o);
        TGAP_FOR_EACH_L(TGAP_CASE)
#undef TGAP_CASE
    }
    return set_error(ctx, TGAP_ERR_HYPERS, "l_max %d out of range", ds.p.l_max);
}

template <class T, class GT, bool CMP, int AMB>
int launch_bwd_amb(tgap_context *ctx, const DeviceSoap &ds, const PairView &pv, const int *d_sites, int n_rows,
                   const SoapOut &o, const void *d_g, int g_ld, const int *site_struct, double *d_forces,
                   double *d_virial)
{
    switch (ds.p.l_max) {
#define TGAP_CASE(l)                                                                                          \
    case l:                                                                                                   \
        return launch_bwd_l<T, GT, CMP, l, AMB>(ctx, ds, pv, d_sites, n_rows, o, d_g, g_ld, site_struct, \
                                                d_forces, d_virial);
        TGAP_FOR_EACH_L(TGAP_CASE)
#undef TGAP_CASE
    }
    return set_error(ctx, TGAP_ERR_HYPERS, "l_max %d out of range", ds.p.l_max);
}

// CMP: the model's descriptor is compressed (ds.p.cmp_row set); the compressed kernels are
// instantiated in translation units of their own.
template <class T, bool SPLIT, bool CMP>
int launch_fwd(tgap_context *ctx, const DeviceSoap &ds, const PairView &pv, const int *d_sites, int n_rows,
               SoapOut &o)
{
    if (ds.p.max_alpha <= 8) return launch_fwd_amb<T, SPLIT, CMP, 8>(ctx, ds, pv, d_sites, n_rows, o);
    return launch_fwd_amb<T, SPLIT, CMP, 16>(ctx, ds, pv, d_sites, n_rows, o);
}

template <class T, class GT, bool CMP>
int launch_bwd(tgap_context *ctx, const DeviceSoap &ds, const PairView &pv, const int *d_sites, int n_rows,
               const SoapOut &o, const void *d_g, int g_ld, const int *site_struct, double *d_forces,
               double *d_virial)
{
    if (ds.p.max_alpha <= 8)
        return launch_bwd_amb<T, GT, CMP, 8>(ctx, ds, pv, d_sites, n_rows, o, d_g, g_ld, site_struct, d_forces,
                                             d_virial);
    return launch_bwd_amb<T, GT, CMP, 16>(ctx, ds, pv, d_sites, n_rows, o, d_g, g_ld, site_struct, d_forces,
                                          d_virial);
}

}  // namespace tgap
